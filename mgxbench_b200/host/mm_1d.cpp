// mm_1d -- drop-in for MGXBench's 1D row-block executable (1D-row-block/mmb.cu), run on one GPU.
//
//   mm_1d <deviceId|auto> <matrix_size> <ABC libraries>
//
// Every emulated rank r owns rows [r*mi, (r+1)*mi) of A and C (mi = N / ranks,
// 1D-row-block/mmb.cu:312) and needs all of B; all ranks' block multiplies run on this device
// and no data moves between ranks, so the library letters select only the compute structure the
// reference uses for them (1D-row-block/mmb.cu:738-864):
//   B letter S, Y or X : C_r = 0, then C_r += A_r[:, chunk] * B_chunk for every K chunk of
//                        MM_PIPELINE_K_CHUNK (default 2048, rounded down to a multiple of 32);
//   any other B letter : one C_r = A_r * B.
// Output records are the reference's: the `mmb node=...` header (mmb.cu:302), the RESULT line
// (mmb.cu:937), the NUMERICAL VALIDATION block (mulmat_kernel.cu:298-319) and one
// BENCHMARK_RESULT line (mmb.cu:964-965); exit status 0 when valid, 2 otherwise (mmb.cu:1036).
// Keys this build adds come after the reference's keys on the same line.
#include "autotune.h"
#include "mm_common.h"

static int pipeline_k_chunk_from_env(int k)  // 1D-row-block/mmb.cu:109-128
{
    int chunk = 2048;
    const int requested = mm::env_int("MM_PIPELINE_K_CHUNK", 0);
    if (requested > 0) chunk = requested;
    if (chunk > k) chunk = k;
    if (chunk >= 32) chunk = (chunk / 32) * 32;
    return (chunk > 0) ? chunk : k;
}

static bool valid_library(char c)
{
    return c == 'M' || c == 'Y' || c == 'C' || c == 'X' || c == 'N' || c == 'S' || c == 'W';
}

int main(int argc, char *argv[])
{
    if (argc < 4) {
        fprintf(stderr,
                "Usage: %s <deviceId> <matrix_size> <ABC libraries>\n"
                "  M=MPI-SYNC, Y=MPI-ASYNC, C=CUDA-Aware MPI-SYNC, X=CUDA-Aware MPI-ASYNC, N=NCCL-SYNC, "
                "S=NVSHMEM-ASYNC, W=NVSHMEM-SYNC\n"
                "  Example: %s 0 8192 SNS\n",
                argv[0], argv[0]);
        return EXIT_FAILURE;
    }
    const int nRanks = mm::emulated_ranks();
    const int myRank = 0;
    int deviceId = atoi(argv[1]);
    if (strcmp(argv[1], "auto") == 0) deviceId = 0;  // one process: local rank 0
    const int matrix_size = atoi(argv[2]);

    char libs[4] = {0, 0, 0, 0};
    strncpy(libs, argv[3], 3);
    libs[3] = '\0';
    if (strlen(libs) != 3 || !valid_library(libs[0]) || !valid_library(libs[1]) || !valid_library(libs[2])) {
        fprintf(stderr, "Invalid communication string. Use exactly 3 characters from M, Y, C, X, N, S, W.\n");
        return EXIT_FAILURE;
    }
    if (matrix_size <= 0 || nRanks <= 0 || matrix_size % nRanks != 0) {
        fprintf(stderr, "matrix size %d must be positive and divisible by the %d emulated ranks\n", matrix_size,
                nRanks);
        return EXIT_FAILURE;
    }
    std::string input_name, form_name;
    const int input = mm::input_kind(&input_name);
    int form = mm::compute_form(&form_name);
    if (input < 0 || form < 0) {
        fprintf(stderr, "MGXBENCH_INPUT must be const|uniform|wide and MGXBENCH_FORM fp64|ozaki|crt|auto\n");
        return EXIT_FAILURE;
    }
    mm::cuda_or_die(cudaSetDevice(deviceId), "cudaSetDevice", EXIT_FAILURE);

    char name[256] = "localhost";
    gethostname(name, sizeof name - 1);
    cudaDeviceProp prop;
    mm::cuda_or_die(cudaGetDeviceProperties(&prop, deviceId), "cudaGetDeviceProperties", EXIT_FAILURE);
    printf("mmb node=%s device=%d:%s libraries=%s\n", name, deviceId, prop.name, libs);

    const int m = matrix_size, n = matrix_size, k = matrix_size;
    const int mi = matrix_size / nRanks;
    const int pipeline_k_chunk = pipeline_k_chunk_from_env(k);
    const char libB = libs[1];
    const bool chunked = (libB == 'S' || libB == 'Y' || libB == 'X');
    int splits = mm::env_int("MGXBENCH_SPLITS", 8);
    int ksplit = mm::env_int("MGXBENCH_KSPLIT", 1);
    int tile_m = mm::env_int("MGXBENCH_TILE_M", 128) == 64 ? 64 : 128;
    const bool batched = mm::env_int("MGXBENCH_BATCH", 1) != 0;
    const int launches = batched ? 1 : nRanks;
    const int rows_per_launch = batched ? m : mi;
    const bool autotuned = form == mm::kAuto;
    // the choice is made for the product one launch runs (its K chunk when chunked)
    mm::resolve_auto_form(&form, &splits, &ksplit, &tile_m, &form_name, rows_per_launch, n,
                          chunked ? std::min(pipeline_k_chunk, k) : k,
                          input == mm::kWide ? mm::env_int("MGXBENCH_EXP_RANGE", 20) : 0, EXIT_FAILURE, chunked);
    if (chunked) ksplit = 1;
    if (form == mm::kCrt && !autotuned)
        splits = mm::env_int("MGXBENCH_MODULI", mgx_crt_choose_moduli(chunked ? std::min(pipeline_k_chunk, k) : k, 1e-15));
    if (form == mm::kCrt) ksplit = 1;
    if (form != mm::kFp64 || chunked) tile_m = 128;  // the 64-row tile is an FP64 whole-multiply option
    if (ksplit < 0 || (ksplit == 0 && form != mm::kFp64)) ksplit = 1;  // 0: FP64 stream-K (64-row tiles)
    if (ksplit == 0) tile_m = 64;
    const int graph = mm::env_int("MGXBENCH_GRAPH", 0);
    printf("mmb one-GPU emulation: ranks=%d rows/rank=%d form=%s%s input=%s B-structure=%s", nRanks, mi,
           form_name.c_str(), mm::form_count(form, splits).c_str(), input_name.c_str(), chunked ? "K-chunked" : "single");
    if (chunked) printf(" K-chunk=%d", pipeline_k_chunk);
    printf(" launches=%s\n", batched ? "one for all ranks" : "one per rank");

    const size_t elems = (size_t)m * k;
    double *d_A = nullptr, *d_B = nullptr, *d_C = nullptr;
    mm::cuda_or_die(cudaMalloc(&d_A, elems * sizeof(double)), "cudaMalloc(A)", EXIT_FAILURE);
    mm::cuda_or_die(cudaMalloc(&d_B, (size_t)k * n * sizeof(double)), "cudaMalloc(B)", EXIT_FAILURE);
    mm::cuda_or_die(cudaMalloc(&d_C, (size_t)m * n * sizeof(double)), "cudaMalloc(C)", EXIT_FAILURE);

    const unsigned long long seed = mm::env_u64("MGXBENCH_SEED", 20240901ull);
    if (input == mm::kConst) {  // A[i,j] = 1, B[i,j] = 2 (1D-row-block/mmb.cu:586-591)
        mm::check_or_die(mgx_fill_matrix(d_A, m, k, k, 0, 1.0, 0, 0, nullptr), "fill A", EXIT_FAILURE);
        mm::check_or_die(mgx_fill_matrix(d_B, k, n, n, 0, 2.0, 0, 0, nullptr), "fill B", EXIT_FAILURE);
    } else {
        const int er = input == mm::kWide ? mm::env_int("MGXBENCH_EXP_RANGE", 20) : 0;
        mm::check_or_die(mgx_fill_matrix(d_A, m, k, k, input, 0.0, er, seed, nullptr), "fill A", EXIT_FAILURE);
        mm::check_or_die(mgx_fill_matrix(d_B, k, n, n, input, 0.0, er, seed + 1, nullptr), "fill B", EXIT_FAILURE);
    }
    mm::cuda_or_die(cudaDeviceSynchronize(), "initialisation", EXIT_FAILURE);

    cudaStream_t stream;
    mm::cuda_or_die(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate", EXIT_FAILURE);
    mm::Workspace ws;

    // One iteration of the hot loop's compute phase for every emulated rank.  The ranks' row
    // blocks are contiguous in A and C, and every element of C comes out of the same arithmetic
    // whatever the launch it belongs to, so by default all ranks' blocks run as one launch
    // (no tail wave per rank); MGXBENCH_BATCH=0 launches rank by rank.
    auto iteration = [&]() -> int {
        for (int r = 0; r < launches; ++r) {
            const double *A_r = d_A + (size_t)r * rows_per_launch * k;
            double *C_r = d_C + (size_t)r * rows_per_launch * n;
            const int mi = rows_per_launch;
            if (chunked) {
                cudaError_t e = cudaMemsetAsync(C_r, 0, (size_t)mi * n * sizeof(double), stream);
                if (e != cudaSuccess) return MGX_E_CUDA;
                const int num_chunks = (k + pipeline_k_chunk - 1) / pipeline_k_chunk;
                for (int c = 0; c < num_chunks; ++c) {
                    const int k_offset = c * pipeline_k_chunk;
                    const int kc = (k - k_offset < pipeline_k_chunk) ? k - k_offset : pipeline_k_chunk;
                    int rc;
                    if (form == mm::kFp64)
                        rc = mgx_ab_multiply_accumulate_async(A_r, d_B + (size_t)k_offset * n, C_r, mi, n, k, k_offset,
                                                              kc, k, n, n, 32, stream);
                    else
                        rc = mm::block_gemm(form, splits, 1, ws, A_r + k_offset, d_B + (size_t)k_offset * n, C_r, mi, n,
                                            kc, k, n, n, 1, stream);
                    if (rc < 0) return rc;
                }
            } else {
                const int rc = mm::block_gemm(form, splits, ksplit, ws, A_r, d_B, C_r, mi, n, k, k, n, n, 0, stream, tile_m);
                if (rc < 0) return rc;
            }
        }
        return MGX_SUCCESS;
    };

    const int loop_count = mm::env_int("MGXBENCH_INNER_LOOPS", 10);
    const int warmup_count = mm::env_int("MGXBENCH_INTERNAL_WARMUP", 0);
    if (loop_count < 1 || warmup_count < 0) {
        fprintf(stderr, "MGXBENCH_INNER_LOOPS must be >= 1 and MGXBENCH_INTERNAL_WARMUP >= 0\n");
        return 4;
    }

    cudaGraphExec_t exec = nullptr;
    if (graph) {
        // Workspace must exist before capture (no allocation inside a graph).
        mm::check_or_die(iteration(), "graph warm-up iteration", EXIT_FAILURE);
        mm::cuda_or_die(cudaStreamSynchronize(stream), "graph warm-up", EXIT_FAILURE);
        cudaGraph_t g;
        mm::cuda_or_die(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture",
                        EXIT_FAILURE);
        const int rc = iteration();
        mm::cuda_or_die(cudaStreamEndCapture(stream, &g), "end capture", EXIT_FAILURE);
        mm::check_or_die(rc, "captured iteration", EXIT_FAILURE);
        mm::cuda_or_die(cudaGraphInstantiate(&exec, g, 0), "graph instantiate", EXIT_FAILURE);
        cudaGraphDestroy(g);
    }

    double start_time = 0.0;
    if (warmup_count == 0) start_time = mm::wall_seconds();
    for (int iter = -warmup_count; iter < loop_count; ++iter) {
        if (iter == 0 && warmup_count > 0) {
            mm::cuda_or_die(cudaDeviceSynchronize(), "warm-up", EXIT_FAILURE);
            start_time = mm::wall_seconds();
        }
        if (exec)
            mm::cuda_or_die(cudaGraphLaunch(exec, stream), "graph launch", EXIT_FAILURE);
        else
            mm::check_or_die(iteration(), "block multiply", EXIT_FAILURE);
        mm::cuda_or_die(cudaStreamSynchronize(stream), "iteration", EXIT_FAILURE);
    }
    mm::cuda_or_die(cudaDeviceSynchronize(), "final synchronize", EXIT_FAILURE);
    const double stop_time = mm::wall_seconds();
    const double avg_time_execution = (stop_time - start_time) / (double)loop_count;
    int dev_status = 0;
    mgx_device_status(&dev_status);

    printf("\n\nmmb myRank=%d\tLibraries=%s\t RESULT: Matrix size: %d\tTime (seconds): %.9f\n\n", myRank, libs,
           matrix_size, avg_time_execution);

    int all_valid = 0;
    mgx_error_t err;
    memset(&err, 0, sizeof err);
    if (input == mm::kConst) {
        // A = 1, B = 2, so C[i,j] = 2 k (1D-row-block/mmb.cu:944-958)
        const double expected_C = 2.0 * (double)k;
        const int v = mgx_validate_matrix_c(d_C, m, n, expected_C, 1.0e-9, 1.0e-12, myRank, 1, nullptr);
        all_valid = (v == 1);
    } else {
        const double tol = autotuned ? mm::auto_target() : mm::int8_form(form) ? 1e-15 : 1e-12;
        all_valid = mm::report_accuracy(d_A, d_B, d_C, m, n, k, mm::env_int("MGXBENCH_CHECK_ROWS", 256), tol, &err);
    }
    if (dev_status != 0) {
        fprintf(stderr, "device status %d: a bounded device wait ran out\n", dev_status);
        all_valid = 0;
    }
    const double tflops = 2.0 * (double)m * n * k / avg_time_execution / 1e12;
    printf("BENCHMARK_RESULT decomposition=1D library=%s size=%d ranks=%d seconds=%.9f valid=%d loops=%d "
           "form=%s tflops=%.3f input=%s",
           libs, matrix_size, nRanks, avg_time_execution, all_valid, loop_count, form_name.c_str(), tflops,
           input_name.c_str());
    printf("%s", mm::form_count(form, splits).c_str());
    if (ksplit > 1) printf(" ksplit=%d", ksplit);
    if (ksplit == 0) printf(" streamk=1");
    if (tile_m != 128) printf(" tile_m=%d", tile_m);
    if (input != mm::kConst) printf(" norm_rel_err=%.3e max_rel_err=%.3e", err.normwise, err.max_rel);
    printf("\n");
    fflush(stdout);

    if (exec) cudaGraphExecDestroy(exec);
    cudaStreamDestroy(stream);
    cudaFree(d_A);
    cudaFree(d_B);
    cudaFree(d_C);
    return all_valid ? 0 : 2;
}
