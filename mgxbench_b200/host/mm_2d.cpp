// mm_2d -- drop-in for MGXBench's 2D SUMMA executable (2D-block-matrix/mmb.cu), run on one GPU.
//
//   mm_2d <auto|device> <N> <MMM|YYY|CCC|XXX|NNN|WWW|SSS>
//
// The Pr x Pc process grid comes from MGXBENCH_GRID_ROWS / MGXBENCH_GRID_COLS or the most
// nearly square factorisation of the emulated rank count (2D-block-matrix/mmb.cu:45-58); block
// (i, j) is C_ij (m x n, m = N/Pr, n = N/Pc), and every panel k0 of width BK
// (MGXBENCH_SUMMA_BK, default 256) adds A_i[:, k0:k0+kc] * B_j[k0:k0+kc, :] into C_ij after
// C = 0 (2D-block-matrix/mmb.cu:239-361).  All blocks and panels run on this GPU from resident
// A and B, so no panel is packed or copied; the library code is a label.
//
// Extensions (environment): MGXBENCH_M / MGXBENCH_N / MGXBENCH_K give a rectangular product
// (default N x N x N); MGXBENCH_UNEVEN=1 accepts grids that do not divide M or N, splitting
// with the first (M mod Pr) block rows one row taller (likewise for columns);
// MGXBENCH_PERSISTENT=0 falls back to one launch per (panel, block) instead of the persistent
// SUMMA kernel; MGXBENCH_GRAPH=1 replays the product from a CUDA graph; MGXBENCH_FORM=ozaki
// uses the INT8 Ozaki form (its panels accumulate exactly in integers, so the panel loop
// becomes the kernel's K loop).
// Records: the SUMMA header (2D-block-matrix/mmb.cu:147-148), the host constant check with its
// stderr message (mmb.cu:377-393) and one BENCHMARK_RESULT line (mmb.cu:398-399); exit status 0
// when valid, 1 otherwise, 2 on usage errors (mmb.cu:31-34, 439).
#include <algorithm>
#include <climits>

#include "autotune.h"
#include "mm_common.h"

static void fail(const char *message)
{
    fprintf(stderr, "2D SUMMA: %s\n", message);
    fflush(stderr);
    exit(2);
}

// Most nearly square Pr x Pc = p with Pr <= Pc (what MPI_Dims_create(p, 2) yields).
static void grid_shape(int p, int *pr, int *pc)
{
    const int r = mm::env_int("MGXBENCH_GRID_ROWS", 0);
    const int c = mm::env_int("MGXBENCH_GRID_COLS", 0);
    if (r < 0 || c < 0) {
        *pr = 0;
        *pc = 0;
        return;
    }
    if (r && c) {
        *pr = r;
        *pc = c;
        return;
    }
    if (r) {
        *pr = r;
        *pc = (p % r == 0 ? p / r : 0);
        return;
    }
    if (c) {
        *pc = c;
        *pr = (p % c == 0 ? p / c : 0);
        return;
    }
    int best = 1;
    for (int d = 1; (long long)d * d <= p; ++d)
        if (p % d == 0) best = d;
    *pr = best;
    *pc = p / best;
}

// Block boundaries of an extent split into `parts`: the first (extent mod parts) parts get one more.
static std::vector<int> split_extent(int extent, int parts)
{
    std::vector<int> cuts(parts + 1, 0);
    const int base = extent / parts, rem = extent % parts;
    for (int i = 0; i < parts; ++i) cuts[i + 1] = cuts[i] + base + (i < rem ? 1 : 0);
    return cuts;
}

int main(int argc, char **argv)
{
    const int p = mm::emulated_ranks();
    if (argc != 4) fail("Usage: mm_2d <auto|device> <N> <MMM|YYY|CCC|XXX|NNN|WWW|SSS>");
    const int N = atoi(argv[2]);
    const char *lib = argv[3];
    const char *codes[] = {"MMM", "YYY", "CCC", "XXX", "NNN", "WWW", "SSS"};
    bool supported = false;
    for (int i = 0; i < 7; ++i)
        if (!strcmp(lib, codes[i])) supported = true;
    if (!supported || N <= 0) fail("invalid matrix size or library");

    int Pr, Pc;
    grid_shape(p, &Pr, &Pc);
    if (Pr <= 0 || Pc <= 0 || (long long)Pr * Pc != p) fail("invalid process grid: rows*cols must equal MPI ranks");
    const int M = mm::env_int("MGXBENCH_M", N), Ncols = mm::env_int("MGXBENCH_N", N), K = mm::env_int("MGXBENCH_K", N);
    if (M <= 0 || Ncols <= 0 || K <= 0) fail("MGXBENCH_M/N/K must be positive");
    const int uneven = mm::env_int("MGXBENCH_UNEVEN", 0);
    if (!uneven && (M % Pr || Ncols % Pc)) fail("N must be divisible by both process-grid dimensions");
    if (Pr > M || Pc > Ncols) fail("process grid larger than the matrix");
    int BK = mm::env_int("MGXBENCH_SUMMA_BK", 256);
    if (BK <= 0) fail("MGXBENCH_SUMMA_BK must be positive");
    BK = std::min(BK, K);

    const int dev = !strcmp(argv[1], "auto") ? 0 : atoi(argv[1]);
    int device_count = 0;
    mm::cuda_or_die(cudaGetDeviceCount(&device_count), "cudaGetDeviceCount", 2);
    if (dev < 0 || dev >= device_count) fail("GPU device mapping invalid");
    mm::cuda_or_die(cudaSetDevice(dev), "cudaSetDevice", 2);

    std::string input_name, form_name;
    const int input = mm::input_kind(&input_name);
    int form = mm::compute_form(&form_name);
    if (input < 0 || form < 0) fail("MGXBENCH_INPUT must be const|uniform|wide and MGXBENCH_FORM fp64|ozaki|crt|auto");
    int splits = mm::env_int("MGXBENCH_SPLITS", 8);
    int ksplit = 1;  // the SUMMA panels are the K split
    int tile_m = 128;  // the SUMMA plan's work list is of 128 x 128 tiles
    const bool autotuned = form == mm::kAuto;
    mm::resolve_auto_form(&form, &splits, &ksplit, &tile_m, &form_name, M, Ncols, K,
                          input == mm::kWide ? mm::env_int("MGXBENCH_EXP_RANGE", 20) : 0, 2, true);
    if (form == mm::kCrt && !autotuned) splits = mm::env_int("MGXBENCH_MODULI", mgx_crt_choose_moduli(K, 1e-15));
    // the persistent SUMMA kernel runs the FP64 and digit-slice forms; the CRT form runs one
    // whole-K product per block (exact integer sums, so the panel order does not matter)
    const int persistent = form == mm::kCrt ? 0 : mm::env_int("MGXBENCH_PERSISTENT", 1);
    // CRT form: every block's result depends only on its rows of A and columns of B (whole-row
    // and whole-column scales, exact integer sums), so all blocks run as one product by default
    // (MGXBENCH_BATCH=1), bit-identical to one product per block (MGXBENCH_BATCH=0)
    const bool crt_batched = form == mm::kCrt && mm::env_int("MGXBENCH_BATCH", 1) != 0;
    const int graph = mm::env_int("MGXBENCH_GRAPH", 0);

    printf("SUMMA rectangular grid=%dx%d N=%d BK=%d library=%s ranks=%d pipeline=2\n", Pr, Pc, N, BK, lib, p);
    const std::vector<int> rcut = split_extent(M, Pr), ccut = split_extent(Ncols, Pc);
    const int mmax = rcut[1] - rcut[0], nmax = ccut[1] - ccut[0];
    {
        const double gib = 1073741824.0;
        const double panel_bytes = ((double)mmax * BK + (double)BK * nmax) * sizeof(double);
        printf("2D explicit device buffers per rank: %.6f GiB (C + panels; excludes runtime/heap reservation)\n",
               ((double)mmax * nmax * sizeof(double) + 2.0 * panel_bytes) / gib);
        printf("2D one-GPU emulation: M=%d N=%d K=%d blocks=%dx%d%s form=%s input=%s panels=%d %s\n", M, Ncols, K, Pr,
               Pc, uneven ? " (uneven split)" : "", form_name.c_str(), input_name.c_str(), (K + BK - 1) / BK,
               persistent ? "persistent"
                          : (crt_batched ? "all blocks in one product"
                                         : (mm::int8_form(form) ? "whole-K block products" : "per-panel launches")));
    }

    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    mm::cuda_or_die(cudaMalloc(&dA, (size_t)M * K * sizeof(double)), "cudaMalloc", 2);
    mm::cuda_or_die(cudaMalloc(&dB, (size_t)K * Ncols * sizeof(double)), "cudaMalloc", 2);
    mm::cuda_or_die(cudaMalloc(&dC, (size_t)M * Ncols * sizeof(double)), "cudaMalloc", 2);
    const unsigned long long seed = mm::env_u64("MGXBENCH_SEED", 20240901ull);
    if (input == mm::kConst) {  // Arow = 1.0, Bcol = 2.0 (2D-block-matrix/mmb.cu:151-154)
        mm::check_or_die(mgx_fill_matrix(dA, M, K, K, 0, 1.0, 0, 0, nullptr), "fill A", 2);
        mm::check_or_die(mgx_fill_matrix(dB, K, Ncols, Ncols, 0, 2.0, 0, 0, nullptr), "fill B", 2);
    } else {
        const int er = input == mm::kWide ? mm::env_int("MGXBENCH_EXP_RANGE", 20) : 0;
        mm::check_or_die(mgx_fill_matrix(dA, M, K, K, input, 0.0, er, seed, nullptr), "fill A", 2);
        mm::check_or_die(mgx_fill_matrix(dB, K, Ncols, Ncols, input, 0.0, er, seed + 1, nullptr), "fill B", 2);
    }
    cudaStream_t stream;
    mm::cuda_or_die(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate", 2);
    mm::cuda_or_die(cudaDeviceSynchronize(), "initialisation", 2);
    mm::Workspace ws;

    mgx_summa_plan_t *plan = nullptr;
    if (persistent) {
        mgx_summa_desc_t d;
        memset(&d, 0, sizeof d);
        d.m = M;
        d.n = Ncols;
        d.k = K;
        d.grid_rows = Pr;
        d.grid_cols = Pc;
        d.row_cuts = rcut.data();
        d.col_cuts = ccut.data();
        d.panel_k = BK;
        d.form = form == mm::kOzaki ? MGX_FORM_OZAKI : MGX_FORM_FP64;
        d.splits = splits;
        mm::check_or_die(mgx_summa_plan_create(&d, &plan), "mgx_summa_plan_create", 2);
    }

    const int numPanels = (K + BK - 1) / BK;
    auto run_product = [&]() -> int {
        if (plan) return mgx_summa_run(plan, dA, K, dB, Ncols, dC, Ncols, stream);
        cudaError_t e = cudaMemsetAsync(dC, 0, (size_t)M * Ncols * sizeof(double), stream);
        if (e != cudaSuccess) return MGX_E_CUDA;
        if (crt_batched)
            return mm::block_gemm(form, splits, 1, ws, dA, dB, dC, M, Ncols, K, K, Ncols, Ncols, 1, stream);
        if (mm::int8_form(form)) {  // integer panel sums are exact: one K loop per block
            for (int bi = 0; bi < Pr; ++bi)
                for (int bj = 0; bj < Pc; ++bj) {
                    const int r0 = rcut[bi], c0 = ccut[bj];
                    const int rc = mm::block_gemm(form, splits, 1, ws, dA + (size_t)r0 * K, dB + c0, dC + (size_t)r0 * Ncols + c0,
                                                  rcut[bi + 1] - r0, ccut[bj + 1] - c0, K, K, Ncols, Ncols, 1, stream);
                    if (rc < 0) return rc;
                }
            return MGX_SUCCESS;
        }
        for (int it = 0; it < numPanels; ++it) {
            const int k0 = it * BK;
            const int kc = std::min(BK, K - k0);
            for (int bi = 0; bi < Pr; ++bi)
                for (int bj = 0; bj < Pc; ++bj) {
                    const int r0 = rcut[bi], c0 = ccut[bj];
                    const int rc = mgx_ab_multiply_accumulate_async(dA + (size_t)r0 * K, dB + (size_t)k0 * Ncols + c0,
                                                                    dC + (size_t)r0 * Ncols + c0, rcut[bi + 1] - r0,
                                                                    ccut[bj + 1] - c0, K, k0, kc, K, Ncols, Ncols, 32,
                                                                    stream);
                    if (rc < 0) return rc;
                }
        }
        return MGX_SUCCESS;
    };

    cudaGraphExec_t exec = nullptr;
    if (graph) {
        mm::check_or_die(run_product(), "graph warm-up", 2);
        mm::cuda_or_die(cudaStreamSynchronize(stream), "graph warm-up", 2);
        cudaGraph_t g;
        mm::cuda_or_die(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture", 2);
        const int rc = run_product();
        mm::cuda_or_die(cudaStreamEndCapture(stream, &g), "end capture", 2);
        mm::check_or_die(rc, "captured product", 2);
        mm::cuda_or_die(cudaGraphInstantiate(&exec, g, 0), "graph instantiate", 2);
        cudaGraphDestroy(g);
    }
    const int warm = mm::env_int("MGXBENCH_INTERNAL_WARMUP", 0);
    for (int w = 0; w < warm; ++w) {
        if (exec) mm::cuda_or_die(cudaGraphLaunch(exec, stream), "graph launch", 2);
        else mm::check_or_die(run_product(), "warm-up product", 2);
    }
    mm::cuda_or_die(cudaDeviceSynchronize(), "cudaDeviceSynchronize", 2);

    const double t0 = mm::wall_seconds();
    if (exec) mm::cuda_or_die(cudaGraphLaunch(exec, stream), "graph launch", 2);
    else mm::check_or_die(run_product(), "SUMMA product", 2);
    mm::cuda_or_die(cudaStreamSynchronize(stream), "cudaStreamSynchronize", 2);
    const double elapsed = mm::wall_seconds() - t0;
    int dev_status = 0;
    mgx_device_status(&dev_status);

    int valid = 1;
    mgx_error_t err;
    memset(&err, 0, sizeof err);
    if (input == mm::kConst) {
        // Host check of every element (2D-block-matrix/mmb.cu:377-393), rank by rank.
        std::vector<double> C((size_t)M * Ncols);
        mm::cuda_or_die(cudaMemcpy(C.data(), dC, C.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy", 2);
        const double expected = 2.0 * K;
        const double tolerance = 1e-9 + 1e-12 * fabs(expected);
        for (int bi = 0; bi < Pr && valid; ++bi)
            for (int bj = 0; bj < Pc && valid; ++bj) {
                const int rank = bi * Pc + bj, ncols = ccut[bj + 1] - ccut[bj];
                for (int r = rcut[bi]; r < rcut[bi + 1] && valid; ++r)
                    for (int c = ccut[bj]; c < ccut[bj + 1]; ++c) {
                        const double value = C[(size_t)r * Ncols + c];
                        if (!std::isfinite(value) || fabs(value - expected) > tolerance) {
                            const size_t local = (size_t)(r - rcut[bi]) * ncols + (c - ccut[bj]);
                            fprintf(stderr, "Rank %d: 2D validation failed at local index=%zu: got %.17g expected %.17g\n",
                                    rank, local, value, expected);
                            valid = 0;
                            break;
                        }
                    }
            }
    } else {
        const double tol = autotuned ? mm::auto_target() : mm::int8_form(form) ? 1e-15 : 1e-12;
        valid = mm::report_accuracy(dA, dB, dC, M, Ncols, K, mm::env_int("MGXBENCH_CHECK_ROWS", 256), tol, &err);
    }
    if (dev_status != 0) {
        fprintf(stderr, "device status %d: a bounded device wait ran out\n", dev_status);
        valid = 0;
    }
    const double tflops = 2.0 * (double)M * Ncols * K / elapsed / 1e12;
    printf("BENCHMARK_RESULT decomposition=2D library=%s size=%d ranks=%d seconds=%.9f valid=%d loops=1 grid=%dx%d "
           "form=%s tflops=%.3f m=%d n=%d k=%d bk=%d input=%s",
           lib, N, p, elapsed, valid, Pr, Pc, form_name.c_str(), tflops, M, Ncols, K, BK, input_name.c_str());
    printf("%s", mm::form_count(form, splits).c_str());
    if (input != mm::kConst) printf(" norm_rel_err=%.3e max_rel_err=%.3e", err.normwise, err.max_rel);
    printf("\n");
    fflush(stdout);

    if (exec) cudaGraphExecDestroy(exec);
    if (plan) mgx_summa_plan_destroy(plan);
    cudaStreamDestroy(stream);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return valid ? 0 : 1;
}
