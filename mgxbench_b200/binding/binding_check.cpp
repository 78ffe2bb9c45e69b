// binding_check.cpp -- a stand-in for MGXBench's drivers that calls the binding
// (mulmat_kernel_mgx.cpp) exactly as they do: the three functions are declared here with the
// drivers' own declarations (1D-row-block/mmb.cu:162-164, 2D-block-matrix/mmb.cu:20-22) and
// linked from the binding, not from mgxgemm.h.
//
//   mgx_binding_check <m> <n> <k> <k_chunk> <dir>
//
// reads <dir>/A.bin (m x k) and <dir>/B.bin (k x n), row-major doubles, and writes
//   <dir>/C_sync.bin   ABMultiply(A, B)                     (the 1D single-multiply libraries)
//   <dir>/C_chunk.bin  C = 0, then ABMultiplyAccumulateAsync per K chunk of k_chunk on one stream
//                      (the 1D chunked libraries, 1D-row-block/mmb.cu:738-858)
// then runs the reference's known-answer check on A = 1, B = 2 through validate_matrix_C
// (expected 2k, abs 1e-9, rel 1e-12) and prints "binding_check validate=<0|1>".
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

extern int validate_matrix_C(const double *d_C, int rows, int cols, double expected, double abs_tol, double rel_tol, int rank);
extern void ABMultiply(double *a, double *b, double *c, int m, int n, int k, int lda, int ldb, int ldc, int w);
extern void ABMultiplyAccumulateAsync(const double *a, const double *b_chunk, double *c, int m, int n, int k_total, int k_offset, int k_chunk, int lda, int ldb, int ldc, int w, cudaStream_t stream);
// the 2D driver's declaration of the same function
extern void ABMultiplyAccumulateAsync(const double *, const double *, double *,
                                      int, int, int, int, int, int, int, int, int,
                                      cudaStream_t);

#define CHECK(call)                                                                           \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));                 \
            return 3;                                                                         \
        }                                                                                     \
    } while (0)

static bool read_file(const std::string &path, std::vector<double> &v)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = fread(v.data(), sizeof(double), v.size(), f);
    fclose(f);
    return got == v.size();
}

static bool write_file(const std::string &path, const std::vector<double> &v)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t put = fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
    return put == v.size();
}

int main(int argc, char **argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: %s <m> <n> <k> <k_chunk> <dir>\n", argv[0]);
        return 1;
    }
    const int m = atoi(argv[1]), n = atoi(argv[2]), k = atoi(argv[3]), kc = atoi(argv[4]);
    const std::string dir = argv[5];
    if (m <= 0 || n <= 0 || k <= 0 || kc <= 0) {
        fprintf(stderr, "invalid sizes\n");
        return 1;
    }
    std::vector<double> A((size_t)m * k), B((size_t)k * n), C((size_t)m * n);
    if (!read_file(dir + "/A.bin", A) || !read_file(dir + "/B.bin", B)) {
        fprintf(stderr, "cannot read %s/A.bin or B.bin\n", dir.c_str());
        return 1;
    }
    double *dA = nullptr, *dB = nullptr, *dC = nullptr;
    CHECK(cudaMalloc(&dA, A.size() * sizeof(double)));
    CHECK(cudaMalloc(&dB, B.size() * sizeof(double)));
    CHECK(cudaMalloc(&dC, C.size() * sizeof(double)));
    CHECK(cudaMemcpy(dA, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(dB, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice));

    ABMultiply(dA, dB, dC, m, n, k, k, n, n, 32);
    CHECK(cudaDeviceSynchronize());
    CHECK(cudaMemcpy(C.data(), dC, C.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (!write_file(dir + "/C_sync.bin", C)) return 1;

    cudaStream_t s;
    CHECK(cudaStreamCreate(&s));
    CHECK(cudaMemsetAsync(dC, 0, C.size() * sizeof(double), s));
    for (int off = 0; off < k; off += kc) {
        const int len = (k - off < kc) ? k - off : kc;
        ABMultiplyAccumulateAsync(dA, dB + (size_t)off * n, dC, m, n, k, off, len, k, n, n, 32, s);
    }
    CHECK(cudaStreamSynchronize(s));
    CHECK(cudaMemcpy(C.data(), dC, C.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (!write_file(dir + "/C_chunk.bin", C)) return 1;

    for (auto &x : A) x = 1.0;
    for (auto &x : B) x = 2.0;
    CHECK(cudaMemcpy(dA, A.data(), A.size() * sizeof(double), cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(dB, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice));
    ABMultiply(dA, dB, dC, m, n, k, k, n, n, 32);
    CHECK(cudaDeviceSynchronize());
    const int ok = validate_matrix_C(dC, m, n, 2.0 * k, 1e-9, 1e-12, 0);
    printf("binding_check validate=%d\n", ok);
    CHECK(cudaStreamDestroy(s));
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return ok ? 0 : 2;
}
