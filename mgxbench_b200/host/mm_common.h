// mm_common.h -- host helpers shared by the drop-in executables mm_1d and mm_2d.
//
// The executables keep MGXBench's command line (<dev|auto> <N> <library>), environment
// variables and stdout records; every emulated rank's blocks run on the one selected GPU.
#pragma once

#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mgxgemm.h"

namespace mm {

inline int env_int(const char *name, int fallback)
{
    const char *s = getenv(name);
    return (s && *s) ? atoi(s) : fallback;
}

inline std::string env_str(const char *name, const char *fallback)
{
    const char *s = getenv(name);
    return (s && *s) ? std::string(s) : std::string(fallback);
}

inline unsigned long long env_u64(const char *name, unsigned long long fallback)
{
    const char *s = getenv(name);
    return (s && *s) ? strtoull(s, nullptr, 0) : fallback;
}

// Ranks emulated on the one GPU.  mgx-onegpu-launch sets MGXBENCH_EMULATED_RANKS to the number
// of MPMD segments benchmark.py asked mpirun to start.
inline int emulated_ranks() { return env_int("MGXBENCH_EMULATED_RANKS", 1); }

inline double wall_seconds()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Input distributions (MGXBENCH_INPUT): "const" is MGXBench's A = 1, B = 2 initialisation.
enum InputKind { kConst = 0, kUniform = 1, kWide = 2 };

inline int input_kind(std::string *name)
{
    *name = env_str("MGXBENCH_INPUT", "const");
    if (*name == "const") return kConst;
    if (*name == "uniform") return kUniform;
    if (*name == "wide") return kWide;
    return -1;
}

// Compute forms (MGXBENCH_FORM): native FP64 tensor-core MMA, the Ozaki INT8 digit-slice form,
// its CRT form (Ozaki scheme II, MGXBENCH_MODULI moduli), or "auto" (the learned cost model picks
// the form and its split or modulus count, see autotune.h).
enum Form { kFp64 = 0, kOzaki = 1, kAuto = 2, kCrt = 3 };

inline int compute_form(std::string *name)
{
    *name = env_str("MGXBENCH_FORM", "fp64");
    if (*name == "fp64") return kFp64;
    if (*name == "ozaki") return kOzaki;
    if (*name == "crt") return kCrt;
    if (*name == "auto") return kAuto;
    return -1;
}

// The INT8 forms compute exact integer products (their results do not depend on how K is cut
// into panels) and are validated against 1e-15.
inline bool int8_form(int form) { return form == kOzaki || form == kCrt; }

// " splits=s" / " moduli=q" for the logs of the INT8 forms, "" for FP64.
inline std::string form_count(int form, int splits)
{
    if (form == kOzaki) return " splits=" + std::to_string(splits);
    if (form == kCrt) return " moduli=" + std::to_string(splits);
    return "";
}

inline void check_or_die(int rc, const char *what, int exit_code)
{
    if (rc < 0) {
        fprintf(stderr, "%s failed: %s (%s)\n", what, mgx_status_string(rc), mgx_last_error_message());
        fflush(stderr);
        exit(exit_code);
    }
}

inline void cuda_or_die(cudaError_t e, const char *what, int exit_code)
{
    if (e != cudaSuccess) {
        fprintf(stderr, "%s failed: %s\n", what, cudaGetErrorString(e));
        fflush(stderr);
        exit(exit_code);
    }
}

// Device workspace for the INT8 forms, grown on demand.
struct Workspace {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need)
    {
        if (need > bytes) {
            if (ptr) cudaFree(ptr);
            ptr = nullptr;
            bytes = 0;
            if (cudaMalloc(&ptr, need) != cudaSuccess) return nullptr;
            bytes = need;
        }
        return ptr;
    }
    ~Workspace()
    {
        if (ptr) cudaFree(ptr);
    }
};

// One block multiply C (+)= A B of the selected form with `ksplit` K slices (0: the FP64
// stream-K schedule; `splits` holds the modulus count for the CRT form; tile_m the FP64 output
// tile height, 64 or 128).
inline int block_gemm(int form, int splits, int ksplit, Workspace &ws, const double *A, const double *B, double *C,
                      int m, int n, int k, int lda, int ldb, int ldc, int beta_one, cudaStream_t s, int tile_m = 128)
{
    if (form == kFp64 && ksplit == 0) {  // stream-K over 64 x 128 tiles
        const size_t need = mgx_fp64_streamk_workspace_size(m, n, k);
        void *w = ws.get(need);
        if (!w && need) return MGX_E_CUDA;
        return mgx_gemm_fp64_streamk(A, B, C, m, n, k, lda, ldb, ldc, beta_one, w, need, s);
    }
    if (form == kFp64 && tile_m != 128) {
        const size_t need = ksplit > 1 ? mgx_fp64_splitk_workspace_size(m, n, k, ksplit) : 0;
        void *w = need ? ws.get(need) : nullptr;
        if (!w && need) return MGX_E_CUDA;
        return mgx_gemm_fp64_tiled(A, B, C, m, n, k, lda, ldb, ldc, beta_one, tile_m, ksplit, w, need, s);
    }
    if (form == kFp64 && ksplit > 1) {
        const size_t need = mgx_fp64_splitk_workspace_size(m, n, k, ksplit);
        void *w = ws.get(need);
        if (!w && need) return MGX_E_CUDA;
        return mgx_gemm_fp64_splitk(A, B, C, m, n, k, lda, ldb, ldc, beta_one, ksplit, w, need, s);
    }
    if (form == kFp64) return mgx_gemm_fp64(A, B, C, m, n, k, lda, ldb, ldc, beta_one, s);
    if (form == kCrt) {
        const size_t need = mgx_crt_workspace_size(m, n, k, splits);
        void *w = ws.get(need);
        if (!w && need) return MGX_E_CUDA;
        return mgx_gemm_ozaki_crt(A, B, C, m, n, k, lda, ldb, ldc, beta_one, splits, w, need, s);
    }
    if (ksplit > 1) {
        const size_t need = mgx_ozaki_splitk_workspace_size(m, n, k, splits, ksplit);
        void *w = ws.get(need);
        if (!w && need) return MGX_E_CUDA;
        return mgx_gemm_ozaki_splitk(A, B, C, m, n, k, lda, ldb, ldc, beta_one, splits, ksplit, w, need, s);
    }
    const size_t need = mgx_ozaki_workspace_size(m, n, k, splits);
    void *w = ws.get(need);
    if (!w && need) return MGX_E_CUDA;
    return mgx_gemm_ozaki(A, B, C, m, n, k, lda, ldb, ldc, beta_one, splits, w, need, s);
}

// Error of the computed product against the double-double GPU check on `rows` sampled rows;
// prints an ACCURACY block and returns whether the normwise error meets `tol`.
inline int report_accuracy(const double *A, const double *B, const double *C, int m, int n, int k, int sample_rows,
                           double tol, mgx_error_t *err)
{
    int rows = sample_rows > 0 && sample_rows < m ? sample_rows : m;
    const int start = (m - rows) / 2;
    const int rc = mgx_error_vs_dd(A, B, C, m, n, k, k, n, n, start, rows, 0x1.0p-40, err);
    if (rc < 0) {
        fprintf(stderr, "double-double check failed: %s\n", mgx_last_error_message());
        return 0;
    }
    printf("\n");
    printf("============================================================\n");
    printf("ACCURACY VS DOUBLE-DOUBLE PRODUCT\n");
    printf("============================================================\n");
    printf("Rows checked       : %llu of %d\n", (unsigned long long)err->rows_checked, m);
    printf("Normwise rel error : %.6e\n", err->normwise);
    printf("Max relative error : %.6e\n", err->max_rel);
    printf("Max componentwise  : %.6e\n", err->max_componentwise);
    printf("Normwise tolerance : %.6e\n", tol);
    printf("Result             : %s\n", err->normwise <= tol ? "PASS" : "FAIL");
    printf("============================================================\n");
    return err->normwise <= tol;
}

}  // namespace mm
