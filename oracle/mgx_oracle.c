/*
 * mgx_oracle.c -- CPU ORACLE. TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the GPU product in mgxbench_b200/. Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py load it.
 * Nothing in the product links or calls it.
 *
 * Contents
 *  1. A restatement of MGXBench's FP64 block multiply kernels
 *       sharedABMultiply            1D-row-block/mulmat_kernel.cu:39-80   (2D copy 2D-block-matrix/mulmat_kernel.cu:36-75)
 *       sharedABMultiplyAccumulate  1D-row-block/mulmat_kernel.cu:100-142 (2D copy 2D-block-matrix/mulmat_kernel.cu:94-136)
 *     Each output is one sequential FMA chain over k starting from +0.0 (nvcc contracts
 *     `sum += a*b` into DFMA); the accumulate form sums the chunk into a partial and then
 *     adds the partial into C with one rounding (mulmat_kernel.cu:141).  The loops below are
 *     blocked for speed, but every output keeps exactly that chain, so results are bit-identical
 *     to the reference kernel (pinned against the reference kernel's own outputs in
 *     tests/golden/).
 *  2. The driver loops that feed them:
 *       pipeline_k_chunk_from_env   1D-row-block/mmb.cu:109-128
 *       1D row-block hot loop       1D-row-block/mmb.cu:738-864 (sync: one ABMultiply;
 *                                   chunked Y/X/S: memset C, then C += A[:,chunk] B_chunk)
 *       2D SUMMA panel loop         2D-block-matrix/mmb.cu:239-361 (C = 0, then C += panel)
 *  3. Validation: validate_C_kernel semantics (1D-row-block/mulmat_kernel.cu:165-222) and the
 *     2D host check (2D-block-matrix/mmb.cu:377-393).
 *  4. A double-double GEMM (Dot2 of Ogita, Rump & Oishi 2005: TwoProd via FMA, TwoSum of
 *     Knuth) used as the exact-ish reference for error metrics.
 *  5. A restatement of this project's Ozaki-scheme split-precision GEMM (Ozaki, Ogita, Oishi &
 *     Rump 2012; Ootomo, Ozaki & Yokota 2024): per-row / per-column power-of-two scaling,
 *     signed radix-2^7 int8 digits, exact integer slice products grouped by digit weight, and
 *     FP64 Horner recombination.  The GPU form must match it bit for bit.
 *
 * Build: oracle/Makefile (gcc -O3 -mavx2 -mfma -fopenmp -ffp-contract=off).
 */
#include <immintrin.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

static int pick_threads(int nthreads)
{
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    return nthreads;
}

/* ------------------------------------------------------------------------------------------
 * 1. FMA-chain GEMM: P[i][j] = fold_k fma(A[i][k], B[k][j], acc), acc0 = +0.0
 *    (the arithmetic of sharedABMultiply's inner loop, mulmat_kernel.cu:72-73).
 *    `a_live` gives the number of leading k for which A is read; beyond it A contributes 0.0
 *    (the zero tile fill of sharedABMultiplyAccumulate, mulmat_kernel.cu:122-126).
 * ------------------------------------------------------------------------------------------ */
#define KC 256
#define NC 512

static void chain_panel(const double *A, int lda, const double *B, int ldb, double *P, int ldp,
                        int m, int n, int k, int a_live, int nthreads)
{
    /* P must hold the chain state; the first k-block starts it from +0.0. */
    double *Bp = (double *)aligned_alloc(64, (size_t)KC * NC * sizeof(double));
    for (int j0 = 0; j0 < n; j0 += NC) {
        const int nc = (n - j0 < NC) ? n - j0 : NC;
        const int nc8 = nc & ~7;
        for (int k0 = 0; k0 < k; k0 += KC) {
            const int kc = (k - k0 < KC) ? k - k0 : KC;
            const int first = (k0 == 0);
            /* pack B[k0:k0+kc, j0:j0+nc8] as [jb][k][8] */
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (int jb = 0; jb < nc8 / 8; ++jb)
                for (int kk = 0; kk < kc; ++kk)
                    memcpy(Bp + ((size_t)jb * kc + kk) * 8, B + (size_t)(k0 + kk) * ldb + j0 + jb * 8,
                           8 * sizeof(double));
            /* one work item = 4 rows x 64 columns of this panel (ragged columns go with jg == 0) */
            const int iblocks = (m + 3) / 4;
            const int jgroups = (nc8 / 8 + 7) / 8 > 0 ? (nc8 / 8 + 7) / 8 : 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4) collapse(2)
            for (int ib = 0; ib < iblocks; ++ib) {
                for (int jg = 0; jg < jgroups; ++jg) {
                    const int i0 = ib * 4;
                    const int mr = (m - i0 < 4) ? m - i0 : 4;
                    double areg[4][KC];
                    for (int r = 0; r < 4; ++r)
                        for (int kk = 0; kk < kc; ++kk) {
                            const int row = (r < mr) ? i0 + r : i0;
                            areg[r][kk] = (k0 + kk < a_live) ? A[(size_t)row * lda + k0 + kk] : 0.0;
                        }
                    for (int jb = jg * 8; jb < jg * 8 + 8 && jb < nc8 / 8; ++jb) {
                        const double *bp = Bp + (size_t)jb * kc * 8;
                        double *pc = P + (size_t)i0 * ldp + j0 + jb * 8;
                        if (mr == 4) {
                            __m256d c00, c01, c10, c11, c20, c21, c30, c31;
                            if (first) {
                                c00 = c01 = c10 = c11 = c20 = c21 = c30 = c31 = _mm256_setzero_pd();
                            } else {
                                c00 = _mm256_loadu_pd(pc + 0 * ldp); c01 = _mm256_loadu_pd(pc + 0 * ldp + 4);
                                c10 = _mm256_loadu_pd(pc + 1 * ldp); c11 = _mm256_loadu_pd(pc + 1 * ldp + 4);
                                c20 = _mm256_loadu_pd(pc + 2 * ldp); c21 = _mm256_loadu_pd(pc + 2 * ldp + 4);
                                c30 = _mm256_loadu_pd(pc + 3 * ldp); c31 = _mm256_loadu_pd(pc + 3 * ldp + 4);
                            }
                            for (int kk = 0; kk < kc; ++kk) {
                                const __m256d b0 = _mm256_load_pd(bp + kk * 8);
                                const __m256d b1 = _mm256_load_pd(bp + kk * 8 + 4);
                                __m256d a = _mm256_broadcast_sd(&areg[0][kk]);
                                c00 = _mm256_fmadd_pd(a, b0, c00); c01 = _mm256_fmadd_pd(a, b1, c01);
                                a = _mm256_broadcast_sd(&areg[1][kk]);
                                c10 = _mm256_fmadd_pd(a, b0, c10); c11 = _mm256_fmadd_pd(a, b1, c11);
                                a = _mm256_broadcast_sd(&areg[2][kk]);
                                c20 = _mm256_fmadd_pd(a, b0, c20); c21 = _mm256_fmadd_pd(a, b1, c21);
                                a = _mm256_broadcast_sd(&areg[3][kk]);
                                c30 = _mm256_fmadd_pd(a, b0, c30); c31 = _mm256_fmadd_pd(a, b1, c31);
                            }
                            _mm256_storeu_pd(pc + 0 * ldp, c00); _mm256_storeu_pd(pc + 0 * ldp + 4, c01);
                            _mm256_storeu_pd(pc + 1 * ldp, c10); _mm256_storeu_pd(pc + 1 * ldp + 4, c11);
                            _mm256_storeu_pd(pc + 2 * ldp, c20); _mm256_storeu_pd(pc + 2 * ldp + 4, c21);
                            _mm256_storeu_pd(pc + 3 * ldp, c30); _mm256_storeu_pd(pc + 3 * ldp + 4, c31);
                        } else {
                            for (int r = 0; r < mr; ++r)
                                for (int c = 0; c < 8; ++c) {
                                    double acc = first ? 0.0 : pc[(size_t)r * ldp + c];
                                    for (int kk = 0; kk < kc; ++kk)
                                        acc = fma(areg[r][kk], bp[kk * 8 + c], acc);
                                    pc[(size_t)r * ldp + c] = acc;
                                }
                        }
                    }
                    if (jg == 0) {
                        /* ragged columns */
                        for (int r = 0; r < mr; ++r)
                            for (int c = j0 + nc8; c < j0 + nc; ++c) {
                                double acc = first ? 0.0 : P[(size_t)(i0 + r) * ldp + c];
                                for (int kk = 0; kk < kc; ++kk)
                                    acc = fma(areg[r][kk], B[(size_t)(k0 + kk) * ldb + c], acc);
                                P[(size_t)(i0 + r) * ldp + c] = acc;
                            }
                    }
                }
            }
        }
        if (k == 0) {
            for (int i = 0; i < m; ++i)
                for (int c = j0; c < j0 + nc; ++c) P[(size_t)i * ldp + c] = 0.0;
        }
    }
    free(Bp);
}

/* AVX-512 form of chain_panel: 8 rows x 16 columns per register block (16 accumulators).  Every
 * output still receives its products one FMA at a time in increasing k, so the results are the
 * same bits as chain_panel's.  Compiled for AVX-512 by attribute and called only when the CPU has
 * it. */
__attribute__((target("avx512f"))) static void chain_panel_avx512(const double *A, int lda, const double *B,
                                                                   int ldb, double *P, int ldp, int m, int n, int k,
                                                                   int a_live, int nthreads)
{
    double *Bp = (double *)aligned_alloc(64, (size_t)KC * NC * sizeof(double));
    for (int j0 = 0; j0 < n; j0 += NC) {
        const int nc = (n - j0 < NC) ? n - j0 : NC;
        const int nc16 = nc & ~15;
        for (int k0 = 0; k0 < k; k0 += KC) {
            const int kc = (k - k0 < KC) ? k - k0 : KC;
            const int first = (k0 == 0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (int jb = 0; jb < nc16 / 16; ++jb)
                for (int kk = 0; kk < kc; ++kk)
                    memcpy(Bp + ((size_t)jb * kc + kk) * 16, B + (size_t)(k0 + kk) * ldb + j0 + jb * 16,
                           16 * sizeof(double));
            const int iblocks = (m + 7) / 8;
            const int jgroups = (nc16 / 16 + 3) / 4 > 0 ? (nc16 / 16 + 3) / 4 : 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 2) collapse(2)
            for (int ib = 0; ib < iblocks; ++ib) {
                for (int jg = 0; jg < jgroups; ++jg) {
                    const int i0 = ib * 8;
                    const int mr = (m - i0 < 8) ? m - i0 : 8;
                    double areg[8][KC];
                    for (int r = 0; r < 8; ++r)
                        for (int kk = 0; kk < kc; ++kk) {
                            const int row = (r < mr) ? i0 + r : i0;
                            areg[r][kk] = (k0 + kk < a_live) ? A[(size_t)row * lda + k0 + kk] : 0.0;
                        }
                    for (int jb = jg * 4; jb < jg * 4 + 4 && jb < nc16 / 16; ++jb) {
                        const double *bp = Bp + (size_t)jb * kc * 16;
                        double *pc = P + (size_t)i0 * ldp + j0 + jb * 16;
                        __m512d c[8][2];
                        for (int r = 0; r < 8; ++r) {
                            if (first || r >= mr) {
                                c[r][0] = _mm512_setzero_pd();
                                c[r][1] = _mm512_setzero_pd();
                            } else {
                                c[r][0] = _mm512_loadu_pd(pc + (size_t)r * ldp);
                                c[r][1] = _mm512_loadu_pd(pc + (size_t)r * ldp + 8);
                            }
                        }
                        for (int kk = 0; kk < kc; ++kk) {
                            const __m512d b0 = _mm512_load_pd(bp + kk * 16);
                            const __m512d b1 = _mm512_load_pd(bp + kk * 16 + 8);
                            for (int r = 0; r < 8; ++r) {
                                const __m512d a = _mm512_set1_pd(areg[r][kk]);
                                c[r][0] = _mm512_fmadd_pd(a, b0, c[r][0]);
                                c[r][1] = _mm512_fmadd_pd(a, b1, c[r][1]);
                            }
                        }
                        for (int r = 0; r < mr; ++r) {
                            _mm512_storeu_pd(pc + (size_t)r * ldp, c[r][0]);
                            _mm512_storeu_pd(pc + (size_t)r * ldp + 8, c[r][1]);
                        }
                    }
                    if (jg == 0) {
                        for (int r = 0; r < mr; ++r)
                            for (int cc = j0 + nc16; cc < j0 + nc; ++cc) {
                                double acc = first ? 0.0 : P[(size_t)(i0 + r) * ldp + cc];
                                for (int kk = 0; kk < kc; ++kk)
                                    acc = fma(areg[r][kk], B[(size_t)(k0 + kk) * ldb + cc], acc);
                                P[(size_t)(i0 + r) * ldp + cc] = acc;
                            }
                    }
                }
            }
        }
        if (k == 0) {
            for (int i = 0; i < m; ++i)
                for (int cc = j0; cc < j0 + nc; ++cc) P[(size_t)i * ldp + cc] = 0.0;
        }
    }
    free(Bp);
}

static int have_avx512(void)
{
    static int cached = -1;
    if (cached < 0) {
        __builtin_cpu_init();
        cached = __builtin_cpu_supports("avx512f") ? 1 : 0;
        const char *e = getenv("MGX_ORACLE_NO_AVX512");
        if (e && *e == '1') cached = 0;
    }
    return cached;
}

/* The same chain written as the plain triple loop of the reference kernel's arithmetic, one
 * output at a time; used to check the blocked form above. */
ORACLE_API void oracle_ab_multiply_naive(const double *A, const double *B, double *C, int m, int n, int k,
                                         int lda, int ldb, int ldc)
{
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double sum = 0.0;
            for (int kk = 0; kk < k; ++kk) sum = fma(A[(size_t)i * lda + kk], B[(size_t)kk * ldb + j], sum);
            C[(size_t)i * ldc + j] = sum;
        }
}

/* sharedABMultiply + ABMultiply (1D-row-block/mulmat_kernel.cu:39-92): C = A B, overwrite. */
ORACLE_API void oracle_ab_multiply(const double *A, const double *B, double *C, int m, int n, int k,
                                   int lda, int ldb, int ldc, int nthreads)
{
    if (m <= 0 || n <= 0) return;
    if (have_avx512())
        chain_panel_avx512(A, lda, B, ldb, C, ldc, m, n, k, k, pick_threads(nthreads));
    else
        chain_panel(A, lda, B, ldb, C, ldc, m, n, k, k, pick_threads(nthreads));
}

/* sharedABMultiplyAccumulate (1D-row-block/mulmat_kernel.cu:100-142):
 * C += A[:, k_offset : k_offset + k_chunk] * B_chunk, the chunk summed into a partial first.
 * A columns at or beyond k_total read as 0.0 (mulmat_kernel.cu:122-126). */
ORACLE_API void oracle_ab_multiply_accumulate(const double *A, const double *Bchunk, double *C, int m, int n,
                                              int k_total, int k_offset, int k_chunk, int lda, int ldb,
                                              int ldc, int nthreads)
{
    if (m <= 0 || n <= 0 || k_chunk <= 0) return;
    nthreads = pick_threads(nthreads);
    double *P = (double *)malloc((size_t)m * n * sizeof(double));
    int a_live = k_total - k_offset;
    if (a_live < 0) a_live = 0;
    if (have_avx512())
        chain_panel_avx512(A + k_offset, lda, Bchunk, ldb, P, n, m, n, k_chunk, a_live, nthreads);
    else
        chain_panel(A + k_offset, lda, Bchunk, ldb, P, n, m, n, k_chunk, a_live, nthreads);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) C[(size_t)i * ldc + j] += P[(size_t)i * n + j];
    free(P);
}

/* ------------------------------------------------------------------------------------------
 * 2. Driver loops
 * ------------------------------------------------------------------------------------------ */

/* pipeline_k_chunk_from_env (1D-row-block/mmb.cu:109-128), with the env value passed in
 * (requested <= 0 means unset). */
ORACLE_API int oracle_pipeline_k_chunk(int k, int requested)
{
    int chunk = 2048;
    if (requested > 0) chunk = requested;
    if (chunk > k) chunk = k;
    if (chunk >= 32) chunk = (chunk / 32) * 32;
    return (chunk > 0) ? chunk : k;
}

/* 1D row-block compute phase (1D-row-block/mmb.cu:738-864) for every emulated rank:
 * rank r owns rows [r*mi, (r+1)*mi), mi = N / ranks (mmb.cu:312).  `chunked` selects the
 * Y/X/S libraries' B pipeline (memset C, then one accumulate per K chunk); otherwise one
 * ABMultiply over the full K.  C is the gathered N x N result. */
ORACLE_API void oracle_mm1d(const double *A, const double *B, double *C, int N, int ranks, int chunked,
                            int k_chunk, int nthreads)
{
    const int mi = N / ranks;
    for (int r = 0; r < ranks; ++r) {
        const double *Ar = A + (size_t)r * mi * N;
        double *Cr = C + (size_t)r * mi * N;
        if (!chunked) {
            oracle_ab_multiply(Ar, B, Cr, mi, N, N, N, N, N, nthreads);
        } else {
            memset(Cr, 0, (size_t)mi * N * sizeof(double));
            const int num_chunks = (N + k_chunk - 1) / k_chunk;
            for (int c = 0; c < num_chunks; ++c) {
                const int k_offset = c * k_chunk;
                const int kc = (N - k_offset < k_chunk) ? N - k_offset : k_chunk;
                oracle_ab_multiply_accumulate(Ar, B + (size_t)k_offset * N, Cr, mi, N, N, k_offset, kc, N, N,
                                              N, nthreads);
            }
        }
    }
}

/* 2D SUMMA panel loop (2D-block-matrix/mmb.cu:239-361) for every block of the process grid:
 * C = 0 (mmb.cu:186); for each panel k0 of width bk: C_ij += A_i[:, k0:k0+kc] B_j[k0:k0+kc, :].
 * Each element's arithmetic does not depend on which block owns it, so the blocks are computed
 * together here; M x K and K x N row-major, C is M x N. */
ORACLE_API void oracle_summa2d(const double *A, const double *B, double *C, int M, int N, int K, int bk,
                               int nthreads)
{
    memset(C, 0, (size_t)M * N * sizeof(double));
    if (bk > K) bk = K;
    const int panels = (K + bk - 1) / bk;
    for (int p = 0; p < panels; ++p) {
        const int k0 = p * bk;
        const int kc = (K - k0 < bk) ? K - k0 : bk;
        oracle_ab_multiply_accumulate(A, B + (size_t)k0 * N, C, M, N, K, k0, kc, K, N, N, nthreads);
    }
}

/* ------------------------------------------------------------------------------------------
 * 3. Validation
 * ------------------------------------------------------------------------------------------ */

/* validate_C_kernel (1D-row-block/mulmat_kernel.cu:165-222): an element is invalid when both
 * its absolute error exceeds abs_tol and its relative error exceeds rel_tol; the maxima of the
 * absolute and relative error are reported.  `count_nonfinite` adds the product's stricter rule:
 * a NaN or infinite element is also invalid (the reference kernel's comparisons are false for
 * NaN, so it never counts one) and NaN errors do not enter the maxima. */
ORACLE_API void oracle_validate_constant(const double *C, size_t count, double expected, double abs_tol,
                                         double rel_tol, int count_nonfinite, uint64_t *n_bad,
                                         double *max_abs, double *max_rel)
{
    uint64_t bad = 0;
    double mabs = 0.0, mrel = 0.0;
    for (size_t i = 0; i < count; ++i) {
        const double v = C[i];
        const double ae = fabs(v - expected);
        const double re = (fabs(expected) > 0.0) ? ae / fabs(expected) : 0.0;
        if ((ae > abs_tol) && (re > rel_tol)) ++bad;
        else if (count_nonfinite && !isfinite(v)) ++bad;
        if (ae > mabs) mabs = ae;
        if (re > mrel) mrel = re;
    }
    *n_bad = bad;
    *max_abs = mabs;
    *max_rel = mrel;
}

/* 2D host check (2D-block-matrix/mmb.cu:377-393): first index with a non-finite value or
 * |C - expected| > 1e-9 + 1e-12 |expected|, or -1 when every element passes. */
ORACLE_API int64_t oracle_validate_2d(const double *C, size_t count, double expected)
{
    const double tol = 1e-9 + 1e-12 * fabs(expected);
    for (size_t i = 0; i < count; ++i) {
        const double v = C[i];
        if (!isfinite(v) || fabs(v - expected) > tol) return (int64_t)i;
    }
    return -1;
}

/* ------------------------------------------------------------------------------------------
 * 4. Double-double GEMM (Dot2): hi + lo ~ sum_k a_ik b_kj as if in twice FP64 precision, and
 *    absprod = sum_k |a_ik| |b_kj| (plain FP64) for componentwise error bounds.
 * ------------------------------------------------------------------------------------------ */
ORACLE_API void oracle_gemm_dd(const double *A, const double *B, double *Chi, double *Clo, double *Cabs,
                               int m, int n, int k, int lda, int ldb, int ldc, int nthreads)
{
    nthreads = pick_threads(nthreads);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i = 0; i < m; ++i) {
        int j = 0;
        for (; j + 4 <= n; j += 4) {
            __m256d s = _mm256_setzero_pd(), c = _mm256_setzero_pd(), ab = _mm256_setzero_pd();
            const __m256d signmask = _mm256_set1_pd(-0.0);
            for (int kk = 0; kk < k; ++kk) {
                const __m256d a = _mm256_set1_pd(A[(size_t)i * lda + kk]);
                const __m256d b = _mm256_loadu_pd(B + (size_t)kk * ldb + j);
                const __m256d p = _mm256_mul_pd(a, b);
                const __m256d q = _mm256_fmsub_pd(a, b, p);              /* TwoProd error */
                const __m256d t = _mm256_add_pd(s, p);                   /* TwoSum(s, p) */
                const __m256d z = _mm256_sub_pd(t, s);
                const __m256d e = _mm256_add_pd(_mm256_sub_pd(s, _mm256_sub_pd(t, z)), _mm256_sub_pd(p, z));
                s = t;
                c = _mm256_add_pd(c, _mm256_add_pd(e, q));
                ab = _mm256_fmadd_pd(_mm256_andnot_pd(signmask, a), _mm256_andnot_pd(signmask, b), ab);
            }
            const __m256d hi = _mm256_add_pd(s, c);                      /* Fast2Sum(s, c) */
            const __m256d lo = _mm256_sub_pd(c, _mm256_sub_pd(hi, s));
            _mm256_storeu_pd(Chi + (size_t)i * ldc + j, hi);
            _mm256_storeu_pd(Clo + (size_t)i * ldc + j, lo);
            if (Cabs) _mm256_storeu_pd(Cabs + (size_t)i * ldc + j, ab);
        }
        for (; j < n; ++j) {
            double s = 0.0, c = 0.0, ab = 0.0;
            for (int kk = 0; kk < k; ++kk) {
                const double a = A[(size_t)i * lda + kk], b = B[(size_t)kk * ldb + j];
                const double p = a * b, q = fma(a, b, -p);
                const double t = s + p, z = t - s, e = (s - (t - z)) + (p - z);
                s = t;
                c += e + q;
                ab = fma(fabs(a), fabs(b), ab);
            }
            const double hi = s + c;
            Chi[(size_t)i * ldc + j] = hi;
            Clo[(size_t)i * ldc + j] = c - (hi - s);
            if (Cabs) Cabs[(size_t)i * ldc + j] = ab;
        }
    }
}

/* Error of C against the double-double reference (hi, lo) over an m x n block:
 *   out[0] normwise  ||C - R||_F / ||R||_F
 *   out[1] max elementwise |C - R| / |R| over elements with |R| >= floor_rel * max|R|
 *   out[2] max componentwise |C - R| / (|A||B|) (absprod may be NULL -> 0)
 *   out[3] max |C - R| */
ORACLE_API void oracle_error_metrics(const double *C, int ldc, const double *Rhi, const double *Rlo,
                                     const double *Rabs, int ldr, int m, int n, double floor_rel, double *out)
{
    double num = 0.0, den = 0.0, maxr = 0.0, maxabsR = 0.0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            const double r = fabs(Rhi[(size_t)i * ldr + j]);
            if (r > maxabsR) maxabsR = r;
        }
    const double floor_v = floor_rel * maxabsR;
    double maxe = 0.0, maxc = 0.0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            const double r = Rhi[(size_t)i * ldr + j];
            const double d = (C[(size_t)i * ldc + j] - r) - Rlo[(size_t)i * ldr + j];
            num += d * d;
            den += r * r;
            const double ad = fabs(d);
            if (ad > maxe) maxe = ad;
            if (fabs(r) >= floor_v && fabs(r) > 0.0) {
                const double rel = ad / fabs(r);
                if (rel > maxr) maxr = rel;
            }
            if (Rabs) {
                const double w = Rabs[(size_t)i * ldr + j];
                if (w > 0.0 && ad / w > maxc) maxc = ad / w;
            }
        }
    out[0] = (den > 0.0) ? sqrt(num) / sqrt(den) : sqrt(num);
    out[1] = maxr;
    out[2] = maxc;
    out[3] = maxe;
}

/* ------------------------------------------------------------------------------------------
 * 5. Ozaki-scheme split-precision GEMM restatement (bit-exact model of the GPU form)
 * ------------------------------------------------------------------------------------------ */

/* frexp exponent of |x| from its bit pattern: |x| in [2^(e-1), 2^e); 0 for x == 0. */
static int frexp_exp_bits(uint64_t absbits)
{
    if (absbits == 0) return 0;
    const int biased = (int)(absbits >> 52);
    if (biased != 0) return biased - 1022;
    const uint64_t mant = absbits & ((1ull << 52) - 1);
    return -1022 - (__builtin_clzll(mant) - 12);
}

static double pow2i(int e) /* 2^e for e in [-1022, 1023] */
{
    uint64_t bits = (uint64_t)(e + 1023) << 52;
    double d;
    memcpy(&d, &bits, sizeof d);
    return d;
}

/* x * 2^e with the two-step form used on the GPU when 2^e is not a normal double. */
static double scale2(double x, int e)
{
    if (e >= -1022 && e <= 1023) return x * pow2i(e);
    const int e1 = e / 2, e2 = e - e1;
    return (x * pow2i(e1)) * pow2i(e2);
}

/* Row exponents of A (m x k) and column exponents of B (k x n).  Returns 1 if a non-finite
 * value was seen (the Ozaki form rejects such inputs). */
ORACLE_API int oracle_ozaki_exponents(const double *A, const double *B, int m, int n, int k, int lda, int ldb,
                                      int32_t *ea, int32_t *eb)
{
    int nonfinite = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : nonfinite)
    for (int i = 0; i < m; ++i) {
        uint64_t mx = 0;
        for (int kk = 0; kk < k; ++kk) {
            uint64_t b;
            memcpy(&b, &A[(size_t)i * lda + kk], 8);
            b &= 0x7fffffffffffffffull;
            if (b >= 0x7ff0000000000000ull) nonfinite = 1;
            if (b > mx) mx = b;
        }
        ea[i] = frexp_exp_bits(mx);
    }
#pragma omp parallel for schedule(dynamic, 16) reduction(| : nonfinite)
    for (int j = 0; j < n; ++j) {
        uint64_t mx = 0;
        for (int kk = 0; kk < k; ++kk) {
            uint64_t b;
            memcpy(&b, &B[(size_t)kk * ldb + j], 8);
            b &= 0x7fffffffffffffffull;
            if (b >= 0x7ff0000000000000ull) nonfinite = 1;
            if (b > mx) mx = b;
        }
        eb[j] = frexp_exp_bits(mx);
    }
    return nonfinite;
}

#define OZ_MAX_SLICES 16

/* Signed radix-2^7 digits of x * 2^(6 - e): |x * 2^(6-e)| < 64, digit_t = rint(r), r <- (r - digit_t) * 128.
 * Every digit lies in [-64, 64]. */
static void digits_of(double v, int e, int s, int8_t *out, size_t stride)
{
    double x = scale2(v, 6 - e);
    for (int t = 0; t < s; ++t) {
        const double d = nearbyint(x);
        out[(size_t)t * stride] = (int8_t)d;
        x = (x - d) * 128.0;
    }
}

/* Digits of A as [t][i][kp] and of B as [u][j][kp] (B transposed), kp = row pitch >= k,
 * padding columns zero. */
ORACLE_API void oracle_ozaki_split(const double *A, const double *B, int m, int n, int k, int lda, int ldb,
                                   int s, int kp, const int32_t *ea, const int32_t *eb, int8_t *da, int8_t *db)
{
    memset(da, 0, (size_t)s * m * kp);
    memset(db, 0, (size_t)s * n * kp);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < m; ++i)
        for (int kk = 0; kk < k; ++kk)
            digits_of(A[(size_t)i * lda + kk], ea[i], s, da + (size_t)i * kp + kk, (size_t)m * kp);
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 0; j < n; ++j)
        for (int kk = 0; kk < k; ++kk)
            digits_of(B[(size_t)kk * ldb + j], eb[j], s, db + (size_t)j * kp + kk, (size_t)n * kp);
}

/* Largest k for which one weight group of s slice products of digits in [-64, 64] cannot leave int32. */
ORACLE_API int oracle_ozaki_kmax(int s)
{
    return (int)(2147483647ll / (4096ll * s));
}

/* C = (beta_one ? C : 0) + A B by the Ozaki form with s digits per operand:
 *   G_d[i][j] = sum_{t+u=d} sum_k DA_t[i][k] DB_u[j][k]        (exact, d = 2..s+1)
 *   h = G_{s+1}; for d = s..2: h = fma(h, 2^-7, G_d)           (Horner, smallest weight first)
 *   C_ij (+)= h * 2^(ea_i + eb_j - 12)
 * K is processed in chunks of at most oracle_ozaki_kmax(s) (rounded down to a multiple of 128),
 * each chunk split with its own exponents and added into C in order.  Returns 1 on non-finite
 * input (C untouched). */
ORACLE_API int oracle_ozaki_gemm(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                 int ldb, int ldc, int s, int beta_one, int nthreads)
{
    nthreads = pick_threads(nthreads);
    if (s < 1 || s > OZ_MAX_SLICES) return 2;
    int kmax = oracle_ozaki_kmax(s) & ~127;
    if (kmax <= 0) kmax = 128;
    int32_t *ea = (int32_t *)malloc(sizeof(int32_t) * (m > 0 ? m : 1));
    int32_t *eb = (int32_t *)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    if (!beta_one)
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < n; ++j) C[(size_t)i * ldc + j] = 0.0;
    int first = 1;
    for (int k0 = 0; k0 < k || (k == 0 && first); k0 += kmax) {
        const int kc = (k - k0 < kmax) ? k - k0 : kmax;
        if (oracle_ozaki_exponents(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, ea, eb)) {
            free(ea);
            free(eb);
            return 1;
        }
        const int kp = (kc + 15) & ~15;
        int8_t *da = (int8_t *)malloc((size_t)s * m * kp + 1);
        int8_t *db = (int8_t *)malloc((size_t)s * n * kp + 1);
        oracle_ozaki_split(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, s, kp, ea, eb, da, db);
        /* over (i, j) pairs, so that a few rows still use every thread */
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64) collapse(2)
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < n; ++j) {
                int64_t g[OZ_MAX_SLICES + 2] = {0};
                for (int d = 0; d < s + 2; ++d) g[d] = 0;
                for (int t = 1; t <= s; ++t)
                    for (int u = 1; t + u <= s + 1; ++u) {
                        const int8_t *pa = da + ((size_t)(t - 1) * m + i) * kp;
                        const int8_t *pb = db + ((size_t)(u - 1) * n + j) * kp;
                        int64_t acc = 0;
                        for (int kk = 0; kk < kc; ++kk) acc += (int64_t)pa[kk] * pb[kk];
                        g[t + u] += acc;
                    }
                double h = (double)(int32_t)g[s + 1];
                for (int d = s; d >= 2; --d) h = fma(h, 0.0078125, (double)(int32_t)g[d]);
                const double r = scale2(h, ea[i] + eb[j] - 12);
                C[(size_t)i * ldc + j] = C[(size_t)i * ldc + j] + r;
            }
        }
        free(da);
        free(db);
        first = 0;
        if (k == 0) break;
    }
    free(ea);
    free(eb);
    return 0;
}

/* Split-K form of the Ozaki product (k <= oracle_ozaki_kmax(s)), as the GPU computes it: the
 * exponents and digits come from the whole K range; the 32-wide K blocks are cut into slices of
 * ceil(kblocks / ksplit) blocks; each slice's group sums are recombined (Horner) and scaled on
 * their own, and the slice results are added in slice order:
 *   v = P_0 + P_1 + ... (left to right);  C = beta_one ? C + v : v.
 * With one slice this is oracle_ozaki_gemm.  Returns 1 on non-finite input, 2 if k > kmax. */
ORACLE_API int oracle_ozaki_gemm_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                        int ldb, int ldc, int s, int ksplit, int beta_one, int nthreads)
{
    nthreads = pick_threads(nthreads);
    if (k > (oracle_ozaki_kmax(s) & ~127)) return 2;
    const int kblocks = (k + 31) / 32 > 0 ? (k + 31) / 32 : 1;
    if (ksplit < 1) ksplit = 1;
    if (ksplit > kblocks) ksplit = kblocks;
    const int kbs = (kblocks + ksplit - 1) / ksplit;
    const int slices = (kblocks + kbs - 1) / kbs;
    int32_t *ea = (int32_t *)malloc(sizeof(int32_t) * (m > 0 ? m : 1));
    int32_t *eb = (int32_t *)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    if (oracle_ozaki_exponents(A, B, m, n, k, lda, ldb, ea, eb)) {
        free(ea);
        free(eb);
        return 1;
    }
    const int kp = (k + 15) & ~15;
    int8_t *da = (int8_t *)malloc((size_t)s * m * kp + 1);
    int8_t *db = (int8_t *)malloc((size_t)s * n * kp + 1);
    oracle_ozaki_split(A, B, m, n, k, lda, ldb, s, kp, ea, eb, da, db);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i = 0; i < m; ++i) {
        int64_t *g = (int64_t *)malloc(sizeof(int64_t) * (s + 2));
        for (int j = 0; j < n; ++j) {
            double v = 0.0;
            for (int sl = 0; sl < slices; ++sl) {
                const int k0 = sl * kbs * 32, k1 = (sl + 1) * kbs * 32 < k ? (sl + 1) * kbs * 32 : k;
                for (int d = 0; d < s + 2; ++d) g[d] = 0;
                for (int t = 1; t <= s; ++t)
                    for (int u = 1; t + u <= s + 1; ++u) {
                        const int8_t *pa = da + ((size_t)(t - 1) * m + i) * kp;
                        const int8_t *pb = db + ((size_t)(u - 1) * n + j) * kp;
                        int64_t acc = 0;
                        for (int kk = k0; kk < k1; ++kk) acc += (int64_t)pa[kk] * pb[kk];
                        g[t + u] += acc;
                    }
                double h = (double)(int32_t)g[s + 1];
                for (int d = s; d >= 2; --d) h = fma(h, 0.0078125, (double)(int32_t)g[d]);
                const double r = scale2(h, ea[i] + eb[j] - 12);
                v = sl == 0 ? r : v + r;
            }
            C[(size_t)i * ldc + j] = beta_one ? C[(size_t)i * ldc + j] + v : v;
        }
        free(g);
    }
    free(da);
    free(db);
    free(ea);
    free(eb);
    return 0;
}

/* ------------------------------------------------------------------------------------------
 * 6. Ozaki scheme II restatement (the CRT form; Ozaki, Uchino & Imamura 2025, "Ozaki Scheme
 *    II: a GEMM-oriented emulation of floating-point matrix multiplication using an integer
 *    modular technique").  Bit-exact model of the GPU form:
 *
 *    moduli  p_1..p_q: the first q of 256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223,
 *            217, 211, 199, 197, 193 (pairwise coprime), P = p_1 ... p_q, L = bit length of P.
 *    scale   row i of A: e = frexp exponent of max|a_ik|; c_k = max(1, ceil(|a_ik| 2^(22-e)))
 *            for a_ik != 0; S = sum c_k^2 (uint64, so independent of the order);
 *            u = ceil(log2(S) / 2) = (bitlen(S - 1) + 1) / 2; sigma_i = alpha - e + 22 - u, so
 *            2^sigma_i ||a_i||_2 <= 2^alpha.  Columns of B likewise with beta.
 *            alpha = (L - 3) / 2, beta = L - 3 - alpha: by Cauchy-Schwarz every exact integer
 *            product C'_ij = sum_k A'_ik B'_kj of the scaled, rounded operands
 *            A' = rint(2^sigma A), B' = rint(B 2^tau) has |C'_ij| < P / 4.
 *    residues  A'_ik mod p_l as int8 in [-(p-1)/2, (p-1)/2] ([-128, 127] for 256); B' likewise.
 *    products  R_l = (sum_k rA_l rB_l) mod p_l in [0, p_l): exact in int32 for k <= 130816.
 *    CRT     w_l = (P / p_l) ((P / p_l)^-1 mod p_l) < P, cut into three 40-bit chunks
 *            w_l = w1 2^E1 + w2 2^E2 + w3 2^E3 (E_t = L - 40 t); P likewise.
 *            s_t = sum_l w_t,l R_l (exact in FP64: < 16 2^40 2^8 = 2^52),
 *            Q = rint(fma(s2, 2^-40, s1) / P~) is the nearest integer to sum w R / P,
 *            d_t = fma(-Q, P_t, s_t) (exact), c = fma(fma(d1, 2^40, d2), 2^40, d3),
 *            C_ij = c 2^(E3 - sigma_i - tau_j) = C'_ij 2^(-sigma_i - tau_j) to FP64 rounding.
 *    K beyond 130816 is processed in chunks, each scaled on its own and added into C in order.
 * ------------------------------------------------------------------------------------------ */
#define CRT_MAX_MODULI 16
#define CRT_KMAX 130816
static const int crt_moduli[CRT_MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233,
                                               229, 227, 223, 217, 211, 199, 197, 193};

typedef struct {
    int q, L, alpha, beta, E3;
    double w[CRT_MAX_MODULI][3];
    double pc[3];
    double inv_phat;
} crt_consts_t;

static void crt_chunks(unsigned __int128 v, int L, double out[3])
{
    for (int t = 0; t < 3; ++t) {
        const int e = L - 40 * (t + 1);
        unsigned __int128 c;
        if (e >= 0) {
            c = v >> e;
            v -= c << e;
        } else {
            c = v << (-e);
            v = 0;
        }
        out[t] = (double)(uint64_t)c; /* < 2^40 */
    }
}

static int crt_consts(int q, crt_consts_t *K)
{
    if (q < 8 || q > CRT_MAX_MODULI) return 1;
    unsigned __int128 P = 1;
    for (int l = 0; l < q; ++l) P *= (unsigned)crt_moduli[l];
    int L = 0;
    for (unsigned __int128 t = P; t; t >>= 1) ++L;
    K->q = q;
    K->L = L;
    K->alpha = (L - 3) / 2;
    K->beta = L - 3 - K->alpha;
    K->E3 = L - 120;
    for (int l = 0; l < q; ++l) {
        const unsigned p = (unsigned)crt_moduli[l];
        const unsigned __int128 M = P / p;
        const unsigned mm = (unsigned)(M % p);
        unsigned inv = 1;
        while ((mm * inv) % p != 1) ++inv;
        crt_chunks(M * inv, L, K->w[l]);
    }
    crt_chunks(P, L, K->pc);
    K->inv_phat = 1.0 / fma(K->pc[1], 0x1p-40, K->pc[0]);
    return 0;
}

static int bitlen64(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

/* sigma of one row (stride 1) or column (stride ldb) of k values; *nonfinite set on Inf/NaN. */
static int crt_sigma(const double *v, size_t stride, int k, int target, int *nonfinite)
{
    uint64_t mx = 0;
    for (int kk = 0; kk < k; ++kk) {
        uint64_t b;
        memcpy(&b, &v[(size_t)kk * stride], 8);
        b &= 0x7fffffffffffffffull;
        if (b >= 0x7ff0000000000000ull) *nonfinite = 1;
        if (b > mx) mx = b;
    }
    if (mx == 0 || mx >= 0x7ff0000000000000ull) return 0;
    const int e = frexp_exp_bits(mx);
    uint64_t S = 0;
    for (int kk = 0; kk < k; ++kk) {
        const double x = fabs(v[(size_t)kk * stride]);
        if (x == 0.0) continue;
        double c = ceil(scale2(x, 22 - e));
        if (c < 1.0) c = 1.0;
        const uint64_t ci = (uint64_t)c;
        S += ci * ci;
    }
    const int u = (bitlen64(S - 1) + 1) / 2;
    return target - e + 22 - u;
}

/* Symmetric residue of the integer x (|x| < 2^63) modulo p. */
static int8_t crt_residue(int64_t x, int p)
{
    if (p == 256) return (int8_t)(uint8_t)(x & 255);
    int64_t r = x % p;
    if (r < 0) r += p;
    if (r > p / 2) r -= p;
    return (int8_t)r;
}

/* Scale exponents (sigma for the rows of A, tau for the columns of B) of one K range.
 * Returns 1 on non-finite input. */
ORACLE_API int oracle_crt_scales(const double *A, const double *B, int m, int n, int k, int lda, int ldb, int q,
                                 int32_t *sigma, int32_t *tau)
{
    crt_consts_t K;
    if (crt_consts(q, &K)) return 2;
    int nonfinite = 0;
    /* each scale depends on its own row or column only: the loops run in parallel */
#pragma omp parallel for schedule(dynamic, 16) reduction(| : nonfinite)
    for (int i = 0; i < m; ++i) sigma[i] = crt_sigma(A + (size_t)i * lda, 1, k, K.alpha, &nonfinite);
#pragma omp parallel for schedule(dynamic, 16) reduction(| : nonfinite)
    for (int j = 0; j < n; ++j) tau[j] = crt_sigma(B + j, (size_t)ldb, k, K.beta, &nonfinite);
    return nonfinite;
}

/* Residues of A as [l][i][kp] and of B^T as [l][j][kp] (int8, padding zero). */
ORACLE_API void oracle_crt_residues(const double *A, const double *B, int m, int n, int k, int lda, int ldb, int q,
                                    int kp, const int32_t *sigma, const int32_t *tau, int8_t *ra, int8_t *rb)
{
    memset(ra, 0, (size_t)q * m * kp);
    memset(rb, 0, (size_t)q * n * kp);
    /* every residue depends on its own element only: the loops run in parallel */
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < m; ++i)
        for (int kk = 0; kk < k; ++kk) {
            const double a = A[(size_t)i * lda + kk];
            if (!isfinite(a)) continue;
            const int64_t x = (int64_t)nearbyint(scale2(a, sigma[i]));
            for (int l = 0; l < q; ++l) ra[((size_t)l * m + i) * kp + kk] = crt_residue(x, crt_moduli[l]);
        }
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 0; j < n; ++j)
        for (int kk = 0; kk < k; ++kk) {
            const double b = B[(size_t)kk * ldb + j];
            if (!isfinite(b)) continue;
            const int64_t x = (int64_t)nearbyint(scale2(b, tau[j]));
            for (int l = 0; l < q; ++l) rb[((size_t)l * n + j) * kp + kk] = crt_residue(x, crt_moduli[l]);
        }
}

/* The CRT recombination of one output from its residues R[0..q) (each in [0, p_l)). */
static double crt_combine(const crt_consts_t *K, const int32_t *R, int scale)
{
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int l = 0; l < K->q; ++l) {
        const double r = (double)R[l];
        s1 = fma(K->w[l][0], r, s1);
        s2 = fma(K->w[l][1], r, s2);
        s3 = fma(K->w[l][2], r, s3);
    }
    const double Q = nearbyint(fma(s2, 0x1p-40, s1) * K->inv_phat);
    const double d1 = fma(-Q, K->pc[0], s1);
    const double d2 = fma(-Q, K->pc[1], s2);
    const double d3 = fma(-Q, K->pc[2], s3);
    const double c = fma(fma(d1, 0x1p40, d2), 0x1p40, d3);
    return scale2(c, K->E3 + scale);
}

ORACLE_API int oracle_crt_kmax(void) { return CRT_KMAX; }

/* C = (beta_one ? C + v : v), v = A B by the CRT form with q moduli (8..16).  Returns 1 on
 * non-finite input (C untouched), 2 on an unsupported q. */
ORACLE_API int oracle_crt_gemm(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                               int ldc, int q, int beta_one, int nthreads)
{
    nthreads = pick_threads(nthreads);
    crt_consts_t K;
    if (crt_consts(q, &K)) return 2;
    int32_t *sg = (int32_t *)malloc(sizeof(int32_t) * (m > 0 ? m : 1));
    int32_t *tu = (int32_t *)malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    for (int k0 = 0; k0 < k || k0 == 0; k0 += CRT_KMAX) {
        const int kc = (k - k0 < CRT_KMAX) ? k - k0 : CRT_KMAX;
        if (oracle_crt_scales(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, q, sg, tu)) {
            free(sg);
            free(tu);
            return 1;
        }
        const int kp = (kc + 15) & ~15;
        int8_t *ra = (int8_t *)malloc((size_t)q * m * kp + 1);
        int8_t *rb = (int8_t *)malloc((size_t)q * n * kp + 1);
        oracle_crt_residues(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, q, kp, sg, tu, ra, rb);
        const int add = (k0 > 0) || beta_one;
        /* over (i, j) pairs, so that a few rows still use every thread */
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64) collapse(2)
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < n; ++j) {
                int32_t R[CRT_MAX_MODULI];
                for (int l = 0; l < q; ++l) {
                    const int8_t *pa = ra + ((size_t)l * m + i) * kp;
                    const int8_t *pb = rb + ((size_t)l * n + j) * kp;
                    int32_t acc = 0;
                    for (int kk = 0; kk < kc; ++kk) acc += (int32_t)pa[kk] * (int32_t)pb[kk];
                    int32_t r = acc % crt_moduli[l];
                    R[l] = r < 0 ? r + crt_moduli[l] : r;
                }
                const double v = crt_combine(&K, R, -sg[i] - tu[j]);
                C[(size_t)i * ldc + j] = add ? C[(size_t)i * ldc + j] + v : v;
            }
        }
        free(ra);
        free(rb);
        if (k == 0) break;
    }
    free(sg);
    free(tu);
    return 0;
}

/* Number of threads OpenMP will use by default (the host cores this process may run on). */
ORACLE_API int oracle_max_threads(void) { return omp_get_max_threads(); }
