// validate.cu -- result checking on the GPU.
//
// 1. Constant check with validate_C_kernel's rule (1D-row-block/mulmat_kernel.cu:165-222): an
//    element is invalid when |v - expected| > abs_tol AND |v - expected| / |expected| > rel_tol;
//    max absolute and relative error are reported.  The reference resolves its maxima with a
//    compare-and-swap loop per element; here each block reduces in registers and shared memory
//    and issues one atomic per quantity.  Non-finite elements also count as invalid (the
//    reference's comparisons are false for NaN, so it would pass them).
// 2. Error of a computed C against a double-double product (Dot2: TwoProd by FMA, Knuth TwoSum),
//    reduced to normwise, max relative, max componentwise and max absolute error.
#include <cfloat>
#include <cstring>
#include <cmath>

#include "mgx_common.cuh"

namespace mgx {
namespace val {

constexpr int THREADS = 256;

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v)
{
    // For non-negative doubles the IEEE bit pattern orders like the value.
    if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

struct ConstAcc {
    unsigned long long invalid;
    unsigned long long max_abs_bits;
    unsigned long long max_rel_bits;
};

__global__ void __launch_bounds__(THREADS) validate_const_kernel(const double *__restrict__ C, size_t count,
                                                                 double expected, double abs_tol, double rel_tol,
                                                                 ConstAcc *acc)
{
    unsigned long long bad = 0;
    double mabs = 0.0, mrel = 0.0;
    const double aexp = fabs(expected);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const double v = C[i];
        const double ae = fabs(v - expected);
        const double re = (aexp > 0.0) ? ae / aexp : 0.0;
        if ((ae > abs_tol && re > rel_tol) || !isfinite(v)) ++bad;
        if (ae > mabs) mabs = ae;  // NaN compares false: it never enters the maxima
        if (re > mrel) mrel = re;
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
        mabs = fmax(mabs, __shfl_xor_sync(0xffffffffu, mabs, o));
        mrel = fmax(mrel, __shfl_xor_sync(0xffffffffu, mrel, o));
    }
    __shared__ unsigned long long s_bad[THREADS / 32];
    __shared__ double s_abs[THREADS / 32], s_rel[THREADS / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        s_bad[w] = bad;
        s_abs[w] = mabs;
        s_rel[w] = mrel;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < THREADS / 32; ++i) {
            bad += s_bad[i];
            mabs = fmax(mabs, s_abs[i]);
            mrel = fmax(mrel, s_rel[i]);
        }
        if (bad) atomicAdd(&acc->invalid, bad);
        atomic_max_nonneg(&acc->max_abs_bits, mabs);
        atomic_max_nonneg(&acc->max_rel_bits, mrel);
    }
}

// ---------------------------------------------------------------- double-double error check
constexpr int DD_TM = 64, DD_TN = 64, DD_TK = 16;

struct ErrAcc {
    double sum_d2;
    double sum_r2;
    unsigned long long max_rel_bits;
    unsigned long long max_comp_bits;
    unsigned long long max_abs_bits;
};

__global__ void __launch_bounds__(256) dd_error_kernel(const double *__restrict__ A, const double *__restrict__ B,
                                                       const double *__restrict__ C, int m, int n, int k, int lda,
                                                       int ldb, int ldc, int row0, int rows, double floor_abs,
                                                       ErrAcc *acc)
{
    __shared__ double As[DD_TM][DD_TK + 1];
    __shared__ double Bs[DD_TK][DD_TN];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int bm = row0 + blockIdx.y * DD_TM, bn = blockIdx.x * DD_TN;
    double s[4][4], c[4][4], ab[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) s[i][j] = c[i][j] = ab[i][j] = 0.0;
    const int row_end = row0 + rows;
    for (int k0 = 0; k0 < k; k0 += DD_TK) {
        for (int idx = threadIdx.x; idx < DD_TM * DD_TK; idx += 256) {
            const int r = idx / DD_TK, kk = idx % DD_TK;
            const int gr = bm + r, gk = k0 + kk;
            As[r][kk] = (gr < row_end && gk < k) ? A[(size_t)gr * lda + gk] : 0.0;
        }
        for (int idx = threadIdx.x; idx < DD_TK * DD_TN; idx += 256) {
            const int kk = idx / DD_TN, cc = idx % DD_TN;
            const int gk = k0 + kk, gc = bn + cc;
            Bs[kk][cc] = (gk < k && gc < n) ? B[(size_t)gk * ldb + gc] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < DD_TK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[ty + 16 * i][kk];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const double p = a[i] * b[j];
                    const double q = fma(a[i], b[j], -p);
                    const double t = s[i][j] + p;
                    const double z = t - s[i][j];
                    const double e = (s[i][j] - (t - z)) + (p - z);
                    s[i][j] = t;
                    c[i][j] += e + q;
                    ab[i][j] = fma(fabs(a[i]), fabs(b[j]), ab[i][j]);
                }
        }
        __syncthreads();
    }
    double d2 = 0.0, r2 = 0.0, mrel = 0.0, mcomp = 0.0, mabs = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gr = bm + ty + 16 * i, gc = bn + tx + 16 * j;
            if (gr < row_end && gc < n) {
                const double hi = s[i][j] + c[i][j];
                const double lo = c[i][j] - (hi - s[i][j]);
                const double d = (C[(size_t)gr * ldc + gc] - hi) - lo;
                const double ad = fabs(d);
                d2 += d * d;
                r2 += hi * hi;
                mabs = fmax(mabs, ad);
                if (fabs(hi) >= floor_abs && hi != 0.0) mrel = fmax(mrel, ad / fabs(hi));
                if (ab[i][j] > 0.0) mcomp = fmax(mcomp, ad / ab[i][j]);
            }
        }
    for (int o = 16; o > 0; o >>= 1) {
        d2 += __shfl_xor_sync(0xffffffffu, d2, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        mrel = fmax(mrel, __shfl_xor_sync(0xffffffffu, mrel, o));
        mcomp = fmax(mcomp, __shfl_xor_sync(0xffffffffu, mcomp, o));
        mabs = fmax(mabs, __shfl_xor_sync(0xffffffffu, mabs, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc->sum_d2, d2);
        atomicAdd(&acc->sum_r2, r2);
        atomic_max_nonneg(&acc->max_rel_bits, mrel);
        atomic_max_nonneg(&acc->max_comp_bits, mcomp);
        atomic_max_nonneg(&acc->max_abs_bits, mabs);
    }
}

__global__ void max_abs_kernel(const double *__restrict__ C, int rows, int n, int ldc,
                               unsigned long long *out_bits)
{
    double mx = 0.0;
    const size_t total = (size_t)rows * n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / n, cidx = i % n;
        mx = fmax(mx, fabs(C[r * ldc + cidx]));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out_bits, mx);
}

}  // namespace val
}  // namespace mgx

using namespace mgx;

static double bits_to_double(unsigned long long b)
{
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}

int mgx_validate_impl(const double *d_c, size_t count, double expected, double abs_tol, double rel_tol,
                      mgx_validation_t *out, cudaStream_t stream)
{
    val::ConstAcc h{0, 0, 0};
    if (count > 0) {
        val::ConstAcc *d_acc = nullptr;
        {
            const int arc = mgx_scratch_alloc(reinterpret_cast<void **>(&d_acc), sizeof(val::ConstAcc), stream);
            if (arc != MGX_SUCCESS) return arc;
        }
        cudaError_t e = cudaMemsetAsync(d_acc, 0, sizeof(val::ConstAcc), stream);
        if (e == cudaSuccess) {
            size_t blocks = (count + val::THREADS - 1) / val::THREADS;
            const size_t cap = (size_t)mgx_sm_count() * 8;
            if (blocks > cap) blocks = cap;
            val::validate_const_kernel<<<(unsigned)blocks, val::THREADS, 0, stream>>>(d_c, count, expected, abs_tol,
                                                                                      rel_tol, d_acc);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_acc, sizeof h, cudaMemcpyDeviceToHost, stream);
        cudaFreeAsync(d_acc, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            mgx_set_last_cuda_error(e, "constant validation", __FILE__, __LINE__);
            return MGX_E_CUDA;
        }
    }
    out->elements = count;
    out->invalid = h.invalid;
    out->max_abs_error = bits_to_double(h.max_abs_bits);
    out->max_rel_error = bits_to_double(h.max_rel_bits);
    return MGX_SUCCESS;
}

extern "C" MGX_API int mgx_error_vs_dd(const double *A, const double *B, const double *C, int m, int n, int k,
                                       int lda, int ldb, int ldc, int row_start, int row_count, double floor_rel,
                                       mgx_error_t *out)
{
    if (!out || m < 0 || n < 0 || k < 0 || !A || !B || !C || row_start < 0 || row_start > m) {
        mgx_set_last_message("mgx_error_vs_dd: invalid arguments");
        return MGX_E_INVALID;
    }
    int rows = (row_count <= 0) ? m - row_start : row_count;
    if (row_start + rows > m) rows = m - row_start;
    memset(out, 0, sizeof *out);
    if (rows <= 0 || n <= 0) return MGX_SUCCESS;
    struct Scratch {
        val::ErrAcc acc;
        unsigned long long cmax_bits;
    };
    Scratch *d = nullptr;
    cudaStream_t s = nullptr;
    {
        const int arc = mgx_scratch_alloc(reinterpret_cast<void **>(&d), sizeof(Scratch), s);
        if (arc != MGX_SUCCESS) return arc;
    }
    Scratch h;
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(Scratch), s);
    if (e == cudaSuccess) {
        val::max_abs_kernel<<<mgx_sm_count() * 4, 256, 0, s>>>(C + (size_t)row_start * ldc, rows, n, ldc, &d->cmax_bits);
        e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
        const double floor_abs = floor_rel * bits_to_double(h.cmax_bits);
        dim3 grid((n + val::DD_TN - 1) / val::DD_TN, (rows + val::DD_TM - 1) / val::DD_TM);
        val::dd_error_kernel<<<grid, 256, 0, s>>>(A, B, C, m, n, k, lda, ldb, ldc, row_start, rows, floor_abs, &d->acc);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFreeAsync(d, s);
    if (e != cudaSuccess) {
        mgx_set_last_cuda_error(e, "double-double error check", __FILE__, __LINE__);
        return MGX_E_CUDA;
    }
    out->normwise = (h.acc.sum_r2 > 0.0) ? sqrt(h.acc.sum_d2) / sqrt(h.acc.sum_r2) : sqrt(h.acc.sum_d2);
    out->max_rel = bits_to_double(h.acc.max_rel_bits);
    out->max_componentwise = bits_to_double(h.acc.max_comp_bits);
    out->max_abs = bits_to_double(h.acc.max_abs_bits);
    out->rows_checked = (uint64_t)rows;
    return MGX_SUCCESS;
}
