// ozaki_crt.cu -- FP64-accurate GEMM on the INT8 tensor cores by Ozaki scheme II (the CRT form;
// Ozaki, Uchino & Imamura 2025, "Ozaki Scheme II: A GEMM-oriented emulation of floating-point
// matrix multiplication using an integer modular technique").
//
// Where the slice form (ozaki.cu) multiplies s digit slices pairwise (s(s+1)/2 INT8 products),
// this form scales each row of A and column of B by a power of two to integers, takes them modulo
// q pairwise-coprime moduli p_l <= 256, multiplies the residues (one INT8 product per modulus)
// and rebuilds the integer product by the Chinese remainder theorem.  q = 15 moduli give FP64
// accuracy at K = 16384, against 36 products for 8 slices.
//
//   moduli   the first q of 256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211,
//            199, 197, 193; P = p_1 ... p_q, L = bit length of P; alpha = (L-3)/2, beta = L-3-alpha.
//   scale    row i of A: e = frexp exponent of max|a_ik|, c_k = max(1, ceil(|a_ik| 2^(22-e))) for
//            a_ik != 0, S = sum c_k^2 (an integer sum, so the result does not depend on the
//            order), u = (bitlen(S-1)+1)/2, sigma_i = alpha - e + 22 - u; then 2^sigma_i ||a_i||
//            <= 2^alpha.  Columns of B likewise (tau_j, beta).  By Cauchy-Schwarz the exact
//            product C'_ij of A' = rint(2^sigma A) and B' = rint(B 2^tau) is below P/4.
//   residues A' mod p_l as int8 (symmetric; [-128, 127] for 256), B' likewise.
//   products R_l = (A'_l B'_l) mod p_l in [0, p_l), exact in int32 while K <= 130816.
//   CRT      w_l = (P/p_l) ((P/p_l)^-1 mod p_l) in three 40-bit chunks; s_t = sum_l w_t,l R_l is
//            exact in FP64; Q = rint((s1 + s2 2^-40) / P~); d_t = s_t - Q P_t (exact);
//            C_ij = fma(fma(d1, 2^40, d2), 2^40, d3) 2^(E3 - sigma_i - tau_j).
//
// Kernels:
//   crt_row_scale   sigma per row of A (one block per row, integer sum of squares)
//   crt_col_max / crt_col_sumsq / crt_col_scale   tau per column of B (integer atomics)
//   crt_split_a     residues of A as swizzled K-major 256-row slabs [modulus][tile][K block]
//   crt_split_b     residues of B^T, same layout (thread per column, coalesced reads)
//   crt_gemm        persistent tcgen05 kernel over (modulus, 256 x 256 tile) work items:
//       warp 0      producer: one bulk copy per operand per stage (KPACK K blocks); at each new
//                   work item it waits (at most 20 us) until every CTA has started its item, so
//                   the CTAs that share an operand tile read it within microseconds of each
//                   other and mostly from L2 (DRAM reads at N = 16384: 118 -> 48 GB per launch)
//       warp 1      TMEM owner and MMA issuer: two M=128 N=256 K=32 kind::i8 MMAs per K block
//                   (rows 0-127 and 128-255), int32 accumulators in all 512 TMEM columns
//       warps 2-17  epilogue (16 warps, two per accumulator and TMEM lane quarter, 128 columns
//                   each): tcgen05.ld, exact reduction mod p_l (biased Barrett), one byte per output
//   crt_combine     CRT recombination of the q residue planes, scaling, (C +) store
// All waits are bounded (mgx_common.cuh); TMEM is always released before the CTA exits.
#include <cstdio>
#include <cstring>

#include "mgx_common.cuh"

#ifndef MGX_CRT_KPACK
#define MGX_CRT_KPACK 4
#endif
#ifndef MGX_CRT_LOCKSTEP
#define MGX_CRT_LOCKSTEP 1
#endif

namespace mgx {
namespace crt {

constexpr int MAXQ = 16;
constexpr int MINQ = 8;
constexpr int KMAX = 130816;           // 4088 K blocks: k * 128 * 128 < 2^31
constexpr int TILE = 256;              // output tile TILE x TILE, operand slabs TILE rows
constexpr int KB = 32;                 // bytes of K per MMA
constexpr int SLAB = TILE * KB;        // 8 KiB: one operand, one K block
constexpr int KPACK = MGX_CRT_KPACK;   // K blocks per pipeline stage
constexpr int STAGE_BYTES = 2 * KPACK * SLAB;
constexpr int STAGES = (232448 - 1280) / STAGE_BYTES;   // 227 KiB of shared memory per CTA
#ifndef MGX_CRT_EPI_WARPS
#define MGX_CRT_EPI_WARPS 16
#endif
constexpr int EPI_WARPS = MGX_CRT_EPI_WARPS;   // 8 or 16: one or two warps per (accumulator, TMEM lane quarter)
constexpr int COL_SPLIT = EPI_WARPS / 8;       // warps sharing the 256 columns of one accumulator's lane quarter
constexpr int EPI_CHUNKS = 8 / COL_SPLIT;      // 32-column chunks each epilogue warp drains
static_assert(EPI_WARPS == 8 || EPI_WARPS == 16, "epilogue warps");
constexpr int THREADS = (2 + EPI_WARPS) * 32;
constexpr int NONFINITE = 0x7fffffff;
constexpr int OUT_TILE_BYTES = TILE * TILE;   // one residue byte per output
#ifndef MGX_CRT_RASTER
#define MGX_CRT_RASTER 16
#endif
constexpr int RASTER = MGX_CRT_RASTER;

static_assert(STAGES >= 2 && STAGES <= 8, "pipeline depth");

__constant__ int c_moduli[MAXQ] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};
static const int h_moduli[MAXQ] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};

// Host-computed constants of one modulus set.
struct Consts {
    int q, L, alpha, beta, E3;
    double w[MAXQ][3];     // CRT weights in 40-bit chunks
    double pc[3];          // P in 40-bit chunks
    double inv_phat;       // 1 / (P / 2^(L-40))
    double c32[MAXQ];      // 2^32 mod p_l
    double inv_p[MAXQ];    // 1 / p_l (rounded)
    uint32_t barrett[MAXQ];  // ceil(2^32 / p_l)
};

// ---------------------------------------------------------------- shared numerics
__host__ __device__ __forceinline__ int frexp_exp_bits(unsigned long long absbits)
{
    if (absbits == 0) return 0;
    const int biased = (int)(absbits >> 52);
    if (biased != 0) return biased - 1022;
    const unsigned long long mant = absbits & ((1ull << 52) - 1);
#ifdef __CUDA_ARCH__
    return -1022 - (__clzll((long long)mant) - 12);
#else
    return -1022 - (__builtin_clzll(mant) - 12);
#endif
}

__device__ __forceinline__ double pow2i(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

__device__ __forceinline__ double scale2(double x, int e)
{
    if (e >= -1022 && e <= 1023) return __dmul_rn(x, pow2i(e));
    const int e1 = e / 2, e2 = e - e1;
    return __dmul_rn(__dmul_rn(x, pow2i(e1)), pow2i(e2));
}

// 2^e as f1 f2, the factors scale2 multiplies by (f2 = 1 when one factor is enough).
__device__ __forceinline__ void scale_factors(int e, double &f1, double &f2)
{
    if (e >= -1022 && e <= 1023) {
        f1 = pow2i(e);
        f2 = 1.0;
    } else {
        const int e1 = e / 2;
        f1 = pow2i(e1);
        f2 = pow2i(e - e1);
    }
}

// ceil(|x| 2^(22-e))^2 for x != 0 (at least 1), 0 for x == 0, with 2^(22-e) = f1 f2 as
// scale_factors gives it (the same products as scale2).  |x| < 2^e, so the ceiling is an integer
// in [1, 2^22]: its low 32 bits come from 2^52 + c, and the square is one 32 x 32 -> 64 multiply.
__device__ __forceinline__ unsigned long long sq_term(double x, double f1, double f2)
{
    const double ax = fabs(x);
    if (ax == 0.0) return 0ull;
    double c = ceil(__dmul_rn(__dmul_rn(ax, f1), f2));
    if (c < 1.0) c = 1.0;
    const uint32_t ci = (uint32_t)__double2loint(__dadd_rn(c, 4503599627370496.0));
    return (unsigned long long)ci * ci;
}

// Scale exponent from the exponent of the maximum and the integer sum of squares.
__device__ __forceinline__ int sigma_of(unsigned long long mx, unsigned long long S, int target)
{
    if (mx == 0) return 0;
    const int e = frexp_exp_bits(mx);
    const int bl = (S - 1) ? 64 - __clzll((long long)(S - 1)) : 0;
    return target - e + 22 - (bl + 1) / 2;
}

// ---------------------------------------------------------------- scale kernels
// One block of ROW_THREADS per row: the row's maximum, then its integer sum of squares.  The
// second pass finds the row in L2: at 4 blocks per SM, 592 rows (77 MB at k = 16384) are in
// flight, against L2's 126 MB, so A is read from DRAM once.
constexpr int ROW_THREADS = 512;

__global__ void __launch_bounds__(ROW_THREADS) crt_row_scale(const double *__restrict__ A, int m, int k, int lda,
                                                             int target, int *__restrict__ sg, int *status)
{
    __shared__ unsigned long long red[ROW_THREADS / 32];
    __shared__ unsigned long long row_max;
    const int row = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (row >= m) return;
    const double *r = A + (size_t)row * lda;
    const unsigned long long *rb = reinterpret_cast<const unsigned long long *>(r);
    unsigned long long mx = 0;
    for (int kk = threadIdx.x; kk < k; kk += ROW_THREADS) {
        const unsigned long long b = __ldg(rb + kk) & 0x7fffffffffffffffull;
        mx = b > mx ? b : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = other > mx ? other : mx;
    }
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (warp == 0) {
        mx = lane < ROW_THREADS / 32 ? red[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = other > mx ? other : mx;
        }
        if (lane == 0) row_max = mx;
    }
    __syncthreads();
    mx = row_max;
    if (mx >= 0x7ff0000000000000ull) {
        if (threadIdx.x == 0) {
            sg[row] = NONFINITE;
            record_status(status, kDevNonFinite);
        }
        return;
    }
    const int e = frexp_exp_bits(mx);
    double f1, f2;
    scale_factors(22 - e, f1, f2);
    unsigned long long S = 0;  // an exact integer sum: the order of its terms does not matter
    if (mx != 0) {
        int kk = threadIdx.x;
        for (; kk + 3 * ROW_THREADS < k; kk += 4 * ROW_THREADS) {
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = __ldg(r + kk + u * ROW_THREADS);
#pragma unroll
            for (int u = 0; u < 4; ++u) S += sq_term(v[u], f1, f2);
        }
        for (; kk < k; kk += ROW_THREADS) S += sq_term(__ldg(r + kk), f1, f2);
    }
    for (int o = 16; o > 0; o >>= 1) S += __shfl_xor_sync(0xffffffffu, S, o);
    if (lane == 0) red[warp] = S;   // warp 0 read red[] before the barrier above
    __syncthreads();
    if (warp == 0) {
        S = lane < ROW_THREADS / 32 ? red[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) S += __shfl_xor_sync(0xffffffffu, S, o);
        if (lane == 0) sg[row] = sigma_of(mx, S, target);
    }
}

// grid (ceil(n/256), ychunks); each thread scans a run of rows of one column.
__global__ void crt_col_max(const double *__restrict__ B, int k, int n, int ldb, unsigned long long *colmax)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int rows_per = (k + gridDim.y - 1) / gridDim.y;
    const int r0 = blockIdx.y * rows_per;
    const int r1 = min(k, r0 + rows_per);
    unsigned long long mx = 0;
    const unsigned long long *b = reinterpret_cast<const unsigned long long *>(B);
    for (int r = r0; r < r1; ++r) {
        const unsigned long long v = __ldg(b + (size_t)r * ldb + j) & 0x7fffffffffffffffull;
        mx = v > mx ? v : mx;
    }
    if (mx) atomicMax(colmax + j, mx);
}

__global__ void crt_col_sumsq(const double *__restrict__ B, int k, int n, int ldb,
                              const unsigned long long *__restrict__ colmax, unsigned long long *colsum)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long mx = colmax[j];
    if (mx == 0 || mx >= 0x7ff0000000000000ull) return;
    const int e = frexp_exp_bits(mx);
    double f1, f2;
    scale_factors(22 - e, f1, f2);
    const int rows_per = (k + gridDim.y - 1) / gridDim.y;
    const int r0 = blockIdx.y * rows_per;
    const int r1 = min(k, r0 + rows_per);
    unsigned long long S = 0;  // an exact integer sum: the order of its terms does not matter
    int r = r0;
    for (; r + 8 <= r1; r += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldg(B + (size_t)(r + u) * ldb + j);
#pragma unroll
        for (int u = 0; u < 8; ++u) S += sq_term(v[u], f1, f2);
    }
    for (; r < r1; ++r) S += sq_term(__ldg(B + (size_t)r * ldb + j), f1, f2);
    if (S) atomicAdd(colsum + j, S);
}

__global__ void crt_col_scale(const unsigned long long *__restrict__ colmax, const unsigned long long *__restrict__ colsum,
                              int n, int target, int *__restrict__ tu, int *status)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long mx = colmax[j];
    if (mx >= 0x7ff0000000000000ull) {
        tu[j] = NONFINITE;
        record_status(status, kDevNonFinite);
    } else {
        tu[j] = sigma_of(mx, colsum[j], target);
    }
}

// ---------------------------------------------------------------- residue kernels
// Residues of one value: x = rint(v 2^sg) (|x| < 2^63) is split exactly into xh 2^32 + xl
// (xl in [0, 2^32)); for each modulus y = xh (2^32 mod p) + xl (|y| < 2^40, exact) and
// r = y - p rint(y / p), in [-(p-1)/2, (p-1)/2] for odd p, +-128 for 256.  A double
// 1.5 * 2^52 + z with |z| < 2^51 an integer holds z mod 2^32 in its low word, so
//   Y = fma(xh, c, xl + 1.5 * 2^52)   (exact)      -> low word y mod 2^32
//   y = Y - 1.5 * 2^52                (exact)
//   t = fma(y, 1/p, 1.5 * 2^52)       (one rounding) -> low word rint(y / p): y / p is never
//       within 2^-9 of a half-integer for odd p, far above the error of the rounded 1/p
// and r = lo(Y) - p lo(t) in 32-bit arithmetic (r is small, so the wrap-around cancels).
// The kernels split 8 values first (split32) and then run each modulus over all 8
// (residue_word): a modulus's constants are read once per 8 values, and the 8 residue bytes
// pack into two words with byte permutes.
constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52

// x = rint(v 2^sg) as xh 2^32 + xl; returns xh and xl + 1.5 * 2^52.
__device__ __forceinline__ void split32(double v, double f1, double f2, double &xh, double &xr)
{
    const double x = rint(__dmul_rn(__dmul_rn(v, f1), f2));
    xh = floor(__dmul_rn(x, 2.3283064365386963e-10));  // x * 2^-32
    xr = __dadd_rn(__fma_rn(-xh, 4294967296.0, x), kRound);
}

// The residue mod p as the low byte of the returned word (c = 2^32 mod p, ip = 1/p).
__device__ __forceinline__ uint32_t residue_word(double xh, double xr, double c, double ip, uint32_t p)
{
    const double Y = __fma_rn(xh, c, xr);
    const double t = __fma_rn(__dsub_rn(Y, kRound), ip, kRound);
    return (uint32_t)__double2loint(Y) - (uint32_t)__double2loint(t) * p;
}

// Low bytes of a, b, c, d as one word (a in the lowest byte).
__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// The 8 residue bytes of xh/xr[0..7] for modulus l, element j in byte j.
__device__ __forceinline__ uint2 residues8(const double (&xh)[8], const double (&xr)[8], const Consts &K, int l)
{
    const double c = K.c32[l], ip = K.inv_p[l];
    const uint32_t p = (uint32_t)c_moduli[l];
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) w[j] = residue_word(xh[j], xr[j], c, ip, p);
    return make_uint2(pack4(w[0], w[1], w[2], w[3]), pack4(w[4], w[5], w[6], w[7]));
}

// Slab layout: byte (row r, k byte c) of K block kb of 256-row tile t of modulus l sits at
// l * mod_stride + (t * kblocks + kb) * 8192 + r * 32 + (c ^ (((r >> 2) & 1) << 4)) -- the
// 32-byte swizzled K-major image the MMA reads, so a stage is one contiguous bulk copy.
__device__ __forceinline__ size_t slab_offset(int tile, int kb, int kblocks, int r, int c)
{
    return ((size_t)tile * kblocks + kb) * (size_t)SLAB + (size_t)r * 32 + (c ^ (((r >> 2) & 1) << 4));
}

// Block: 64 rows of A x one 32-wide K block; warp w takes rows 8w..8w+7, lane -> row (lane / 4)
// and 8 consecutive k (lane % 4), so four lanes read one 256-byte row segment and write the 32
// residue bytes of that row, one 8-byte store each per modulus.
template <int Q>
__global__ void __launch_bounds__(256, 3) crt_split_a(const double *__restrict__ A, int m, int k, int lda, int mp,
                                                      int kblocks, const int *__restrict__ sg, uint8_t *__restrict__ ra,
                                                      size_t mod_stride, const __grid_constant__ Consts K)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kb = blockIdx.y;
    const int row = blockIdx.x * 64 + warp * 8 + (lane >> 2), kq = lane & 3;
    if (row >= mp) return;
    const int k0 = kb * 32 + kq * 8;
    int s = (row < m) ? sg[row] : 0;
    const bool live = row < m && s != NONFINITE;
    if (!live) s = 0;
    double f1, f2;
    scale_factors(s, f1, f2);
    const double *arow = A + (size_t)(live ? row : 0) * lda;
    double xh[8], xr[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int kk = k0 + j;
        double v = (live && kk < k) ? __ldg(arow + kk) : 0.0;
        if (!isfinite(v)) v = 0.0;
        split32(v, f1, f2, xh[j], xr[j]);
    }
    const size_t off = slab_offset(row / TILE, kb, kblocks, row % TILE, kq * 8);
#pragma unroll
    for (int l = 0; l < Q; ++l)
        *reinterpret_cast<uint2 *>(ra + (size_t)l * mod_stride + off) = residues8(xh, xr, K, l);
}

// Block: 64 consecutive columns of B x one 32-wide K block.  Warp w takes 32 of the columns
// (lane = column, so every load is one coalesced 256-byte row segment) and K quarter w % 4
// (8 consecutive k).  The 8 residue bytes of each (column, quarter) go to their swizzled place
// in a shared-memory copy of the block's slab rows; the 64 rows x 32 bytes of each modulus are
// one contiguous 2 KiB run of the slab (column j of B is row j % 256 of slab tile j / 256),
// written out with 16-byte stores.
template <int Q>
__global__ void __launch_bounds__(256, 3) crt_split_b(const double *__restrict__ B, int k, int n, int ldb, int kblocks,
                                                      const int *__restrict__ tu, uint8_t *__restrict__ rb,
                                                      size_t mod_stride, const __grid_constant__ Consts K)
{
    __shared__ __align__(16) unsigned char st[Q][64 * 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kb = blockIdx.y, kq = warp & 3;
    const int rl = (warp >> 2) * 32 + lane;          // row of the block's 64
    const int col = blockIdx.x * 64 + rl;
    int s = (col < n) ? tu[col] : 0;
    const bool live = col < n && s != NONFINITE;
    if (!live) s = 0;
    const double *bcol = B + (live ? col : 0);
    double f1, f2;
    scale_factors(s, f1, f2);
    double xh[8], xr[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int kk = kb * 32 + kq * 8 + j;
        double v = (live && kk < k) ? __ldg(bcol + (size_t)kk * ldb) : 0.0;
        if (!isfinite(v)) v = 0.0;
        split32(v, f1, f2, xh[j], xr[j]);
    }
    const int soff = rl * 32 + ((kq * 8) ^ (((rl >> 2) & 1) << 4));
#pragma unroll
    for (int l = 0; l < Q; ++l) *reinterpret_cast<uint2 *>(&st[l][soff]) = residues8(xh, xr, K, l);
    __syncthreads();
    const int c0 = blockIdx.x * 64;
    unsigned char *dst = rb + ((size_t)(c0 / TILE) * kblocks + kb) * (size_t)SLAB + (size_t)(c0 % TILE) * 32;
    for (int idx = threadIdx.x; idx < Q * 128; idx += 256) {
        const int l = idx >> 7, o = (idx & 127) * 16;
        *reinterpret_cast<uint4 *>(dst + (size_t)l * mod_stride + o) = *reinterpret_cast<const uint4 *>(&st[l][o]);
    }
}

// ---------------------------------------------------------------- tcgen05 helpers
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// K-major operand tile (rows 32 bytes apart) with the 32-byte swizzle: groups of 8 rows 256 B
// apart (SBO), LBO unused (1), descriptor version 1, layout type 6.
__device__ __forceinline__ uint64_t sw32_desc(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(256 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)6 << 61;
    return d;
}

// kind::i8 instruction descriptor: D s32, A s8, B s8, both K-major, M = 128, N = 256.
constexpr uint32_t IDESC_S8_128x256 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) |
                                      ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// g mod p in [0, p) for any int32 g: Barrett with M = ceil(2^32 / p) on |g| gives floor(|g|/p)
// or one more (the error of M is below 2^31 / 2^32), corrected by one add; then the sign.
// Checked exhaustively over all int32 for every modulus of the set.
__device__ __forceinline__ uint32_t mod_p(int32_t g, uint32_t p, uint32_t M)
{
    const uint32_t a = g < 0 ? 0u - (uint32_t)g : (uint32_t)g;
    const uint32_t qq = __umulhi(a, M);
    int32_t r = (int32_t)(a - qq * p);
    if (r < 0) r += (int32_t)p;
    return (g >= 0 || r == 0) ? (uint32_t)r : p - (uint32_t)r;
}

// g mod p in [0, p) for an accumulator of K <= KMAX int8 x int8 products (|g| <= 2^14 K <
// 2^31 - 2^22): a = g + bias with bias = p floor(2^31 / p) lies in (0, 2^32) and a = g (mod p).
// Barrett with M = ceil(2^32 / p) gives q = floor(a / p) or one more, so r = a - q p is the
// residue or the residue minus p (wrapped); the unsigned min of r and r + p is the residue.
__device__ __forceinline__ uint32_t mod_p_acc(uint32_t g, uint32_t p, uint32_t M, uint32_t bias)
{
    const uint32_t a = g + bias;
    const uint32_t r = a - __umulhi(a, M) * p;
    return min(r, r + p);
}

struct GemmParams {
    const uint8_t *ra, *rb;   // residue slabs [modulus][tile][K block][256 x 32 B], at the block's first tile
    uint8_t *rc;              // output residues [modulus][tile row][tile column][64 KiB], at the block's first tile
    size_t ra_mod, rb_mod, rc_mod;
    int tiles_m, tiles_n;     // tiles of this block of the product
    int rc_tile_ld;           // tiles per row of the residue planes (the whole product's)
    int kblocks, q;
    int ksplit;               // K slices per (modulus, tile): 1, or the split-K form's count
    int kb_split;             // K blocks per slice
    size_t rc_slice;          // bytes between the residue planes of consecutive K slices
    int *status;
    unsigned int *sync;       // this launch's arrival counter (zeroed before the launch), or nullptr
    uint32_t barrett[MAXQ];
    uint32_t bias[MAXQ];      // p floor(2^31 / p), for mod_p_acc
};

// Work item w: modulus w / (tiles), then groups of RASTER tile rows sweeping the columns
// together (the group's rows of A stay in L2 while each column tile of B is read once per group).
__device__ __forceinline__ void item_of(const GemmParams &p, int w, int &l, int &tm, int &tn, int &ks)
{
    ks = w % p.ksplit;       // K slice (consecutive items: the same tile's slices)
    w /= p.ksplit;
    const int per = p.tiles_m * p.tiles_n;
    l = w / per;
    const int t = w - l * per;
    const int per_group = RASTER * p.tiles_n;
    const int g = t / per_group, r = t % per_group;
    const int first = g * RASTER;
    const int gsize = min(p.tiles_m - first, RASTER);
    tm = first + r % gsize;
    tn = r / gsize;
}

__global__ void __launch_bounds__(THREADS, 1) crt_gemm(const __grid_constant__ GemmParams p)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                            ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;
    uint64_t *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int items = p.q * p.tiles_m * p.tiles_n * p.ksplit;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, EPI_WARPS);
        mbar_init(drain, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ bulk-copy producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int armed[STAGES];
            for (int s = 0; s < STAGES; ++s) armed[s] = -1;
            bool ok = true;
            for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
                int l, tm, tn, ks;
                item_of(p, w, l, tm, tn, ks);
                const int kb_begin = ks * p.kb_split, kb_end = min(p.kblocks, kb_begin + p.kb_split);
#if MGX_CRT_LOCKSTEP
                // Soft lockstep: CTAs that share an operand tile read it from L2 only while they
                // stay within a few microseconds of each other, so every producer waits at each
                // new item until all CTAs have started theirs -- or 20 us, then goes on anyway.
                // Nothing depends on it for correctness, so it cannot deadlock (two launches that
                // share the GPU just wait out the 20 us).
                if (p.sync) {
                    atomicAdd(p.sync, 1u);
                    const unsigned int target = (unsigned int)min((long long)(w / gridDim.x + 1) * gridDim.x,
                                                                  (long long)items);
                    const unsigned long long t0 = global_ns();
                    while (*reinterpret_cast<volatile unsigned int *>(p.sync) < target &&
                           global_ns() - t0 < 20000ull)
                        __nanosleep(64);
                }
#endif
                const uint8_t *ga = p.ra + (size_t)l * p.ra_mod + (size_t)tm * p.kblocks * SLAB;
                const uint8_t *gb = p.rb + (size_t)l * p.rb_mod + (size_t)tn * p.kblocks * SLAB;
                for (int kb0 = kb_begin; kb0 < kb_end; kb0 += KPACK) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, p.status, kDevTimeoutEmpty)) {
                        ok = false;
                        break;
                    }
                    const int nkb = min(KPACK, kb_end - kb0);
                    const uint32_t bytes = (uint32_t)(nkb * SLAB);
                    unsigned char *sa = smem + stage * STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], 2u * bytes);
                    armed[stage] = (int)phase;
                    bulk_load(sa, ga + (size_t)kb0 * SLAB, bytes, &full[stage]);
                    bulk_load(sa + KPACK * SLAB, gb + (size_t)kb0 * SLAB, bytes, &full[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            for (int s = 0; s < STAGES; ++s)
                if (armed[s] >= 0) mbar_wait_bounded(&full[s], (uint32_t)armed[s], p.status, kDevTimeoutFull);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true;
            const uint32_t smem_base = smem_u32(smem);
            for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
                if (!mbar_wait_bounded(acc_empty, acc_phase ^ 1u, p.status, kDevTimeoutAcc)) {
                    ok = false;
                    break;
                }
                acc_phase ^= 1u;
                tc_fence_after();
                const int kb_begin = (w % p.ksplit) * p.kb_split, kb_end = min(p.kblocks, kb_begin + p.kb_split);
                for (int kb0 = kb_begin; kb0 < kb_end; kb0 += KPACK) {
                    if (!mbar_wait_bounded(&full[stage], phase, p.status, kDevTimeoutFull)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const int nkb = min(KPACK, kb_end - kb0);
                    const uint32_t sa = smem_base + stage * STAGE_BYTES;
                    const uint64_t a0 = sw32_desc(sa), b0 = sw32_desc(sa + KPACK * SLAB);
#pragma unroll
                    for (int j = 0; j < KPACK; ++j) {
                        if (j < nkb) {
                            const uint32_t acc = (kb0 + j > kb_begin) ? 1u : 0u;
                            const uint64_t bj = b0 + (uint64_t)((j * SLAB) >> 4);
                            tc_mma_i8(tmem_base, a0 + (uint64_t)((j * SLAB) >> 4), bj, IDESC_S8_128x256, acc);
                            tc_mma_i8(tmem_base + 256, a0 + (uint64_t)((j * SLAB + SLAB / 2) >> 4), bj,
                                      IDESC_S8_128x256, acc);
                        }
                    }
                    tc_commit(&empty[stage]);  // frees the stage once these MMAs have read it
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (ok) tc_commit(acc_full);
            }
            // Drain: all MMAs this thread issued have finished before TMEM is released.
            tc_commit(drain);
            mbar_wait_bounded(drain, 0, p.status, kDevTimeoutAcc);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..)
        const int qd = warp & 3;            // TMEM lane quarter this warp may access
        const int h = ((warp - 2) >> 2) & 1;  // accumulator: tile rows 0-127 or 128-255
        const int c0 = ((warp - 2) >> 3) * EPI_CHUNKS;  // first 32-column chunk of this warp
        uint32_t acc_phase = 0;
        for (int w = blockIdx.x; w < items; w += gridDim.x) {
            bool got = true;
            if (lane == 0) got = mbar_wait_sleepy(acc_full, acc_phase, p.status, kDevTimeoutAcc);
            got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
            if (!got) break;
            acc_phase ^= 1u;
            tc_fence_after();
            int l, tm, tn, ks;
            item_of(p, w, l, tm, tn, ks);
            const uint32_t pm = (uint32_t)c_moduli[l], M = p.barrett[l], bias = p.bias[l];
            uint8_t *dst = p.rc + (size_t)ks * p.rc_slice + (size_t)l * p.rc_mod +
                           ((size_t)tm * p.rc_tile_ld + tn) * OUT_TILE_BYTES +
                           (size_t)((h * 4 + qd) * 32) * 256 + lane * 8;
            const uint32_t tbase = tmem_base + ((uint32_t)(32 * qd) << 16) + h * 256;
            // two 32-column loads in flight per wait, then their reduction and stores
#pragma unroll 1
            for (int c = c0; c < c0 + EPI_CHUNKS; c += 2) {
                uint32_t r[2][32];
                tmem_ld32(tbase + c * 32, r[0]);
                tmem_ld32(tbase + (c + 1) * 32, r[1]);
                tmem_wait_ld();
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    uint32_t pk[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        pk[j] = mod_p_acc(r[b][4 * j], pm, M, bias) | (mod_p_acc(r[b][4 * j + 1], pm, M, bias) << 8) |
                                (mod_p_acc(r[b][4 * j + 2], pm, M, bias) << 16) |
                                (mod_p_acc(r[b][4 * j + 3], pm, M, bias) << 24);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        *reinterpret_cast<uint2 *>(dst + (size_t)(4 * (c + b) + u) * 256) =
                            make_uint2(pk[2 * u], pk[2 * u + 1]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty);
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    __syncwarp();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512) : "memory");
}

// ---------------------------------------------------------------- CRT recombination
// Product residues of one 256 x 256 tile are stored [h][quarter][8-column chunk][lane][8 B]: the
// epilogue warp of TMEM lane quarter `quarter` and accumulator h writes 256 contiguous bytes per
// chunk.  One warp here takes one (tile, h, quarter, chunk): lane = row within the quarter,
// 8 columns.  beta_one: C (+)= result.
struct CombineParams {
    const uint8_t *rc;        // the block's first tile of the residue planes
    size_t rc_mod;
    int ksplit;               // K slices whose residues are added mod p first (1: none)
    size_t rc_slice;          // bytes between the residue planes of consecutive K slices
    double *C;                // the block's first element of C
    int m, n, ldc, tiles_n, rc_tile_ld, beta_one, vec_store;
    const int *sg, *tu;
    Consts K;
};

// SPLITK: the residue planes of p.ksplit K slices are added modulo p first (a separate
// instantiation with a larger register budget, so the whole-K kernel keeps its own).
template <int Q, bool SPLITK>
__global__ void __launch_bounds__(256, SPLITK ? 2 : 3) crt_combine(const __grid_constant__ CombineParams p, long long units)
{
    const int lane = threadIdx.x & 31;
    const long long unit = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (unit >= units) return;
    const int c = (int)(unit & 31), qd = (int)((unit >> 5) & 3), h = (int)((unit >> 7) & 1);
    const long long tile = unit >> 8;
    const int tm = (int)(tile / p.tiles_n), tn = (int)(tile % p.tiles_n);
    const int row = tm * TILE + h * 128 + qd * 32 + lane;
    const int col0 = tn * TILE + c * 8;
    if (row >= p.m || col0 >= p.n) return;
    const uint8_t *src = p.rc + ((size_t)tm * p.rc_tile_ld + tn) * OUT_TILE_BYTES +
                         (size_t)((h * 4 + qd) * 32 + c) * 256 + lane * 8;
    double s1[8], s2[8], s3[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) s1[j] = s2[j] = s3[j] = 0.0;
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        uint32_t res[8];
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(src + (size_t)l * p.rc_mod));
#pragma unroll
        for (int j = 0; j < 8; ++j) res[j] = ((j < 4 ? v.x : v.y) >> (8 * (j & 3))) & 255u;
        if (SPLITK) {
            // the slices' residues (each < p) add modulo p
            for (int t = 1; t < p.ksplit; ++t) {
                const uint2 u = __ldg(reinterpret_cast<const uint2 *>(src + (size_t)t * p.rc_slice + (size_t)l * p.rc_mod));
#pragma unroll
                for (int j = 0; j < 8; ++j) res[j] += ((j < 4 ? u.x : u.y) >> (8 * (j & 3))) & 255u;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) res[j] = mod_p((int32_t)res[j], (uint32_t)c_moduli[l], p.K.barrett[l]);
        }
        const double w1 = p.K.w[l][0], w2 = p.K.w[l][1], w3 = p.K.w[l][2];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            // (double) of a residue: 2^52 + r from the bit pattern, minus 2^52 (exact)
            const double r = __dsub_rn(__hiloint2double(0x43300000, res[j]), 4503599627370496.0);
            s1[j] = __fma_rn(w1, r, s1[j]);
            s2[j] = __fma_rn(w2, r, s2[j]);
            s3[j] = __fma_rn(w3, r, s3[j]);
        }
    }
    const int srow = p.sg[row];
    double *crow = p.C + (size_t)row * p.ldc;
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
        double v[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int col = col0 + j + u;
            const int scol = col < p.n ? p.tu[col] : 0;
            const double Qd = rint(__dmul_rn(__fma_rn(s2[j + u], 0x1p-40, s1[j + u]), p.K.inv_phat));
            const double d1 = __fma_rn(-Qd, p.K.pc[0], s1[j + u]);
            const double d2 = __fma_rn(-Qd, p.K.pc[1], s2[j + u]);
            const double d3 = __fma_rn(-Qd, p.K.pc[2], s3[j + u]);
            const double cc = __fma_rn(__fma_rn(d1, 0x1p40, d2), 0x1p40, d3);
            v[u] = (srow == NONFINITE || scol == NONFINITE) ? __longlong_as_double(0x7ff8000000000000ll)
                                                            : scale2(cc, p.K.E3 - srow - scol);
        }
        const int col = col0 + j;
        if (col + 1 < p.n && p.vec_store) {
            double2 *dst = reinterpret_cast<double2 *>(crow + col);
            if (p.beta_one) {
                const double2 o = *dst;
                v[0] = __dadd_rn(o.x, v[0]);
                v[1] = __dadd_rn(o.y, v[1]);
            }
            *dst = make_double2(v[0], v[1]);
        } else {
            if (col < p.n) crow[col] = p.beta_one ? __dadd_rn(crow[col], v[0]) : v[0];
            if (col + 1 < p.n) crow[col + 1] = p.beta_one ? __dadd_rn(crow[col + 1], v[1]) : v[1];
        }
    }
}

// ---------------------------------------------------------------- host constants
static void chunks40(unsigned __int128 v, int L, double out[3])
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
        out[t] = (double)(uint64_t)c;
    }
}

static bool make_consts(int q, Consts &K)
{
    if (q < MINQ || q > MAXQ) return false;
    memset(&K, 0, sizeof K);
    unsigned __int128 P = 1;
    for (int l = 0; l < q; ++l) P *= (unsigned)h_moduli[l];
    int L = 0;
    for (unsigned __int128 t = P; t; t >>= 1) ++L;
    K.q = q;
    K.L = L;
    K.alpha = (L - 3) / 2;
    K.beta = L - 3 - K.alpha;
    K.E3 = L - 120;
    for (int l = 0; l < q; ++l) {
        const unsigned p = (unsigned)h_moduli[l];
        const unsigned __int128 M = P / p;
        const unsigned mm = (unsigned)(M % p);
        unsigned inv = 1;
        while ((mm * inv) % p != 1) ++inv;
        chunks40(M * inv, L, K.w[l]);
        K.c32[l] = (double)((1ull << 32) % p);
        K.inv_p[l] = 1.0 / (double)p;
        K.barrett[l] = (uint32_t)(0xffffffffull / p + 1);
    }
    chunks40(P, L, K.pc);
    K.inv_phat = 1.0 / fma(K.pc[1], 0x1p-40, K.pc[0]);
    return true;
}

}  // namespace crt
}  // namespace mgx

using namespace mgx;

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct CrtLayout {
    size_t ra, rb, rc, sg, tu, colmax, colsum, sync, total;
    size_t ra_mod, rb_mod, rc_mod;
    int kblocks, tiles_m, tiles_n;
    int ksplit, kb_split;   // K slices (1: whole K) and K blocks per slice
};

// Workspace of one K range of at most KMAX: residue slabs of A and B^T (rows rounded up to 256,
// K to 32), the residue planes of the product, the scale exponents and the column sums.
// With ksplit > 1 (the split-K form, k <= KMAX) the 32-wide K blocks are cut into slices of
// ceil(kblocks / ksplit) blocks, and the product residues get one set of planes per slice.
CrtLayout crt_layout(int m, int n, int k, int q, int ksplit = 1)
{
    CrtLayout L;
    int kc = k < crt::KMAX ? k : crt::KMAX;
    L.kblocks = (kc + 31) / 32;
    if (L.kblocks == 0) L.kblocks = 1;
    if (ksplit < 1) ksplit = 1;
    if (ksplit > L.kblocks) ksplit = L.kblocks;
    L.kb_split = (L.kblocks + ksplit - 1) / ksplit;
    L.ksplit = (L.kblocks + L.kb_split - 1) / L.kb_split;
    L.tiles_m = (m + crt::TILE - 1) / crt::TILE;
    L.tiles_n = (n + crt::TILE - 1) / crt::TILE;
    L.ra_mod = (size_t)L.tiles_m * L.kblocks * crt::SLAB;
    L.rb_mod = (size_t)L.tiles_n * L.kblocks * crt::SLAB;
    L.rc_mod = (size_t)L.tiles_m * L.tiles_n * crt::OUT_TILE_BYTES;
    size_t off = 0;
    L.ra = off;
    off = align256(off + (size_t)q * L.ra_mod);
    L.rb = off;
    off = align256(off + (size_t)q * L.rb_mod);
    L.rc = off;
    off = align256(off + (size_t)q * L.rc_mod * L.ksplit);
    L.sg = off;
    off = align256(off + sizeof(int) * (size_t)m);
    L.tu = off;
    off = align256(off + sizeof(int) * (size_t)n);
    L.colmax = off;
    off = align256(off + sizeof(unsigned long long) * (size_t)n);
    L.colsum = off;
    off = align256(off + sizeof(unsigned long long) * (size_t)n);
    L.sync = off;                       // arrival counters of the products launches (two slots)
    off = align256(off + 2 * sizeof(unsigned int));
    L.total = off;
    return L;
}

template <template <int> class F, typename... Args>
int dispatch_q(int q, Args... args)
{
    switch (q) {
    case 8: return F<8>::run(args...);
    case 9: return F<9>::run(args...);
    case 10: return F<10>::run(args...);
    case 11: return F<11>::run(args...);
    case 12: return F<12>::run(args...);
    case 13: return F<13>::run(args...);
    case 14: return F<14>::run(args...);
    case 15: return F<15>::run(args...);
    case 16: return F<16>::run(args...);
    default:
        mgx_set_last_message("mgx_gemm_ozaki_crt: %d moduli is outside 8..16", q);
        return MGX_E_INVALID;
    }
}

template <int Q>
struct SplitA {
    static int run(const double *A, int m, int k, int lda, const CrtLayout &L, const int *sg, uint8_t *ra,
                   const crt::Consts &K, cudaStream_t stream)
    {
        const int tiles = (m + crt::TILE - 1) / crt::TILE;
        crt::crt_split_a<Q><<<dim3(tiles * 4, L.kblocks), 256, 0, stream>>>(A, m, k, lda, tiles * crt::TILE,
                                                                            L.kblocks, sg, ra, L.ra_mod, K);
        MGX_HOST_CHECK(cudaGetLastError());
        return MGX_SUCCESS;
    }
};

template <int Q>
struct SplitB {
    static int run(const double *B, int n, int k, int ldb, const CrtLayout &L, const int *tu, uint8_t *rb,
                   const crt::Consts &K, cudaStream_t stream)
    {
        const int tiles = (n + crt::TILE - 1) / crt::TILE;
        crt::crt_split_b<Q><<<dim3(tiles * 4, L.kblocks), 256, 0, stream>>>(B, k, n, ldb, L.kblocks, tu, rb, L.rb_mod,
                                                                            K);
        MGX_HOST_CHECK(cudaGetLastError());
        return MGX_SUCCESS;
    }
};

template <int Q>
struct Combine {
    static int run(const crt::CombineParams &cp, long long units, cudaStream_t stream)
    {
        const long long blocks = (units + 7) / 8;
        if (cp.ksplit > 1)
            crt::crt_combine<Q, true><<<(unsigned)blocks, 256, 0, stream>>>(cp, units);
        else
            crt::crt_combine<Q, false><<<(unsigned)blocks, 256, 0, stream>>>(cp, units);
        MGX_HOST_CHECK(cudaGetLastError());
        return MGX_SUCCESS;
    }
};

// Scale exponents and residues of rows [r0, r0 + m) of A (m x k, k <= KMAX; r0 a multiple of
// 256) into the whole-problem workspace.
int crt_split_a_impl(const double *A, int m, int k, int lda, int r0, const crt::Consts &K, unsigned char *ws,
                     const CrtLayout &L, cudaStream_t stream)
{
    if (m <= 0) return MGX_SUCCESS;
    int *status = mgx_device_status_ptr();
    int *sg = reinterpret_cast<int *>(ws + L.sg) + r0;
    uint8_t *ra = ws + L.ra + (size_t)(r0 / crt::TILE) * L.kblocks * crt::SLAB;
    crt::crt_row_scale<<<m, crt::ROW_THREADS, 0, stream>>>(A, m, k, lda, K.alpha, sg, status);
    MGX_HOST_CHECK(cudaGetLastError());
    return dispatch_q<SplitA>(K.q, A, m, k, lda, L, (const int *)sg, ra, K, stream);
}

// The same for columns [c0, c0 + n) of B (k x n).
int crt_split_b_impl(const double *B, int n, int k, int ldb, int c0, const crt::Consts &K, unsigned char *ws,
                     const CrtLayout &L, cudaStream_t stream)
{
    if (n <= 0) return MGX_SUCCESS;
    int *status = mgx_device_status_ptr();
    int *tu = reinterpret_cast<int *>(ws + L.tu) + c0;
    unsigned long long *colmax = reinterpret_cast<unsigned long long *>(ws + L.colmax) + c0;
    unsigned long long *colsum = reinterpret_cast<unsigned long long *>(ws + L.colsum) + c0;
    uint8_t *rb = ws + L.rb + (size_t)(c0 / crt::TILE) * L.kblocks * crt::SLAB;
    MGX_HOST_CHECK(cudaMemsetAsync(colmax, 0, sizeof(unsigned long long) * (size_t)n, stream));
    MGX_HOST_CHECK(cudaMemsetAsync(colsum, 0, sizeof(unsigned long long) * (size_t)n, stream));
    const int sms = mgx_sm_count();
    int ych = (sms * 8) / ((n + 255) / 256);
    if (ych > (k + 63) / 64) ych = (k + 63) / 64;
    if (ych < 1) ych = 1;
    crt::crt_col_max<<<dim3((n + 255) / 256, ych), 256, 0, stream>>>(B, k, n, ldb, colmax);
    MGX_HOST_CHECK(cudaGetLastError());
    crt::crt_col_sumsq<<<dim3((n + 255) / 256, ych), 256, 0, stream>>>(B, k, n, ldb, colmax, colsum);
    MGX_HOST_CHECK(cudaGetLastError());
    crt::crt_col_scale<<<(n + 255) / 256, 256, 0, stream>>>(colmax, colsum, n, K.beta, tu, status);
    MGX_HOST_CHECK(cudaGetLastError());
    return dispatch_q<SplitB>(K.q, B, n, k, ldb, L, (const int *)tu, rb, K, stream);
}

int crt_split_impl(const double *A, const double *B, int m, int n, int k, int lda, int ldb, const crt::Consts &K,
                   unsigned char *ws, const CrtLayout &L, cudaStream_t stream)
{
    int rc = crt_split_a_impl(A, m, k, lda, 0, K, ws, L, stream);
    if (rc == MGX_SUCCESS) rc = crt_split_b_impl(B, n, k, ldb, 0, K, ws, L, stream);
    return rc;
}

// A block of the product inside a whole-problem workspace: rows [r0, r0 + m) and columns
// [c0, c0 + n), r0 and c0 multiples of 256.
struct CrtView {
    const uint8_t *ra, *rb;
    uint8_t *rc;
    const int *sg, *tu;
    int m, n, tiles_m, tiles_n;
};

CrtView crt_view(const CrtLayout &L, unsigned char *ws, int r0, int c0, int m, int n)
{
    CrtView v;
    const int tm0 = r0 / crt::TILE, tn0 = c0 / crt::TILE;
    v.ra = ws + L.ra + (size_t)tm0 * L.kblocks * crt::SLAB;
    v.rb = ws + L.rb + (size_t)tn0 * L.kblocks * crt::SLAB;
    v.rc = ws + L.rc + ((size_t)tm0 * L.tiles_n + tn0) * crt::OUT_TILE_BYTES;
    v.sg = reinterpret_cast<const int *>(ws + L.sg) + r0;
    v.tu = reinterpret_cast<const int *>(ws + L.tu) + c0;
    v.m = m;
    v.n = n;
    v.tiles_m = (m + crt::TILE - 1) / crt::TILE;
    v.tiles_n = (n + crt::TILE - 1) / crt::TILE;
    return v;
}

// Residue products of a block on the tensor cores (one persistent launch).
int crt_products_impl(const crt::Consts &K, const CrtLayout &L, const CrtView &v, cudaStream_t stream,
                      unsigned int *sync = nullptr)
{
    crt::GemmParams p;
    memset(&p, 0, sizeof p);
    p.ra = v.ra;
    p.rb = v.rb;
    p.rc = v.rc;
    p.ra_mod = L.ra_mod;
    p.rb_mod = L.rb_mod;
    p.rc_mod = L.rc_mod;
    p.tiles_m = v.tiles_m;
    p.tiles_n = v.tiles_n;
    p.rc_tile_ld = L.tiles_n;
    p.kblocks = L.kblocks;
    p.q = K.q;
    p.ksplit = L.ksplit;
    p.kb_split = L.kb_split;
    p.rc_slice = (size_t)K.q * L.rc_mod;
    p.status = mgx_device_status_ptr();
    for (int l = 0; l < crt::MAXQ; ++l) {
        p.barrett[l] = K.barrett[l];
        p.bias[l] = (uint32_t)crt::h_moduli[l] * (0x80000000u / (uint32_t)crt::h_moduli[l]);
    }
    const int smem = crt::STAGES * crt::STAGE_BYTES + 1024 + 256;
    const long long items = (long long)K.q * v.tiles_m * v.tiles_n * L.ksplit;
    if (items <= 0) return MGX_SUCCESS;
    if (items > 0x7fffffffll) {
        mgx_set_last_message("mgx_gemm_ozaki_crt: product too large (%lld work items)", items);
        return MGX_E_UNSUPPORTED;
    }
    const int sms = mgx_sm_count();
    const int grid = (long long)sms < items ? sms : (int)items;
    if (sync) {
        MGX_HOST_CHECK(cudaMemsetAsync(sync, 0, sizeof(unsigned int), stream));
        p.sync = sync;
    }
    MGX_HOST_CHECK(cudaFuncSetAttribute(crt::crt_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    crt::crt_gemm<<<grid, crt::THREADS, smem, stream>>>(p);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

// CRT recombination of a block into C (the block's first element; leading dimension ldc).
int crt_combine_impl(double *C, int ldc, int beta_one, const crt::Consts &K, const CrtLayout &L, const CrtView &v,
                     cudaStream_t stream)
{
    crt::CombineParams cp;
    memset(&cp, 0, sizeof cp);
    cp.rc = v.rc;
    cp.rc_mod = L.rc_mod;
    cp.ksplit = L.ksplit;
    cp.rc_slice = (size_t)K.q * L.rc_mod;
    cp.C = C;
    cp.m = v.m;
    cp.n = v.n;
    cp.ldc = ldc;
    cp.tiles_n = v.tiles_n;
    cp.rc_tile_ld = L.tiles_n;
    cp.beta_one = beta_one;
    cp.vec_store = ((ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    cp.sg = v.sg;
    cp.tu = v.tu;
    cp.K = K;
    const long long units = (long long)v.tiles_m * v.tiles_n * 256;
    if (units <= 0) return MGX_SUCCESS;
    return dispatch_q<Combine>(K.q, cp, units, stream);
}

int crt_multiply_impl(double *C, int m, int n, int ldc, int beta_one, const crt::Consts &K, unsigned char *ws,
                      const CrtLayout &L, cudaStream_t stream)
{
    const CrtView v = crt_view(L, ws, 0, 0, m, n);
    int rc = crt_products_impl(K, L, v, stream, reinterpret_cast<unsigned int *>(ws + L.sync));
    if (rc == MGX_SUCCESS) rc = crt_combine_impl(C, ldc, beta_one, K, L, v, stream);
    return rc;
}

}  // namespace

extern "C" MGX_API size_t mgx_crt_workspace_size(int m, int n, int k, int moduli)
{
    if (m < 0 || n < 0 || k < 0 || moduli < crt::MINQ || moduli > crt::MAXQ) return 0;
    return crt_layout(m, n, k, moduli).total;
}

extern "C" MGX_API int mgx_crt_kmax(void) { return crt::KMAX; }

int mgx_crt_run(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb, int ldc,
                int beta_one, int moduli, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    crt::Consts K;
    if (m < 0 || n < 0 || k < 0 || !crt::make_consts(moduli, K) || (m > 0 && n > 0 && (!C || ldc < n)) ||
        (m > 0 && n > 0 && k > 0 && (!A || !B || lda < k || ldb < n))) {
        mgx_set_last_message("mgx_gemm_ozaki_crt: invalid arguments m=%d n=%d k=%d moduli=%d (8..16)", m, n, k, moduli);
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0) return MGX_SUCCESS;
    if (k == 0) {
        if (beta_one) return MGX_SUCCESS;
        MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)n * sizeof(double), m, stream));
        return MGX_SUCCESS;
    }
    const CrtLayout L = crt_layout(m, n, k, moduli);
    if (!workspace || workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        mgx_set_last_message("mgx_gemm_ozaki_crt: workspace needs %zu bytes, 256-byte aligned (got %zu)", L.total,
                             workspace_bytes);
        return MGX_E_WORKSPACE;
    }
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    for (int k0 = 0; k0 < k; k0 += crt::KMAX) {
        const int kc = (k - k0 < crt::KMAX) ? k - k0 : crt::KMAX;
        int rc = crt_split_impl(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, K, ws, L, stream);
        if (rc != MGX_SUCCESS) return rc;
        rc = crt_multiply_impl(C, m, n, ldc, (k0 > 0) ? 1 : beta_one, K, ws, L, stream);
        if (rc != MGX_SUCCESS) return rc;
    }
    return MGX_SUCCESS;
}

static int crt_phase_check(int m, int n, int k, int moduli, const void *workspace, size_t workspace_bytes,
                           const char *who, crt::Consts &K, CrtLayout &L)
{
    if (m < 0 || n < 0 || k < 0 || k > crt::KMAX || !crt::make_consts(moduli, K)) {
        mgx_set_last_message("%s: invalid arguments m=%d n=%d k=%d (<= %d) moduli=%d (8..16)", who, m, n, k, crt::KMAX,
                             moduli);
        return MGX_E_INVALID;
    }
    L = crt_layout(m, n, k, moduli);
    if (!workspace || workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        mgx_set_last_message("%s: workspace needs %zu bytes, 256-byte aligned (got %zu)", who, L.total, workspace_bytes);
        return MGX_E_WORKSPACE;
    }
    return MGX_SUCCESS;
}

extern "C" MGX_API int mgx_crt_split(const double *A, const double *B, int m, int n, int k, int lda, int ldb,
                                     int moduli, void *workspace, size_t workspace_bytes, void *stream)
{
    crt::Consts K;
    CrtLayout L;
    int rc = crt_phase_check(m, n, k, moduli, workspace, workspace_bytes, "mgx_crt_split", K, L);
    if (rc != MGX_SUCCESS) return rc;
    if ((m > 0 && k > 0 && (!A || lda < k)) || (n > 0 && k > 0 && (!B || ldb < n))) {
        mgx_set_last_message("mgx_crt_split: invalid operand pointers or leading dimensions");
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0 || k == 0) return MGX_SUCCESS;
    return crt_split_impl(A, B, m, n, k, lda, ldb, K, static_cast<unsigned char *>(workspace), L, (cudaStream_t)stream);
}

extern "C" MGX_API int mgx_crt_products(int m, int n, int k, int moduli, void *workspace, size_t workspace_bytes,
                                        void *stream)
{
    crt::Consts K;
    CrtLayout L;
    int rc = crt_phase_check(m, n, k, moduli, workspace, workspace_bytes, "mgx_crt_products", K, L);
    if (rc != MGX_SUCCESS) return rc;
    if (m == 0 || n == 0 || k == 0) return MGX_SUCCESS;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    return crt_products_impl(K, L, crt_view(L, ws, 0, 0, m, n), (cudaStream_t)stream,
                             reinterpret_cast<unsigned int *>(ws + L.sync));
}

extern "C" MGX_API int mgx_crt_combine(double *C, int m, int n, int k, int ldc, int beta_one, int moduli,
                                       void *workspace, size_t workspace_bytes, void *stream)
{
    crt::Consts K;
    CrtLayout L;
    int rc = crt_phase_check(m, n, k, moduli, workspace, workspace_bytes, "mgx_crt_combine", K, L);
    if (rc != MGX_SUCCESS) return rc;
    if (m > 0 && n > 0 && (!C || ldc < n)) {
        mgx_set_last_message("mgx_crt_combine: invalid C or ldc");
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0) return MGX_SUCCESS;
    if (k == 0) {
        if (beta_one) return MGX_SUCCESS;
        MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)n * sizeof(double), m,
                                         (cudaStream_t)stream));
        return MGX_SUCCESS;
    }
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    return crt_combine_impl(C, ldc, beta_one ? 1 : 0, K, L, crt_view(L, ws, 0, 0, m, n), (cudaStream_t)stream);
}

// Hooks for the host-buffer schedule (mgx_gemm_host in ozaki.cu): a workspace for the whole
// M x N x K product (K <= KMAX), panels prepared as they arrive and blocks computed from them.
size_t mgx_crt_host_ws_bytes(int M, int N, int K, int q) { return crt_layout(M, N, K, q).total; }

int mgx_crt_host_rows(const double *A, int m, int lda, int r0, int M, int N, int K, int q, unsigned char *ws,
                      cudaStream_t stream)
{
    crt::Consts C;
    if (!crt::make_consts(q, C)) return MGX_E_INVALID;
    return crt_split_a_impl(A, m, K, lda, r0, C, ws, crt_layout(M, N, K, q), stream);
}

int mgx_crt_host_cols(const double *B, int n, int ldb, int c0, int M, int N, int K, int q, unsigned char *ws,
                      cudaStream_t stream)
{
    crt::Consts C;
    if (!crt::make_consts(q, C)) return MGX_E_INVALID;
    return crt_split_b_impl(B, n, K, ldb, c0, C, ws, crt_layout(M, N, K, q), stream);
}

int mgx_crt_host_block(double *Cb, int ldc, int r0, int c0, int m, int n, int M, int N, int K, int q,
                       unsigned char *ws, cudaStream_t stream, int slot)
{
    crt::Consts C;
    if (!crt::make_consts(q, C)) return MGX_E_INVALID;
    const CrtLayout L = crt_layout(M, N, K, q);
    const CrtView v = crt_view(L, ws, r0, c0, m, n);
    int rc = crt_products_impl(C, L, v, stream, reinterpret_cast<unsigned int *>(ws + L.sync) + (slot & 1));
    if (rc == MGX_SUCCESS) rc = crt_combine_impl(Cb, ldc, 0, C, L, v, stream);
    return rc;
}

extern "C" MGX_API size_t mgx_crt_splitk_workspace_size(int m, int n, int k, int moduli, int ksplit)
{
    if (m < 0 || n < 0 || k < 0 || moduli < crt::MINQ || moduli > crt::MAXQ || ksplit < 1 || k > crt::KMAX) return 0;
    return crt_layout(m, n, k, moduli, ksplit).total;
}

extern "C" MGX_API int mgx_gemm_ozaki_crt_splitk(const double *A, const double *B, double *C, int m, int n, int k,
                                                 int lda, int ldb, int ldc, int beta_one, int moduli, int ksplit,
                                                 void *workspace, size_t workspace_bytes, void *stream)
{
    crt::Consts K;
    if (m < 0 || n < 0 || k < 0 || ksplit < 1 || !crt::make_consts(moduli, K) || (m > 0 && n > 0 && (!C || ldc < n)) ||
        (m > 0 && n > 0 && k > 0 && (!A || !B || lda < k || ldb < n))) {
        mgx_set_last_message("mgx_gemm_ozaki_crt_splitk: invalid arguments m=%d n=%d k=%d moduli=%d ksplit=%d", m, n, k,
                             moduli, ksplit);
        return MGX_E_INVALID;
    }
    if (k > crt::KMAX) {
        mgx_set_last_message("mgx_gemm_ozaki_crt_splitk: k = %d is above one int32 residue accumulation (%d)", k,
                             crt::KMAX);
        return MGX_E_UNSUPPORTED;
    }
    if (ksplit == 1 || m == 0 || n == 0 || k == 0)
        return mgx_crt_run(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, moduli, workspace, workspace_bytes,
                           (cudaStream_t)stream);
    const CrtLayout L = crt_layout(m, n, k, moduli, ksplit);
    if (!workspace || workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        mgx_set_last_message("mgx_gemm_ozaki_crt_splitk: workspace needs %zu bytes, 256-byte aligned (got %zu)", L.total,
                             workspace_bytes);
        return MGX_E_WORKSPACE;
    }
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = crt_split_impl(A, B, m, n, k, lda, ldb, K, ws, L, st);
    if (rc == MGX_SUCCESS) rc = crt_multiply_impl(C, m, n, ldc, beta_one ? 1 : 0, K, ws, L, st);
    return rc;
}

extern "C" MGX_API int mgx_gemm_ozaki_crt(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                          int ldb, int ldc, int beta_one, int moduli, void *workspace,
                                          size_t workspace_bytes, void *stream)
{
    return mgx_crt_run(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, moduli, workspace, workspace_bytes,
                       (cudaStream_t)stream);
}

// A-priori modulus count.  With alpha + beta = L - 3 bits shared by the two operands, the
// rounding of A' and B' to integers leaves a normwise error close to sqrt(k / 6) 2^(-(L-3)/2)
// (each entry is rounded to within 1/2, the scale puts row and column norms at 2^alpha, 2^beta);
// measured on the oracle it stays within 2x of that, floored near 5e-17 by the FP64 result.
// Returns the smallest q in 8..16 whose prediction, times 2 and a 1.25 safety factor, meets
// `target`, else 16.
extern "C" MGX_API int mgx_crt_choose_moduli(int k, double target)
{
    if (!(target > 0.0)) target = 1e-15;
    const double kk = k > 1 ? (double)k : 1.0;
    double lp = 0.0;
    for (int q = 1; q <= crt::MAXQ; ++q) {
        lp += log2((double)crt::h_moduli[q - 1]);
        if (q < crt::MINQ) continue;
        const int L = (int)floor(lp) + 1;
        double e = 2.0 * sqrt(kk / 6.0) * exp2(-0.5 * (L - 3));
        if (e < 5e-17) e = 5e-17;
        if (e * 1.25 <= target) return q;
    }
    return crt::MAXQ;
}
