// ozaki.cu -- FP64-accurate GEMM on the INT8 tensor cores (Ozaki scheme; Ozaki, Ogita, Oishi &
// Rump 2012, "Error-free transformations of matrix multiplication by using fast routines of
// matrix multiplication and its applications"; Ootomo, Ozaki & Yokota 2024, "DGEMM on integer
// matrix multiplication unit").
//
// Algorithm (s = number of slices):
//   ea_i = e such that max_k |a_ik| in [2^(e-1), 2^e); eb_j likewise for column j of B.
//   x = a_ik * 2^(6 - ea_i) (|x| < 64); digit_t = rint(x), x <- (x - digit_t) * 128, t = 1..s.
//   Every digit is an integer in [-64, 64]; a_ik = 2^(ea_i - 6) sum_t digit_t 2^(-7(t-1)) + tail.
//   G_d = sum_{t+u=d} sum_k DA_t[i,k] DB_u[j,k] for d = 2..s+1 is exact in int32 while
//   s * 64 * 64 * K < 2^31 (the host splits K beyond that).
//   h = 0; for d = s+1 down to 2: h = fma(h, 2^-7, G_d);   C_ij (+)= h * 2^(ea_i + eb_j - 12).
//
// Kernels:
//   ozaki_row_exp   row maxima of A (one warp per row)
//   ozaki_col_max   column maxima of B (atomicMax on the bit pattern of |b|)
//   ozaki_split_a   digits of A as swizzled K-major tiles, blocked [row tile][K block][slice]
//   ozaki_split_b   digits of B^T in the same layout, transposed through shared memory
//   ozaki_gemm      persistent tcgen05 kernel, one 128 x 128 output tile at a time:
//       warp 0      producer: one bulk copy per operand and K block moves every slice a weight
//                   set needs (already in the MMA's 32-byte-swizzled tile image), for
//                   floor(s / slices) consecutive 32-byte K blocks per stage, so every stage
//                   carries about 2s tiles, into a 3-stage ring
//       warp 1      TMEM owner and MMA issuer: tcgen05.mma.kind::i8, M=128 N=128 K=32, one
//                   int32 accumulator (128 TMEM columns) per weight group, four groups per set
//       warps 2-9   epilogue: tcgen05.ld of each group, FP64 Horner update held in registers
//                   across sets (highest weights first), final power-of-two scaling and store
// All waits are bounded (mgx_common.cuh); TMEM is always released before the CTA exits.
#include <cstdio>
#include <cstring>
#include <mutex>

#include <vector>

#include "mgx_common.cuh"

namespace mgx {
namespace oz {

constexpr int TILE = 128;              // output tile is TILE x TILE
constexpr int KBLK = 32;               // bytes of K per stage (one MMA instruction)
constexpr int SLICE_TILE_BYTES = TILE * KBLK;  // 4 KiB
constexpr int MAX_SPLITS = 12;
constexpr int MAX_SETS = 3;            // ceil(12 / 4): up to four weight groups (4 x 128 TMEM columns) per set
constexpr int EPI_WARPS = 8;
constexpr int THREADS = (2 + EPI_WARPS) * 32;
constexpr int NONFINITE_EXP = 0x7fffffff;

struct GemmParams {
    double *C;
    int m, n, ldc;
    int kblocks;              // ceil(kp / 32)
    int splits;
    int num_sets;
    int set_dhi[MAX_SETS];    // highest weight of each set (sets ordered by decreasing weight)
    int set_dlo[MAX_SETS];
    int stage_bytes;          // 2 * splits * 4 KiB
    int stages;
    const int *ea;            // row exponents of A
    const int *eb;            // column exponents of B
    const uint8_t *da;        // digit tiles of A: [m/128][kblocks][splits][128 x 32 B], swizzled
    const uint8_t *db;        // digit tiles of B^T, same layout over n
    int beta_one;
    int vec_store;
    int *status;
    int ksplit;               // > 1: work item w is (tile w / ksplit, K slice w % ksplit)
    int kb_split;             // K blocks per slice
    double *partial;          // split-K: slice s's scaled result goes to partial + s * partial_stride
    int partial_ld;           // even
    size_t partial_stride;
    unsigned int *sync;       // this launch's arrival counter (zeroed before the launch), or nullptr
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
    if (e >= -1022 && e <= 1023) return x * pow2i(e);
    const int e1 = e / 2, e2 = e - e1;
    return (x * pow2i(e1)) * pow2i(e2);
}

// ---------------------------------------------------------------- split kernels
__global__ void ozaki_row_exp(const double *__restrict__ A, int m, int k, int lda, int *__restrict__ ea,
                              int *status)
{
    const int warps = blockDim.x >> 5;
    const int row = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= m) return;
    const unsigned long long *r = reinterpret_cast<const unsigned long long *>(A + (size_t)row * lda);
    unsigned long long mx = 0;
    for (int kk = lane; kk < k; kk += 32) {
        const unsigned long long b = __ldg(r + kk) & 0x7fffffffffffffffull;
        mx = b > mx ? b : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = other > mx ? other : mx;
    }
    if (lane == 0) {
        if (mx >= 0x7ff0000000000000ull) {
            ea[row] = NONFINITE_EXP;
            record_status(status, kDevNonFinite);
        } else {
            ea[row] = frexp_exp_bits(mx);
        }
    }
}

// grid (ceil(n/256), ychunks); each thread scans a run of rows of one column.
__global__ void ozaki_col_max(const double *__restrict__ B, int k, int n, int ldb, unsigned long long *colmax)
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

__global__ void ozaki_col_exp(const unsigned long long *__restrict__ colmax, int n, int *__restrict__ eb,
                              int *status)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long mx = colmax[j];
    if (mx >= 0x7ff0000000000000ull) {
        eb[j] = NONFINITE_EXP;
        record_status(status, kDevNonFinite);
    } else {
        eb[j] = frexp_exp_bits(mx);
    }
}

// Digits of one value (the oracle's digits_of: d = rint(x), x <- (x - d) * 128).  rint is
// computed by adding 1.5 * 2^52: for |x| < 2^51 the sum is rounded to an integer by the add
// itself, to nearest with ties to even (as rint), and the integer sits in the low bits of the
// sum.  Subtracting the constant back gives rint(x) exactly.  Two full-rate adds replace a
// round and a float-to-int conversion per digit.
template <int S>
__device__ __forceinline__ void digits(double v, int e, int8_t (&d)[S], int s)
{
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
    double x = scale2(v, 6 - e);
#pragma unroll
    for (int t = 0; t < S; ++t) {
        if (t < s) {
            const double y = __dadd_rn(x, kRound);
            const double r = __dsub_rn(y, kRound);
            d[t] = (int8_t)__double2loint(y);
            x = (x - r) * 128.0;
        } else {
            d[t] = 0;
        }
    }
}

// Digit tiles are stored exactly as the MMA reads them from shared memory: for every 128-row
// tile and 32-byte K block, the s slices follow each other, each a 128 x 32-byte K-major tile
// with the 32-byte swizzle (the 16-byte half of row r is flipped when bit 2 of r is set).  One
// bulk copy then moves every slice a stage needs.  Byte (row r, k byte c) of slice t of tile
// (tm, kb) sits at ((tm * kblocks + kb) * s + t) * 4096 + r * 32 + (c ^ (((r >> 2) & 1) << 4)).
__device__ __forceinline__ size_t slab_offset(int tile, int kb, int kblocks, int s, int r, int c)
{
    return ((size_t)tile * kblocks + kb) * (size_t)s * SLICE_TILE_BYTES + (size_t)r * 32 + (c ^ (((r >> 2) & 1) << 4));
}

// One warp per (8-row group, K block): lane -> row (lane / 4), 8 consecutive k (lane % 4).
// Rows up to the 128-row padding and k up to the 32 padding get zero digits.
template <int S>
__global__ void __launch_bounds__(256) ozaki_split_a(const double *__restrict__ A, int m, int k, int lda, int mp,
                                                     int kblocks, const int *__restrict__ ea, uint8_t *__restrict__ da)
{
    const int lane = threadIdx.x & 31;
    const long long wpb = blockDim.x >> 5;
    const long long items = (long long)(mp / 8) * kblocks;
    for (long long it = blockIdx.x * wpb + (threadIdx.x >> 5); it < items; it += (long long)gridDim.x * wpb) {
        const int ro = (int)(it / kblocks), kb = (int)(it % kblocks);
        const int row = ro * 8 + (lane >> 2), kq = lane & 3;
        const int k0 = kb * 32 + kq * 8;
        int e = (row < m) ? ea[row] : 0;
        if (e == NONFINITE_EXP) e = 0;
        unsigned long long packed[S];
#pragma unroll
        for (int t = 0; t < S; ++t) packed[t] = 0;
        const double *arow = A + (size_t)(row < m ? row : 0) * lda;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int kk = k0 + j;
            double v = (row < m && kk < k) ? __ldg(arow + kk) : 0.0;
            if (!isfinite(v)) v = 0.0;
            int8_t dg[S];
            digits<S>(v, e, dg, S);
#pragma unroll
            for (int t = 0; t < S; ++t) packed[t] |= (unsigned long long)(uint8_t)dg[t] << (8 * j);
        }
        const size_t off = slab_offset(row >> 7, kb, kblocks, S, row & 127, kq * 8);
#pragma unroll
        for (int t = 0; t < S; ++t)
            *reinterpret_cast<unsigned long long *>(da + off + (size_t)t * SLICE_TILE_BYTES) = packed[t];
    }
}

// Block: 32 k x 128 columns of B through shared memory (coalesced reads along the columns),
// written as the digit tiles of B^T (column j of B is row j of the tile).
template <int S>
__global__ void __launch_bounds__(256) ozaki_split_b(const double *__restrict__ B, int k, int n, int ldb, int kblocks,
                                                     const int *__restrict__ eb, uint8_t *__restrict__ db)
{
    __shared__ double tb[32][129];
    const int tn = blockIdx.x, kb = blockIdx.y;
    const int n0 = tn * 128, k0 = kb * 32;
    for (int idx = threadIdx.x; idx < 32 * 128; idx += 256) {
        const int kk = idx >> 7, c = idx & 127;
        double v = (k0 + kk < k && n0 + c < n) ? __ldg(B + (size_t)(k0 + kk) * ldb + n0 + c) : 0.0;
        if (!isfinite(v)) v = 0.0;
        tb[kk][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int item = threadIdx.x + 256 * half;
        const int r = item >> 2, kq = item & 3;   // tile row r = column n0 + r of B
        int e = (n0 + r < n) ? eb[n0 + r] : 0;
        if (e == NONFINITE_EXP) e = 0;
        unsigned long long packed[S];
#pragma unroll
        for (int t = 0; t < S; ++t) packed[t] = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            int8_t dg[S];
            digits<S>(tb[kq * 8 + j][r], e, dg, S);
#pragma unroll
            for (int t = 0; t < S; ++t) packed[t] |= (unsigned long long)(uint8_t)dg[t] << (8 * j);
        }
        const size_t off = slab_offset(tn, kb, kblocks, S, r, kq * 8);
#pragma unroll
        for (int t = 0; t < S; ++t)
            *reinterpret_cast<unsigned long long *>(db + off + (size_t)t * SLICE_TILE_BYTES) = packed[t];
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

// K-major operand tile of 128 rows x 32 bytes written by TMA with the 32-byte swizzle:
// rows 32 B apart, groups of 8 rows 256 B apart (SBO), LBO unused (1), layout type 6.
__device__ __forceinline__ uint64_t sw32_desc(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(256 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                 // descriptor version (sm100)
    d |= (uint64_t)6 << 61;                 // SWIZZLE_32B
    return d;
}

// kind::i8 instruction descriptor: D s32, A s8, B s8, both K-major, M = 128, N = 128.
constexpr uint32_t IDESC_S8_128x128 =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TILE >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tile_of(const GemmParams &p, int w, int &m0, int &n0)
{
    // groups of 8 tile rows sweep the columns together so their A slices stay in L2
    const int tiles_n = (p.n + TILE - 1) / TILE;
    const int tiles_m = (p.m + TILE - 1) / TILE;
    const int per_group = 8 * tiles_n;
    const int g = w / per_group, r = w % per_group;
    const int first = g * 8;
    const int gsize = min(tiles_m - first, 8);
    m0 = (first + r % gsize) * TILE;
    n0 = (r / gsize) * TILE;
}

// Work item w: its output tile (8-tile-row raster over the tiles) and its K blocks
// [kb_begin, kb_end) -- all of K, or one slice of it in the split-K form.
__device__ __forceinline__ void item_of(const GemmParams &p, int w, int &m0, int &n0, int &kb_begin, int &kb_end)
{
    const int ks = p.ksplit > 1 ? p.ksplit : 1;
    tile_of(p, w / ks, m0, n0);
    kb_begin = (w % ks) * p.kb_split;
    kb_end = min(p.kblocks, kb_begin + p.kb_split);
}

// Weight sets of up to four consecutive groups, highest weights first (the same rule as the
// host's, at compile time so the MMA issue sequence can be unrolled completely).
__host__ __device__ constexpr int set_lo_of(int dhi) { return (dhi - 3 > 2) ? dhi - 3 : 2; }
__host__ __device__ constexpr int set_hi(int S, int si)
{
    int d = S + 1;
    for (int i = 0; i < si; ++i) d = set_lo_of(d) - 1;
    return d;
}
__host__ __device__ constexpr int num_sets_of(int S)
{
    int d = S + 1, n = 0;
    while (d >= 2) {
        d = set_lo_of(d) - 1;
        ++n;
    }
    return n;
}
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Issues every MMA of one stage of weight set SI (NKB <= KPACK K blocks, slices 1..NSL of each
// operand per K block, tiles laid out [K block][slice]).  All loop bounds are compile-time, so
// each MMA costs a descriptor add and the instruction itself.  The first product into each
// group's accumulator in the first K block overwrites it (accumulate flag 0).
template <int S, int SI>
__device__ __forceinline__ void issue_stage(uint32_t tmem_base, uint64_t a0, uint64_t b0, int nkb, bool first_kb)
{
    constexpr int DHI = set_hi(S, SI), DLO = set_lo_of(DHI), NSL = cmin(S, DHI - 1), KPACK = S / NSL;
#pragma unroll
    for (int j = 0; j < KPACK; ++j) {
        if (j < nkb) {
            const uint32_t fresh = (first_kb && j == 0) ? 1u : 0u;
#pragma unroll
            for (int t = 1; t <= NSL; ++t) {
#pragma unroll
                for (int u = 1; u <= NSL; ++u) {
                    if (t + u >= DLO && t + u <= DHI) {
                        const int slot = DHI - (t + u);
                        const bool first_of_slot = (t == cmax(1, (t + u) - NSL));
                        const uint32_t acc = (first_of_slot && fresh) ? 0u : 1u;
                        tc_mma_i8(tmem_base + slot * TILE,
                                  a0 + (uint64_t)((j * NSL + t - 1) * (SLICE_TILE_BYTES >> 4)),
                                  b0 + (uint64_t)((j * NSL + u - 1) * (SLICE_TILE_BYTES >> 4)), IDESC_S8_128x128, acc);
                    }
                }
            }
        }
    }
}

// Runs weight set SI of one tile on the MMA thread: waits for the epilogue to free the
// accumulators, then walks the K blocks stage by stage.  Returns false if a wait ran out.
template <int S, int SI>
__device__ __forceinline__ bool mma_set(const GemmParams &p, uint32_t smem_base, uint32_t tmem_base, uint64_t *full,
                                        uint64_t *empty, uint64_t *acc_full, uint64_t *acc_empty, int &stage,
                                        uint32_t &phase, uint32_t &acc_phase, int kb_begin, int kb_end)
{
    constexpr int DHI = set_hi(S, SI), NSL = cmin(S, DHI - 1), KPACK = S / NSL;
    if (!mbar_wait_bounded(acc_empty, acc_phase ^ 1u, p.status, kDevTimeoutAcc)) return false;
    acc_phase ^= 1u;
    tc_fence_after();
    for (int kb0 = kb_begin; kb0 < kb_end; kb0 += KPACK) {
        if (!mbar_wait_bounded(&full[stage], phase, p.status, kDevTimeoutFull)) return false;
        tc_fence_after();
        const uint32_t sa = smem_base + stage * p.stage_bytes;
        issue_stage<S, SI>(tmem_base, sw32_desc(sa), sw32_desc(sa + S * SLICE_TILE_BYTES), min(KPACK, kb_end - kb0),
                           kb0 == kb_begin);
        tc_commit(&empty[stage]);  // frees the stage once these MMAs have read it
        if (++stage == p.stages) {
            stage = 0;
            phase ^= 1u;
        }
    }
    tc_commit(acc_full);
    return true;
}

template <int S>
__global__ void __launch_bounds__(THREADS, 1) ozaki_gemm(const __grid_constant__ GemmParams p)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                            ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + p.stages * p.stage_bytes);
    uint64_t *empty = full + 4;
    uint64_t *acc_full = empty + 4;
    uint64_t *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = ((p.m + TILE - 1) / TILE) * ((p.n + TILE - 1) / TILE);
    const int items = total * (p.ksplit > 1 ? p.ksplit : 1);

    if (threadIdx.x == 0) {
        for (int s = 0; s < p.stages; ++s) {
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
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int armed[4] = {-1, -1, -1, -1};
            bool ok = true;
            const size_t slab = (size_t)p.splits * SLICE_TILE_BYTES;  // all slices of one 128-row tile, one K block
            for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
                int m0, n0, kb_begin, kb_end;
                item_of(p, w, m0, n0, kb_begin, kb_end);
                // Soft lockstep: the CTAs that share a digit slab read it from L2 only while they
                // stay within a few microseconds of each other, so every producer waits at each
                // new item until all CTAs have started theirs -- or 20 us, then goes on anyway.
                // Nothing depends on it for correctness, so it cannot deadlock.
                if (p.sync) {
                    atomicAdd(p.sync, 1u);
                    const unsigned int target = (unsigned int)min((long long)(w / gridDim.x + 1) * gridDim.x,
                                                                  (long long)items);
                    const unsigned long long t0 = global_ns();
                    while (*reinterpret_cast<volatile unsigned int *>(p.sync) < target &&
                           global_ns() - t0 < 20000ull)
                        __nanosleep(64);
                }
                const uint8_t *ga = p.da + (size_t)(m0 / TILE) * p.kblocks * slab;
                const uint8_t *gb = p.db + (size_t)(n0 / TILE) * p.kblocks * slab;
                for (int si = 0; si < p.num_sets && ok; ++si) {
                    const int nsl = min(p.splits, p.set_dhi[si] - 1);
                    const int kpack = p.splits / nsl;   // K blocks per stage: every stage ~2s tiles
                    const uint32_t bytes = (uint32_t)(nsl * SLICE_TILE_BYTES);
                    for (int kb0 = kb_begin; kb0 < kb_end; kb0 += kpack) {
                        if (!mbar_wait_bounded(&empty[stage], phase ^ 1u, p.status, kDevTimeoutEmpty)) {
                            ok = false;
                            break;
                        }
                        const int nkb = min(kpack, kb_end - kb0);
                        unsigned char *sa = smem + stage * p.stage_bytes;
                        unsigned char *sb = sa + p.splits * SLICE_TILE_BYTES;
                        mbar_arrive_expect_tx(&full[stage], 2u * (uint32_t)nkb * bytes);
                        armed[stage] = (int)phase;
                        for (int j = 0; j < nkb; ++j) {
                            // slices 1..nsl of K block kb0+j are contiguous: one bulk copy per operand
                            bulk_load(sa + j * bytes, ga + (size_t)(kb0 + j) * slab, bytes, &full[stage]);
                            bulk_load(sb + j * bytes, gb + (size_t)(kb0 + j) * slab, bytes, &full[stage]);
                        }
                        if (++stage == p.stages) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                }
            }
            for (int s = 0; s < p.stages; ++s)
                if (armed[s] >= 0) mbar_wait_bounded(&full[s], (uint32_t)armed[s], p.status, kDevTimeoutFull);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true;
            const uint32_t smem_base = smem_u32(smem);
            constexpr int NS = num_sets_of(S);
            for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
                int m0, n0, kb_begin, kb_end;
                item_of(p, w, m0, n0, kb_begin, kb_end);
                ok = mma_set<S, 0>(p, smem_base, tmem_base, full, empty, acc_full, acc_empty, stage, phase, acc_phase,
                                   kb_begin, kb_end);
                if (NS > 1 && ok)
                    ok = mma_set<S, (NS > 1 ? 1 : 0)>(p, smem_base, tmem_base, full, empty, acc_full, acc_empty, stage,
                                                      phase, acc_phase, kb_begin, kb_end);
                if (NS > 2 && ok)
                    ok = mma_set<S, (NS > 2 ? 2 : 0)>(p, smem_base, tmem_base, full, empty, acc_full, acc_empty, stage,
                                                      phase, acc_phase, kb_begin, kb_end);
            }
            // Drain: all MMAs this thread issued have finished before TMEM is released.
            tc_commit(drain);
            mbar_wait_bounded(drain, 0, p.status, kDevTimeoutAcc);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..9)
        const int q = warp & 3;             // TMEM lane quarter this warp may access
        const int half = (warp - 2) >> 2;   // which 64 of the 128 columns
        uint32_t acc_phase = 0;
        bool ok = true;
        for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
            int m0, n0, kb_begin, kb_end;
            item_of(p, w, m0, n0, kb_begin, kb_end);
            const int m_end = p.m, n_end = p.n;
            // destination: C, or this K slice's partial results (plain stores, summed later)
            const bool split = p.ksplit > 1;
            double *const dbase = split ? p.partial + (size_t)(w % p.ksplit) * p.partial_stride : p.C;
            const int dld = split ? p.partial_ld : p.ldc;
            const int dvec = split ? 1 : p.vec_store;
            const int dbeta = split ? 0 : p.beta_one;
            double h[64];
#pragma unroll
            for (int j = 0; j < 64; ++j) h[j] = 0.0;
            for (int si = 0; si < p.num_sets; ++si) {
                bool got = true;
                if (lane == 0) got = mbar_wait_sleepy(acc_full, acc_phase, p.status, kDevTimeoutAcc);
                got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
                if (!got) {
                    ok = false;
                    break;
                }
                acc_phase ^= 1u;
                tc_fence_after();
                const int ngroups = p.set_dhi[si] - p.set_dlo[si] + 1;
                for (int slot = 0; slot < ngroups; ++slot) {
                    const uint32_t tbase = tmem_base + ((uint32_t)(32 * q) << 16) + slot * TILE + half * 64;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        uint32_t r[16];
                        tmem_ld16(tbase + c * 16, r);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            h[c * 16 + j] = fma(h[c * 16 + j], 0.0078125, (double)(int)r[j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty);
            }
            if (!ok) break;
            const int row = m0 + 32 * q + lane;
            if (row < m_end) {
                const int er = p.ea[row];
                double *crow = dbase + (size_t)row * dld;
                const int cbase = n0 + half * 64;
#pragma unroll
                for (int j = 0; j < 64; j += 2) {
                    const int col = cbase + j;
                    if (col >= n_end) break;
                    const int e0 = p.eb[col];
                    double v0 = (er == NONFINITE_EXP || e0 == NONFINITE_EXP) ? __longlong_as_double(0x7ff8000000000000ll)
                                                                              : scale2(h[j], er + e0 - 12);
                    if (col + 1 < n_end) {
                        const int e1 = p.eb[col + 1];
                        double v1 = (er == NONFINITE_EXP || e1 == NONFINITE_EXP)
                                        ? __longlong_as_double(0x7ff8000000000000ll)
                                        : scale2(h[j + 1], er + e1 - 12);
                        if (dvec) {
                            double2 *dst = reinterpret_cast<double2 *>(crow + col);
                            if (dbeta) {
                                const double2 o = *dst;
                                v0 = o.x + v0;
                                v1 = o.y + v1;
                            }
                            *dst = make_double2(v0, v1);
                        } else {
                            crow[col] = dbeta ? crow[col] + v0 : v0;
                            crow[col + 1] = dbeta ? crow[col + 1] + v1 : v1;
                        }
                    } else {
                        crow[col] = dbeta ? crow[col] + v0 : v0;
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    __syncwarp();
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(512) : "memory");
}

}  // namespace oz
}  // namespace mgx

using namespace mgx;

namespace {

struct WsLayout {
    size_t da, db, ea, eb, colmax, total;
    int kblocks;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int ozaki_kmax(int s) { return (int)((2147483647ll / (4096ll * s)) & ~127ll); }

// Workspace for one K range of at most ozaki_kmax(s): digit tiles of A (m rounded up to 128) and
// of B^T (n rounded up to 128), each K block 32 bytes wide, then the exponents.
WsLayout ws_layout(int m, int n, int k, int s)
{
    WsLayout L;
    int kc = k;
    const int kmax = ozaki_kmax(s);
    if (kc > kmax) kc = kmax;
    L.kblocks = (kc + 31) / 32;
    if (L.kblocks == 0) L.kblocks = 1;
    const size_t mp = (size_t)((m + 127) / 128) * 128, np = (size_t)((n + 127) / 128) * 128;
    size_t off = 0;
    L.da = off;
    off = align256(off + (size_t)s * mp * L.kblocks * 32);
    L.db = off;
    off = align256(off + (size_t)s * np * L.kblocks * 32);
    L.ea = off;
    off = align256(off + sizeof(int) * (size_t)m);
    L.eb = off;
    off = align256(off + sizeof(int) * (size_t)n);
    L.colmax = off;
    off = align256(off + sizeof(unsigned long long) * (size_t)n);
    L.total = off;
    return L;
}

}  // namespace

// Phase 1: exponents and digit tiles of A (m x k) and B (k x n) into the workspace (k <= kmax).
// Calls F<S>() for the runtime split count s (2..12).
template <template <int> class F, typename... Args>
static int dispatch_splits(int s, Args... args)
{
    switch (s) {
    case 2: return F<2>::run(args...);
    case 3: return F<3>::run(args...);
    case 4: return F<4>::run(args...);
    case 5: return F<5>::run(args...);
    case 6: return F<6>::run(args...);
    case 7: return F<7>::run(args...);
    case 8: return F<8>::run(args...);
    case 9: return F<9>::run(args...);
    case 10: return F<10>::run(args...);
    case 11: return F<11>::run(args...);
    case 12: return F<12>::run(args...);
    default:
        mgx_set_last_message("mgx_gemm_ozaki: %d splits is outside 2..12", s);
        return MGX_E_INVALID;
    }
}

template <int S>
struct SplitA {
    static int run(const double *A, int m, int k, int lda, int mp, int kblocks, const int *ea, uint8_t *da,
                   cudaStream_t stream)
    {
        oz::ozaki_split_a<S><<<mgx_sm_count() * 16, 256, 0, stream>>>(A, m, k, lda, mp, kblocks, ea, da);
        MGX_HOST_CHECK(cudaGetLastError());
        return MGX_SUCCESS;
    }
};

template <int S>
struct SplitB {
    static int run(const double *B, int k, int n, int ldb, int np, int kblocks, const int *eb, uint8_t *db,
                   cudaStream_t stream)
    {
        oz::ozaki_split_b<S><<<dim3(np / 128, kblocks), 256, 0, stream>>>(B, k, n, ldb, kblocks, eb, db);
        MGX_HOST_CHECK(cudaGetLastError());
        return MGX_SUCCESS;
    }
};

static int ozaki_split_a_impl(const double *A, int m, int k, int lda, int s, unsigned char *ws, const WsLayout &L,
                              cudaStream_t stream)
{
    int *status = mgx_device_status_ptr();
    int *ea = reinterpret_cast<int *>(ws + L.ea);
    const int kblocks = (k + 31) / 32;
    const int mp = (m + 127) / 128 * 128;
    oz::ozaki_row_exp<<<(m + 7) / 8, 256, 0, stream>>>(A, m, k, lda, ea, status);
    MGX_HOST_CHECK(cudaGetLastError());
    return dispatch_splits<SplitA>(s, A, m, k, lda, mp, kblocks, (const int *)ea, ws + L.da, stream);
}

static int ozaki_split_b_impl(const double *B, int n, int k, int ldb, int s, unsigned char *ws, const WsLayout &L,
                              cudaStream_t stream)
{
    int *status = mgx_device_status_ptr();
    int *eb = reinterpret_cast<int *>(ws + L.eb);
    unsigned long long *colmax = reinterpret_cast<unsigned long long *>(ws + L.colmax);
    const int kblocks = (k + 31) / 32;
    const int np = (n + 127) / 128 * 128;
    const int sms = mgx_sm_count();
    MGX_HOST_CHECK(cudaMemsetAsync(colmax, 0, sizeof(unsigned long long) * (size_t)n, stream));
    int ych = (sms * 8) / ((n + 255) / 256);
    if (ych > (k + 63) / 64) ych = (k + 63) / 64;
    if (ych < 1) ych = 1;
    oz::ozaki_col_max<<<dim3((n + 255) / 256, ych), 256, 0, stream>>>(B, k, n, ldb, colmax);
    MGX_HOST_CHECK(cudaGetLastError());
    oz::ozaki_col_exp<<<(n + 255) / 256, 256, 0, stream>>>(colmax, n, eb, status);
    MGX_HOST_CHECK(cudaGetLastError());
    return dispatch_splits<SplitB>(s, B, k, n, ldb, np, kblocks, (const int *)eb, ws + L.db, stream);
}

static int ozaki_split_impl(const double *A, const double *B, int m, int n, int k, int lda, int ldb, int s,
                            unsigned char *ws, const WsLayout &L, cudaStream_t stream)
{
    int rc = ozaki_split_a_impl(A, m, k, lda, s, ws, L, stream);
    if (rc == MGX_SUCCESS) rc = ozaki_split_b_impl(B, n, k, ldb, s, ws, L, stream);
    return rc;
}

// Phase 2: C (+)= recombined slice products (tcgen05 kernel).
int mgx_launch_splitk_reduce(double *C, int ldc, int beta_one, const double *P, int ld, size_t stride, int slices,
                             int m, int n, cudaStream_t stream);

// Split-K geometry of the Ozaki kernel (the FP64 kernel's rule): K blocks per slice and the
// number of non-empty slices.
static void ozaki_splitk_geometry(int k, int ksplit, int *kb_split, int *slices)
{
    const int kblocks = (k + 31) / 32 > 0 ? (k + 31) / 32 : 1;
    if (ksplit < 1) ksplit = 1;
    if (ksplit > kblocks) ksplit = kblocks;
    *kb_split = (kblocks + ksplit - 1) / ksplit;
    *slices = (kblocks + *kb_split - 1) / *kb_split;
}

static size_t ozaki_partial_bytes(int m, int n, int k, int ksplit)
{
    int kbs, slices;
    ozaki_splitk_geometry(k, ksplit, &kbs, &slices);
    if (slices <= 1 || m <= 0 || n <= 0) return 0;
    return align256((size_t)slices * (size_t)m * (size_t)((n + 1) & ~1) * sizeof(double));
}

// Arrival counters of the products launches' soft lockstep: two per device (one per stream of
// the host-buffer schedule), library-owned because the workspace of mgx_ozaki_multiply is const.
// Launches that run at the same time on other streams share them, which only weakens the
// lockstep (a wait ends after 20 us).
static __device__ unsigned int g_oz_sync[2];

static unsigned int *oz_sync_ptr(int slot)
{
    // optional: without it the products run with no lockstep
    void *p = mgx_symbol_address(reinterpret_cast<const void *>(&g_oz_sync), kMgxSymOzSync);
    return p ? static_cast<unsigned int *>(p) + (slot & 1) : nullptr;
}

static int ozaki_multiply_impl(double *C, int m, int n, int k, int ldc, int beta_one, int s, const unsigned char *ws,
                               const WsLayout &L, cudaStream_t stream, int ksplit = 1, double *partial = nullptr,
                               int slot = 0)
{
    oz::GemmParams p;
    memset(&p, 0, sizeof p);
    p.C = C;
    p.m = m;
    p.n = n;
    p.ldc = ldc;
    p.kblocks = (k + 31) / 32;
    p.splits = s;
    // weight sets of up to four groups, highest weights first
    int d = s + 1, ns = 0;
    while (d >= 2) {
        p.set_dhi[ns] = d;
        p.set_dlo[ns] = (d - 3 > 2) ? d - 3 : 2;
        d = p.set_dlo[ns] - 1;
        ++ns;
    }
    p.num_sets = ns;
    p.stage_bytes = 2 * s * oz::SLICE_TILE_BYTES;
    const int budget = 220 * 1024;
    p.stages = budget / p.stage_bytes;
    if (p.stages > 4) p.stages = 4;
    if (p.stages < 2) {
        mgx_set_last_message("mgx_gemm_ozaki: %d splits do not fit two pipeline stages", s);
        return MGX_E_UNSUPPORTED;
    }
    p.ea = reinterpret_cast<const int *>(ws + L.ea);
    p.eb = reinterpret_cast<const int *>(ws + L.eb);
    p.da = ws + L.da;
    p.db = ws + L.db;
    p.beta_one = beta_one;
    p.vec_store = ((ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    int kb_split = p.kblocks, slices = 1;
    if (ksplit > 1) ozaki_splitk_geometry(k, ksplit, &kb_split, &slices);
    p.ksplit = slices;
    p.kb_split = kb_split;
    p.partial = slices > 1 ? partial : nullptr;
    p.partial_ld = (n + 1) & ~1;
    p.partial_stride = (size_t)m * (size_t)p.partial_ld;
    if (slices > 1 && (!partial || (reinterpret_cast<uintptr_t>(partial) & 255))) {
        mgx_set_last_message("mgx_gemm_ozaki_splitk: no 256-byte aligned partial-product buffer");
        return MGX_E_WORKSPACE;
    }
    p.status = mgx_device_status_ptr();
    p.sync = oz_sync_ptr(slot);
    if (p.sync) MGX_HOST_CHECK(cudaMemsetAsync(p.sync, 0, sizeof(unsigned int), stream));
    const int smem = p.stages * p.stage_bytes + 1024 + 256;
    const int total = ((m + oz::TILE - 1) / oz::TILE) * ((n + oz::TILE - 1) / oz::TILE) * slices;
    const int sms = mgx_sm_count();
    const int grid = sms < total ? sms : total;
    if (grid < 1) return MGX_SUCCESS;
    auto launch = [&](auto kernel) -> int {
        MGX_HOST_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kernel<<<grid, oz::THREADS, smem, stream>>>(p);
        MGX_HOST_CHECK(cudaGetLastError());
        if (slices > 1)  // C (+)= slice 0 + slice 1 + ..., in slice order
            return mgx_launch_splitk_reduce(C, ldc, beta_one, partial, p.partial_ld, p.partial_stride, slices, m, n,
                                            stream);
        return MGX_SUCCESS;
    };
    switch (s) {
    case 2: return launch(oz::ozaki_gemm<2>);
    case 3: return launch(oz::ozaki_gemm<3>);
    case 4: return launch(oz::ozaki_gemm<4>);
    case 5: return launch(oz::ozaki_gemm<5>);
    case 6: return launch(oz::ozaki_gemm<6>);
    case 7: return launch(oz::ozaki_gemm<7>);
    case 8: return launch(oz::ozaki_gemm<8>);
    case 9: return launch(oz::ozaki_gemm<9>);
    case 10: return launch(oz::ozaki_gemm<10>);
    case 11: return launch(oz::ozaki_gemm<11>);
    case 12: return launch(oz::ozaki_gemm<12>);
    default:
        mgx_set_last_message("mgx_gemm_ozaki: %d splits is outside 2..12", s);
        return MGX_E_INVALID;
    }
}

static bool ozaki_args_ok(int m, int n, int k, int splits)
{
    return m >= 0 && n >= 0 && k >= 0 && splits >= 2 && splits <= oz::MAX_SPLITS;
}

static int ozaki_ws_check(void *workspace, size_t workspace_bytes, const WsLayout &L, const char *who)
{
    if (!workspace || workspace_bytes < L.total || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        mgx_set_last_message("%s: workspace needs %zu bytes, 256-byte aligned (got %zu)", who, L.total,
                             workspace_bytes);
        return MGX_E_WORKSPACE;
    }
    return MGX_SUCCESS;
}

extern "C" MGX_API size_t mgx_ozaki_workspace_size(int m, int n, int k, int splits)
{
    if (m < 0 || n < 0 || k < 0 || splits < 2 || splits > oz::MAX_SPLITS) return 0;
    return ws_layout(m, n, k, splits).total;
}

int mgx_ozaki_run(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb, int ldc,
                  int beta_one, int splits, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    if (!ozaki_args_ok(m, n, k, splits) || (m > 0 && n > 0 && !C) ||
        (m > 0 && n > 0 && k > 0 && (!A || !B || lda < k || ldb < n)) || (m > 0 && n > 0 && ldc < n)) {
        mgx_set_last_message("mgx_gemm_ozaki: invalid arguments m=%d n=%d k=%d splits=%d", m, n, k, splits);
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0) return MGX_SUCCESS;
    if (k == 0) {
        if (beta_one) return MGX_SUCCESS;
        MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)n * sizeof(double), m, stream));
        return MGX_SUCCESS;
    }
    const WsLayout L = ws_layout(m, n, k, splits);
    const int wrc = ozaki_ws_check(workspace, workspace_bytes, L, "mgx_gemm_ozaki");
    if (wrc != MGX_SUCCESS) return wrc;
    const int kmax = ozaki_kmax(splits);
    for (int k0 = 0; k0 < k; k0 += kmax) {
        const int kc = (k - k0 < kmax) ? k - k0 : kmax;
        unsigned char *ws = static_cast<unsigned char *>(workspace);
        int rc = ozaki_split_impl(A + k0, B + (size_t)k0 * ldb, m, n, kc, lda, ldb, splits, ws, L, stream);
        if (rc != MGX_SUCCESS) return rc;
        rc = ozaki_multiply_impl(C, m, n, kc, ldc, (k0 > 0) ? 1 : beta_one, splits, ws, L, stream);
        if (rc != MGX_SUCCESS) return rc;
    }
    return MGX_SUCCESS;
}

extern "C" MGX_API int mgx_gemm_ozaki(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                      int ldb, int ldc, int beta_one, int splits, void *workspace,
                                      size_t workspace_bytes, void *stream)
{
    return mgx_ozaki_run(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, splits, workspace, workspace_bytes,
                         (cudaStream_t)stream);
}

extern "C" MGX_API size_t mgx_ozaki_splitk_workspace_size(int m, int n, int k, int splits, int ksplit)
{
    if (m < 0 || n < 0 || k < 0 || splits < 2 || splits > oz::MAX_SPLITS || ksplit < 1) return 0;
    if (k > ozaki_kmax(splits)) return 0;
    return ws_layout(m, n, k, splits).total + ozaki_partial_bytes(m, n, k, ksplit);
}

extern "C" MGX_API int mgx_gemm_ozaki_splitk(const double *A, const double *B, double *C, int m, int n, int k,
                                             int lda, int ldb, int ldc, int beta_one, int splits, int ksplit,
                                             void *workspace, size_t workspace_bytes, void *stream)
{
    if (!ozaki_args_ok(m, n, k, splits) || ksplit < 1 || (m > 0 && n > 0 && !C) ||
        (m > 0 && n > 0 && k > 0 && (!A || !B || lda < k || ldb < n)) || (m > 0 && n > 0 && ldc < n)) {
        mgx_set_last_message("mgx_gemm_ozaki_splitk: invalid arguments m=%d n=%d k=%d splits=%d ksplit=%d", m, n, k,
                             splits, ksplit);
        return MGX_E_INVALID;
    }
    if (k > ozaki_kmax(splits)) {
        mgx_set_last_message("mgx_gemm_ozaki_splitk: k = %d is above one int32 accumulation (%d) for %d splits", k,
                             ozaki_kmax(splits), splits);
        return MGX_E_UNSUPPORTED;
    }
    if (ksplit == 1 || m == 0 || n == 0 || k == 0)
        return mgx_ozaki_run(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, splits, workspace, workspace_bytes,
                             (cudaStream_t)stream);
    const WsLayout L = ws_layout(m, n, k, splits);
    const size_t need = L.total + ozaki_partial_bytes(m, n, k, ksplit);
    if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
        mgx_set_last_message("mgx_gemm_ozaki_splitk: workspace of %zu bytes (aligned to 256) needed, %zu given", need,
                             workspace_bytes);
        return MGX_E_WORKSPACE;
    }
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ozaki_split_impl(A, B, m, n, k, lda, ldb, splits, ws, L, st);
    if (rc != MGX_SUCCESS) return rc;
    return ozaki_multiply_impl(C, m, n, k, ldc, beta_one ? 1 : 0, splits, ws, L, st, ksplit,
                               reinterpret_cast<double *>(ws + L.total));
}

// A-priori split choice.  The normwise error of the Ozaki form falls by close to two decimal
// digits per added slice and does not grow with K (exact integer accumulation); its level is
// set by how far the entries of a row or column spread below the row's (column's) maximum,
// which saturates after about ten binades.  Fitted on the oracle for uniform and wide-exponent
// inputs (K = 256 .. 1024):
//     err(s, R) ~= c(R) * 10^(-2 (s - 4)),  c(0) = 8.5e-9,  c(R >= 10) = 7.2e-8,
// floored at 5e-17 by the FP64 recombination.  The smallest s whose prediction, with a 1.25
// safety factor, meets `target` is returned (2..12).
extern "C" MGX_API int mgx_ozaki_choose_splits(int k, double exp_range, double target)
{
    (void)k;
    if (!(target > 0.0)) target = 1e-15;
    const double r = exp_range < 0.0 ? 0.0 : (exp_range > 10.0 ? 10.0 : exp_range);
    const double c = 8.5e-9 * pow(10.0, 0.93 * r / 10.0);
    for (int s = 2; s <= oz::MAX_SPLITS; ++s) {
        double e = c * pow(10.0, -2.0 * (s - 4));
        if (e < 5e-17) e = 5e-17;
        if (e * 1.25 <= target) return s;
    }
    return oz::MAX_SPLITS;
}

extern "C" MGX_API int mgx_ozaki_split(const double *A, const double *B, int m, int n, int k, int lda, int ldb,
                                       int splits, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!ozaki_args_ok(m, n, k, splits) || k > ozaki_kmax(splits) || (m > 0 && k > 0 && (!A || lda < k)) ||
        (n > 0 && k > 0 && (!B || ldb < n))) {
        mgx_set_last_message("mgx_ozaki_split: invalid arguments (k must be <= %d for %d splits)",
                             splits >= 2 && splits <= oz::MAX_SPLITS ? ozaki_kmax(splits) : 0, splits);
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0 || k == 0) return MGX_SUCCESS;
    const WsLayout L = ws_layout(m, n, k, splits);
    const int wrc = ozaki_ws_check(workspace, workspace_bytes, L, "mgx_ozaki_split");
    if (wrc != MGX_SUCCESS) return wrc;
    return ozaki_split_impl(A, B, m, n, k, lda, ldb, splits, static_cast<unsigned char *>(workspace), L,
                            (cudaStream_t)stream);
}

extern "C" MGX_API int mgx_ozaki_multiply(double *C, int m, int n, int k, int ldc, int beta_one, int splits,
                                          const void *workspace, size_t workspace_bytes, void *stream)
{
    if (!ozaki_args_ok(m, n, k, splits) || k > ozaki_kmax(splits) || (m > 0 && n > 0 && (!C || ldc < n))) {
        mgx_set_last_message("mgx_ozaki_multiply: invalid arguments");
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0) return MGX_SUCCESS;
    if (k == 0) {
        if (beta_one) return MGX_SUCCESS;
        MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)n * sizeof(double), m,
                                         (cudaStream_t)stream));
        return MGX_SUCCESS;
    }
    const WsLayout L = ws_layout(m, n, k, splits);
    const int wrc = ozaki_ws_check(const_cast<void *>(workspace), workspace_bytes, L, "mgx_ozaki_multiply");
    if (wrc != MGX_SUCCESS) return wrc;
    return ozaki_multiply_impl(C, m, n, k, ldc, beta_one ? 1 : 0, splits, static_cast<const unsigned char *>(workspace),
                               L, (cudaStream_t)stream);
}

extern "C" MGX_API int mgx_ozaki_kmax(int splits)
{
    if (splits < 2 || splits > oz::MAX_SPLITS) return 0;
    return ozaki_kmax(splits);
}

// ------------------------------------------------------------------------------------------
// Host-buffer entry point: PCIe copies overlapped with the product in a 2D block schedule.
//
// A is cut into row panels A_0..A_{Pm-1} and B into column panels B_0..B_{Pn-1} (multiples of
// 128 so every panel starts on a tile).  The copy stream sends A_0, B_0, A_1, B_1, ...; at step
// t the compute streams prepare the new panels (Ozaki: exponents and digit tiles) and compute
// every block (i, j) with max(i, j) = t, so the product grows as a square and work starts after
// the first two panels instead of after all of B.  Blocks alternate between two compute streams
// so one block's last wave overlaps the next block's first, and each finished block is copied
// back while the rest compute.  Every element is computed by the same kernel arithmetic as in
// one mgx_gemm_ozaki / mgx_gemm_fp64 call (exponents per row of A and per column of B over the
// whole K), so the result is bit-identical to it.
int mgx_launch_dgemm(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                     int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic);

// CRT form hooks (ozaki_crt.cu): whole-product workspace, panel preparation, block products.
size_t mgx_crt_host_ws_bytes(int M, int N, int K, int q);
int mgx_crt_host_rows(const double *A, int m, int lda, int r0, int M, int N, int K, int q, unsigned char *ws,
                      cudaStream_t stream);
int mgx_crt_host_cols(const double *B, int n, int ldb, int c0, int M, int N, int K, int q, unsigned char *ws,
                      cudaStream_t stream);
int mgx_crt_host_block(double *Cb, int ldc, int r0, int c0, int m, int n, int M, int N, int K, int q,
                       unsigned char *ws, cudaStream_t stream, int slot);
extern "C" MGX_API int mgx_crt_kmax(void);

namespace {

// Layout of rows [r0, ...) and columns [c0, ...) of a whole-problem workspace (r0, c0 multiples
// of 128): the digit tiles, exponents and column maxima of that sub-block.
WsLayout ws_sub(const WsLayout &L, int r0, int c0, int s)
{
    WsLayout S = L;
    const size_t tile_slab = (size_t)L.kblocks * s * oz::SLICE_TILE_BYTES;
    S.da = L.da + (size_t)(r0 / 128) * tile_slab;
    S.db = L.db + (size_t)(c0 / 128) * tile_slab;
    S.ea = L.ea + sizeof(int) * (size_t)r0;
    S.eb = L.eb + sizeof(int) * (size_t)c0;
    S.colmax = L.colmax + sizeof(unsigned long long) * (size_t)c0;
    return S;
}

int round_up(int x, int q) { return (x + q - 1) / q * q; }

}  // namespace

extern "C" MGX_API int mgx_gemm_host(const double *hA, const double *hB, double *hC, int m, int n, int k, int lda,
                                     int ldb, int ldc, int form, int splits, int panels, void *stream)
{
    if (m < 0 || n < 0 || k < 0 || (m > 0 && n > 0 && (!hC || ldc < n)) ||
        (m > 0 && n > 0 && k > 0 && (!hA || !hB || lda < k || ldb < n)) ||
        (form != MGX_FORM_FP64 && form != MGX_FORM_OZAKI && form != MGX_FORM_CRT) ||
        (form == MGX_FORM_OZAKI && (splits < 2 || splits > oz::MAX_SPLITS)) ||
        (form == MGX_FORM_CRT && (splits < 8 || splits > 16))) {
        mgx_set_last_message("mgx_gemm_host: invalid arguments");
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0) return MGX_SUCCESS;
    cudaStream_t s0 = (cudaStream_t)stream;
    if (panels < 1) panels = 1;
    if (panels > 64) panels = 64;  // 64 x 64 blocks at most: one event per block
    const bool ozaki = form == MGX_FORM_OZAKI && k > 0;
    const bool crt = form == MGX_FORM_CRT && k > 0;
    if (ozaki && k > ozaki_kmax(splits)) {
        mgx_set_last_message("mgx_gemm_host: k = %d is above one int32 accumulation (%d) for %d splits", k,
                             ozaki_kmax(splits), splits);
        return MGX_E_UNSUPPORTED;
    }
    if (crt && k > mgx_crt_kmax()) {
        mgx_set_last_message("mgx_gemm_host: k = %d is above one int32 residue accumulation (%d)", k, mgx_crt_kmax());
        return MGX_E_UNSUPPORTED;
    }
    const int align = crt ? 256 : 128;  // panels start on output tiles of the form
    const int prow = round_up((m + panels - 1) / panels, align), pcol = round_up((n + panels - 1) / panels, align);
    const int Pm = (m + prow - 1) / prow, Pn = (n + pcol - 1) / pcol, T = Pm > Pn ? Pm : Pn;
    auto r_at = [&](int i) { return i * prow < m ? i * prow : m; };
    auto c_at = [&](int j) { return j * pcol < n ? j * pcol : n; };
    const size_t kk = (size_t)(k > 0 ? k : 1);
    const WsLayout L = ozaki ? ws_layout(m, n, k, splits) : WsLayout{};
    // device copies of A, B and C, then the Ozaki workspace of the whole product
    const size_t bA = align256((size_t)m * kk * sizeof(double)), bB = align256(kk * n * sizeof(double)),
                 bC = align256((size_t)m * n * sizeof(double)),
                 bW = ozaki ? L.total : (crt ? mgx_crt_host_ws_bytes(m, n, k, splits) : 0);
    char *mem = nullptr;
    {
        const int arc = mgx_scratch_alloc(reinterpret_cast<void **>(&mem), bA + bB + bC + bW, s0);
        if (arc != MGX_SUCCESS) return arc;
    }
    double *dA = reinterpret_cast<double *>(mem);
    double *dB = reinterpret_cast<double *>(mem + bA);
    double *dC = reinterpret_cast<double *>(mem + bA + bB);
    unsigned char *ws = reinterpret_cast<unsigned char *>(mem + bA + bB + bC);

    cudaStream_t sin = nullptr, sout = nullptr, s1 = nullptr;
    // events: [0] start, [1] s1 done, [2] copies in done, [3] copies out done, then one per A panel,
    // per B panel, per step (panels prepared) and two per step (its row and column strips)
    const int nev = 4 + Pm + Pn + T + 2 * T;
    std::vector<cudaEvent_t> ev(nev, nullptr);
    cudaEvent_t *evA = ev.data() + 4, *evB = evA + Pm, *evS = evB + Pn, *evBlk = evS + T;
    int rc = MGX_SUCCESS;
    auto fail = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == MGX_SUCCESS) {
            mgx_set_last_cuda_error(e, what, __FILE__, __LINE__);
            rc = MGX_E_CUDA;
        }
    };
    fail(cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking), "stream");
    fail(cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking), "stream");
    fail(cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < nev && rc == MGX_SUCCESS; ++i) fail(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming), "event");
    if (rc == MGX_SUCCESS) {
        fail(cudaEventRecord(ev[0], s0), "record");
        fail(cudaStreamWaitEvent(sin, ev[0], 0), "wait");
        fail(cudaStreamWaitEvent(sout, ev[0], 0), "wait");
        fail(cudaStreamWaitEvent(s1, ev[0], 0), "wait");
    }
    // copies in: A_0, B_0, A_1, B_1, ...
    for (int t = 0; t < T && rc == MGX_SUCCESS; ++t) {
        if (t < Pm) {
            const int r0 = r_at(t), r1 = r_at(t + 1);
            if (k > 0)
                fail(cudaMemcpy2DAsync(dA + (size_t)r0 * kk, kk * sizeof(double), hA + (size_t)r0 * lda,
                                       (size_t)lda * sizeof(double), kk * sizeof(double), r1 - r0,
                                       cudaMemcpyHostToDevice, sin), "copy A panel");
            fail(cudaEventRecord(evA[t], sin), "record");
        }
        if (t < Pn) {
            const int c0 = c_at(t), c1 = c_at(t + 1);
            if (k > 0)
                fail(cudaMemcpy2DAsync(dB + c0, (size_t)n * sizeof(double), hB + c0, (size_t)ldb * sizeof(double),
                                       (size_t)(c1 - c0) * sizeof(double), k, cudaMemcpyHostToDevice, sin),
                     "copy B panel");
            fail(cudaEventRecord(evB[t], sin), "record");
        }
    }
    // One rectangle of C, rows [r0, r1) x columns [c0, c1) (on the panel grid), computed as one
    // product on s0 or s1 (alternating) and copied back on sout as soon as it is done.
    int blk = 0;
    auto run_rect = [&](int r0, int r1, int c0, int c1) {
        if (rc != MGX_SUCCESS || r1 <= r0 || c1 <= c0) return;
        cudaStream_t cs = (blk & 1) ? s1 : s0;
        double *Cb = dC + (size_t)r0 * n + c0;
        if (ozaki) {
            const WsLayout S = ws_sub(L, r0, c0, splits);
            rc = ozaki_multiply_impl(Cb, r1 - r0, c1 - c0, k, n, 0, splits, ws, S, cs, 1, nullptr, blk & 1);
        } else if (crt) {
            rc = mgx_crt_host_block(Cb, n, r0, c0, r1 - r0, c1 - c0, m, n, k, splits, ws, cs, blk & 1);
        } else {
            rc = mgx_launch_dgemm(dA + (size_t)r0 * kk, dB + c0, Cb, r1 - r0, c1 - c0, k, 0, k, k, (int)kk, n, n, 0, cs,
                                  0);
        }
        fail(cudaEventRecord(evBlk[blk], cs), "record");
        fail(cudaStreamWaitEvent(sout, evBlk[blk], 0), "wait");
        fail(cudaMemcpy2DAsync(hC + (size_t)r0 * ldc + c0, (size_t)ldc * sizeof(double), Cb, (size_t)n * sizeof(double),
                               (size_t)(c1 - c0) * sizeof(double), r1 - r0, cudaMemcpyDeviceToHost, sout),
             "copy C block");
        ++blk;
    };
    for (int t = 0; t < T && rc == MGX_SUCCESS; ++t) {
        // prepare the panels that arrived at this step (on s0, in order)
        if (t < Pm) {
            fail(cudaStreamWaitEvent(s0, evA[t], 0), "wait");
            if (ozaki && rc == MGX_SUCCESS) {
                const int r0 = r_at(t), r1 = r_at(t + 1);
                rc = ozaki_split_a_impl(dA + (size_t)r0 * kk, r1 - r0, k, (int)kk, splits, ws, ws_sub(L, r0, 0, splits),
                                        s0);
            }
            if (crt && rc == MGX_SUCCESS) {
                const int r0 = r_at(t), r1 = r_at(t + 1);
                rc = mgx_crt_host_rows(dA + (size_t)r0 * kk, r1 - r0, (int)kk, r0, m, n, k, splits, ws, s0);
            }
        }
        if (t < Pn) {
            fail(cudaStreamWaitEvent(s0, evB[t], 0), "wait");
            if (ozaki && rc == MGX_SUCCESS) {
                const int c0 = c_at(t), c1 = c_at(t + 1);
                rc = ozaki_split_b_impl(dB + c0, c1 - c0, k, n, splits, ws, ws_sub(L, 0, c0, splits), s0);
            }
            if (crt && rc == MGX_SUCCESS) {
                const int c0 = c_at(t), c1 = c_at(t + 1);
                rc = mgx_crt_host_cols(dB + c0, c1 - c0, n, c0, m, n, k, splits, ws, s0);
            }
        }
        fail(cudaEventRecord(evS[t], s0), "record");
        fail(cudaStreamWaitEvent(s1, evS[t], 0), "wait");
        // every block (i, j) with max(i, j) = t, as two products: the row strip (t, 0..t) and the
        // column strip (0..t-1, t).  Each element's arithmetic does not depend on the rectangle it
        // is computed in, so the result is that of the device-buffer entry points.
        if (t < Pm) run_rect(r_at(t), r_at(t + 1), 0, c_at(t + 1 < Pn ? t + 1 : Pn));
        if (t < Pn) run_rect(0, r_at(t < Pm ? t : Pm), c_at(t), c_at(t + 1));
    }
    // join the side streams back into the caller's stream, then release the buffers
    if (s1) {
        cudaEventRecord(ev[1], s1);
        cudaStreamWaitEvent(s0, ev[1], 0);
    }
    if (sin) {
        cudaEventRecord(ev[2], sin);
        cudaStreamWaitEvent(s0, ev[2], 0);
    }
    if (sout) {
        cudaEventRecord(ev[3], sout);
        cudaStreamWaitEvent(s0, ev[3], 0);
    }
    cudaFreeAsync(mem, s0);
    for (int i = 0; i < nev; ++i)
        if (ev[i]) cudaEventDestroy(ev[i]);
    if (sin) cudaStreamDestroy(sin);
    if (sout) cudaStreamDestroy(sout);
    if (s1) cudaStreamDestroy(s1);
    return rc;
}

// ------------------------------------------------------------------------------------------
// Ozaki product with no device allocation.
//
// Some callers cannot allocate device memory when they call in:
//   - code inside a CUDA stream capture that must not add allocation nodes to its graph;
//   - applications whose own allocator already owns the device memory (an MPI or NVSHMEM
//     symmetric heap, a framework's caching allocator);
//   - services that forbid allocation after start-up (real-time loops).
// For them this entry point uses a fixed workspace: the file-scope device array below,
// MGX_OZAKI_NOALLOC_BYTES (32 MiB) long.  Every GPU that loads this library holds it until the
// process exits.  Products whose workspace would not fit are rejected.
static __device__ __align__(256) unsigned char g_ozaki_noalloc_ws[MGX_OZAKI_NOALLOC_BYTES];

extern "C" MGX_API int mgx_gemm_ozaki_noalloc(const double *A, const double *B, double *C, int m, int n, int k,
                                              int lda, int ldb, int ldc, int beta_one, int splits, void *stream)
{
    if (splits < 2 || splits > oz::MAX_SPLITS || m < 0 || n < 0 || k < 0) {
        mgx_set_last_message("mgx_gemm_ozaki_noalloc: invalid arguments m=%d n=%d k=%d splits=%d", m, n, k, splits);
        return MGX_E_INVALID;
    }
    const size_t need = ws_layout(m, n, k, splits).total;
    if (need > (size_t)MGX_OZAKI_NOALLOC_BYTES) {
        mgx_set_last_message("mgx_gemm_ozaki_noalloc: this product needs %zu bytes of workspace, more than the "
                             "fixed %u-byte array; use mgx_gemm_ozaki with a caller-provided workspace",
                             need, (unsigned)MGX_OZAKI_NOALLOC_BYTES);
        return MGX_E_WORKSPACE;
    }
    // The array's name is a host-side stand-in; the kernels need its device address, taken with
    // that device current on the first call on each device (which should therefore come before
    // any stream capture) and again only if the device's context has changed since.
    cudaError_t e = cudaSuccess;
    void *ws = mgx_symbol_address(reinterpret_cast<const void *>(&g_ozaki_noalloc_ws), kMgxSymOzakiNoalloc, &e);
    if (!ws) {
        mgx_set_last_cuda_error(e, "cudaGetSymbolAddress(g_ozaki_noalloc_ws)", __FILE__, __LINE__);
        return MGX_E_CUDA;
    }
    // Calls share the array: two calls whose work overlaps on the GPU (different streams, no
    // ordering between them) race on it.  Everything a call reads from the array it first writes
    // (the column maxima are cleared by the split phase), so the previous call's contents do not
    // matter.
    return mgx_ozaki_run(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, splits, ws,
                         (size_t)MGX_OZAKI_NOALLOC_BYTES, (cudaStream_t)stream);
}
