// fp64_gemm.cu -- native FP64 GEMM for sm_100a on the FP64 tensor-core path (DMMA).
//
// Replaces the arithmetic of MGXBench's sharedABMultiply / sharedABMultiplyAccumulate
// (1D-row-block/mulmat_kernel.cu:39-80 and 100-142): C = A*B, or C += (A*B summed over the chunk).
//
// Design (one CTA per SM, persistent):
//   * warpgroup 0 (producer, 40 registers): one lane of warp 0 issues TMA 2D tile loads of A
//     (128 x 32 doubles, two 128-byte swizzled boxes) and B (32 x 128 doubles, eight boxes) into
//     a 3-stage ring, each stage guarded by a full/empty mbarrier pair.  No multicast.
//   * warpgroups 1-2 (consumers, 232 registers): a 2 x 4 warp grid, each warp owning a 64 x 32 block of the
//     128 x 128 output tile as 4 x 4 DMMA m16n8k8 accumulators (64 doubles per lane).
//   * The reduction index is permuted inside every group of 8 (physical order 0,1,4,5 | 2,3,6,7)
//     identically for A and B, so each fragment load from the swizzled tiles hits every shared
//     memory bank exactly twice (the minimum for 256 bytes).
//   * Epilogue: C = acc (beta 0) or C = C + acc (beta 1), one rounding, as the reference.
// Operands TMA cannot describe (odd leading dimension, odd K offset, unaligned base) are first
// copied into stream-ordered scratch with an even pitch.  A variant whose producer warp loads
// with plain global loads covers the one case with nothing to copy (a chunk wholly past k_total).
#include <atomic>
#include <cstdio>

#include "mgx_common.cuh"

namespace mgx {
namespace fp64 {

// Output tiles are BM x 128 with BM = 128 (the default) or 64 (the small-product tile: twice the
// work items, so a product with few 128 x 128 tiles fills more of the 148 SMs); both reduce each
// element over K in the same order, so their results are bit-identical.
constexpr int BM = 128, BN = 128, BK = 32;
constexpr int BM_SMALL = 64;
constexpr int CWARPS = 8;
constexpr int PRODUCER_WARPS = 4;                         // one warpgroup; its warp 0 issues the loads
constexpr int THREADS = (CWARPS + PRODUCER_WARPS) * 32;   // 384 = 3 warpgroups
// Register split (setmaxnreg): the block launches with 384 x 168 registers; the producer
// warpgroup gives back down to 40 each and the two consumer warpgroups take 232 each:
// 128 x 40 + 256 x 232 = 64512 = 384 x 168.  The host refuses to launch unless the compiled
// kernel has exactly LAUNCH_REGS registers per thread, so the split always adds up.
constexpr int LAUNCH_REGS = 168, PRODUCER_REGS = 40, CONSUMER_REGS = 232;
static_assert(PRODUCER_WARPS * 32 * PRODUCER_REGS + CWARPS * 32 * CONSUMER_REGS == THREADS * LAUNCH_REGS,
              "register split must equal the launch budget");
constexpr int B_BOX_BYTES = BK * 128;        // 32 rows x 16 doubles
constexpr int B_STAGE_BYTES = 8 * B_BOX_BYTES;

// Shared-memory geometry of a BM-row tile: A as two boxes of BM rows x 16 doubles, B as eight
// boxes of 32 rows x 16 doubles; 3 stages of 64 KiB for BM = 128, 4 of 48 KiB for BM = 64.
template <int TBM>
struct Geo {
    static constexpr int A_BOX_BYTES = TBM * 128;
    static constexpr int A_STAGE_BYTES = 2 * A_BOX_BYTES;
    static constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
    static constexpr int STAGES = TBM == 128 ? 3 : 4;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr int MT = TBM / 32;          // 16-row MMA tiles per consumer warp (2 x 4 warp grid)
    static constexpr int GROUP_M = 1024 / TBM;   // raster groups of 1024 rows
};

struct Params {
    const double *A;  // generic loader only
    const double *B;
    double *C;
    int m, n;
    int k_len;        // reduction length handled by this call
    int a_x0;         // first column of A (k_offset)
    int a_x_end;      // A columns >= a_x_end read as zero (min(k_total, k_offset + k_chunk))
    int b_rows;       // rows of B (chunk) that exist; rows >= b_rows read as zero
    int lda, ldb, ldc;
    int beta_one;
    int vec_store;    // C rows 16-byte aligned (ldc even, C aligned)
    int *status;
    const int4 *tiles;  // optional work list (m0, n0, m_end, n_end); null -> regular tiling of m x n
    int num_tiles;
    int panel_kb;       // > 0: add the accumulator into C after every panel_kb K blocks (SUMMA panels)
    int streamk;        // stream-K (64-row tiles, regular tiling): CTA c takes the K-block units
                        // [c U / G, (c + 1) U / G) of all U = tiles x kblocks, G = gridDim.x
    unsigned long long *sk_tickets;  // stream-K: one arrival ticket per tile and consumer warp
    unsigned long long sk_epoch;     // stream-K: this launch's ticket tag (a ticket of another tag counts 0)
    double *sk_partial; // stream-K: two partial accumulators per CTA (its first and last segment)
    int ksplit;         // > 1: split-K -- work item w is (tile w / ksplit, K slice w % ksplit)
    int kb_split;       // K blocks per slice
    double *partial;    // split-K: slice s of the product goes to partial + s * partial_stride
    int partial_ld;     // even, so the partial rows are 16-byte aligned
    size_t partial_stride;
};

template <int TBM>
__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int &tm, int &tn);

// Tile geometry.  n0 is where the tile's columns start in B and C; it is always even, because it
// is the x coordinate of B's TMA boxes and TMA needs x * 8 bytes to be a multiple of 16.  A work
// item may begin at an odd column n_lo (uneven SUMMA blocks): its tile then starts one column
// earlier and the columns below n_lo, which belong to the neighbouring block, are not stored.
template <int TBM>
__device__ __forceinline__ void tile_bounds(const Params &p, int tile, int tiles_m, int tiles_n, int &m0, int &n0,
                                            int &m_end, int &n_end, int &n_lo)
{
    if (p.tiles) {
        const int4 t = p.tiles[tile];
        m0 = t.x;
        n_lo = t.y;
        n0 = t.y & ~1;
        m_end = t.z;
        n_end = t.w;
    } else {
        int tm, tn;
        tile_coords<TBM>(tile, tiles_m, tiles_n, tm, tn);
        m0 = tm * TBM;
        n0 = tn * BN;
        n_lo = n0;
        m_end = p.m;
        n_end = p.n;
    }
}

template <int TBM>
__device__ __forceinline__ void tile_coords(int tile, int tiles_m, int tiles_n, int &tm, int &tn)
{
    constexpr int GROUP_M = Geo<TBM>::GROUP_M;
    const int per_group = GROUP_M * tiles_n;
    const int group = tile / per_group;
    const int first_m = group * GROUP_M;
    const int gsize = min(tiles_m - first_m, GROUP_M);
    const int r = tile % per_group;
    tm = first_m + r % gsize;
    tn = r / gsize;
}

// Work item w: its output tile and the K blocks [kb_begin, kb_end) it reduces over.
template <int TBM>
__device__ __forceinline__ void item_bounds(const Params &p, int w, int tiles_m, int tiles_n, int kblocks, int &m0,
                                            int &n0, int &m_end, int &n_end, int &n_lo, int &kb_begin, int &kb_end,
                                            int &slice)
{
    const int tile = p.ksplit > 1 ? w / p.ksplit : w;
    slice = p.ksplit > 1 ? w % p.ksplit : 0;
    tile_bounds<TBM>(p, tile, tiles_m, tiles_n, m0, n0, m_end, n_end, n_lo);
    kb_begin = slice * p.kb_split;
    kb_end = min(kblocks, kb_begin + p.kb_split);
}

// The work of one CTA, shared by the producer and the consumers: regular items (tiles or
// (tile, K slice) pairs, every gridDim.x-th), or in stream-K mode the segments -- pieces of
// consecutive tiles' K ranges -- of this CTA's contiguous share of all K-block units.
struct Walk {
    long long u, u_end;  // stream-K: next unit and the end of this CTA's share
    int w;               // regular: next work item
};

__device__ __forceinline__ long long sk_begin(long long c, long long U, long long G) { return c * U / G; }

// CTA whose share holds unit u (sk_begin(c) <= u < sk_begin(c + 1)).
__device__ __forceinline__ int sk_owner(long long u, long long U, long long G)
{
    return (int)(((u + 1) * G + U - 1) / U - 1);
}

__device__ __forceinline__ void walk_init(const Params &p, int tiles, int kblocks, Walk &s)
{
    const long long U = (long long)tiles * kblocks;
    s.u = sk_begin(blockIdx.x, U, gridDim.x);
    s.u_end = sk_begin(blockIdx.x + 1, U, gridDim.x);
    s.w = blockIdx.x;
    (void)p;
}

template <int TBM>
__device__ __forceinline__ bool walk_next(const Params &p, int tiles_m, int tiles_n, int kblocks, int items, Walk &s,
                                          int &tile, int &m0, int &n0, int &m_end, int &n_end, int &n_lo,
                                          int &kb_begin, int &kb_end, int &slice)
{
    if (p.streamk) {
        if (s.u >= s.u_end) return false;
        tile = (int)(s.u / kblocks);
        kb_begin = (int)(s.u - (long long)tile * kblocks);
        const long long left = s.u_end - s.u;
        kb_end = (long long)(kblocks - kb_begin) < left ? kblocks : kb_begin + (int)left;
        slice = 0;
        s.u += kb_end - kb_begin;
        tile_bounds<TBM>(p, tile, tiles_m, tiles_n, m0, n0, m_end, n_end, n_lo);
        return true;
    }
    if (s.w >= items) return false;
    tile = p.ksplit > 1 ? s.w / p.ksplit : s.w;
    item_bounds<TBM>(p, s.w, tiles_m, tiles_n, kblocks, m0, n0, m_end, n_end, n_lo, kb_begin, kb_end, slice);
    s.w += gridDim.x;
    return true;
}

// Swizzled byte offset of element (row, col16) inside a box whose rows are 128 bytes.
__device__ __forceinline__ uint32_t sw128(int row, int col16)
{
    return row * 128 + ((((col16 >> 1) ^ (row & 7)) & 7) << 4) + ((col16 & 1) << 3);
}

// Stream-K tickets: (launch tag << 8) | arrivals.  A ticket written by an earlier launch (another
// tag), or never written, counts as no arrivals, so the tickets need no reset between launches.
// Arrivals per tile are at most the grid size, below 256.
__device__ __forceinline__ int ticket_count(unsigned long long *tk, unsigned long long tag)
{
    const unsigned long long v = atomicAdd(tk, 0ull);
    return (v >> 8) == tag ? (int)(v & 255u) : 0;
}

// Takes a ticket; returns the arrivals before this one, or -1 (status set) if the compare-and-swap
// never got through (each failure is another arrival's success, so this does not happen).
__device__ __forceinline__ int ticket_take(unsigned long long *tk, unsigned long long tag, int *status)
{
    unsigned long long old = atomicAdd(tk, 0ull);
    for (int it = 0; it < 4096; ++it) {
        const unsigned long long cur = (old >> 8) == tag ? old : (tag << 8);
        const unsigned long long prev = atomicCAS(tk, old, cur + 1);
        if (prev == old) return (int)(cur & 255u);
        old = prev;
    }
    record_status(status, kDevTicket);
    return -1;
}

template <int TBM, bool USE_TMA, bool PANELS>
__global__ void __launch_bounds__(THREADS, 1)
    dgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params p)
{
    using G = Geo<TBM>;
    constexpr int STAGES = G::STAGES, STAGE_BYTES = G::STAGE_BYTES, A_STAGE_BYTES = G::A_STAGE_BYTES;
    constexpr int A_BOX_BYTES = G::A_BOX_BYTES, MT = G::MT;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                            ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], USE_TMA ? 1 : 32);
            mbar_init(&empty[s], CWARPS);
        }
        fence_barrier_init();
    }
    if (USE_TMA && warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    __syncthreads();
    // Launched as a programmatic dependent: everything above overlapped the previous kernel in the
    // stream; nothing below reads or writes memory before that kernel has finished.  The next
    // kernel may be scheduled now (it cannot share an SM with this one, and waits the same way).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    const int tiles_m = (p.m + TBM - 1) / TBM;
    const int tiles_n = (p.n + BN - 1) / BN;
    const int tiles = p.tiles ? p.num_tiles : tiles_m * tiles_n;
    const int kblocks = (p.k_len + BK - 1) / BK;
    const int items = tiles * (p.ksplit > 1 ? p.ksplit : 1);

    if (warp < PRODUCER_WARPS) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(PRODUCER_REGS));
        if (warp != 0) return;
        // ------------------------------------------------------------ producer
        int stage = 0;
        uint32_t phase = 0;
        int armed_parity[STAGES];
        for (int s = 0; s < STAGES; ++s) armed_parity[s] = -1;
        bool ok = true;
        Walk walk;
        walk_init(p, tiles, kblocks, walk);
        int tile, m0, n0, m_end, n_end, n_lo, kb_begin, kb_end, slice;
        while (ok && walk_next<TBM>(p, tiles_m, tiles_n, kblocks, items, walk, tile, m0, n0, m_end, n_end, n_lo,
                                    kb_begin, kb_end, slice)) {
            for (int kb = kb_begin; kb < kb_end; ++kb) {
                bool got = true;
                if (lane == 0) got = mbar_wait_bounded(&empty[stage], phase ^ 1u, p.status, kDevTimeoutEmpty);
                got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
                __syncwarp();
                if (!got) {
                    ok = false;
                    break;
                }
                unsigned char *sA = smem + stage * STAGE_BYTES;
                unsigned char *sB = sA + A_STAGE_BYTES;
                const int k0 = kb * BK;
                if (USE_TMA) {
                    if (lane == 0) {
                        mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                        armed_parity[stage] = (int)phase;
                        tma_load_2d(sA, &tmA, p.a_x0 + k0, m0, &full[stage]);
                        tma_load_2d(sA + A_BOX_BYTES, &tmA, p.a_x0 + k0 + 16, m0, &full[stage]);
                        for (int j = 0; j < 8; ++j) tma_load_2d(sB + j * B_BOX_BYTES, &tmB, n0 + 16 * j, k0, &full[stage]);
                    }
                } else {
                    // A tile: TBM rows x 32 columns, one row per warp iteration (coalesced)
                    for (int r = 0; r < TBM; ++r) {
                        const int row = m0 + r;
                        const int kk = k0 + lane;
                        const int acol = p.a_x0 + kk;
                        double v = 0.0;
                        if (row < p.m && kk < p.k_len && acol < p.a_x_end) v = p.A[(size_t)row * p.lda + acol];
                        const int h = lane >> 4;
                        *reinterpret_cast<double *>(sA + h * A_BOX_BYTES + sw128(r, lane & 15)) = v;
                    }
                    // B tile: 32 rows x 128 columns
                    for (int r = 0; r < BK; ++r) {
                        const int brow = k0 + r;
                        for (int c = lane; c < BN; c += 32) {
                            const int col = n0 + c;
                            double v = 0.0;
                            if (brow < p.b_rows && brow < p.k_len && col < p.n) v = p.B[(size_t)brow * p.ldb + col];
                            *reinterpret_cast<double *>(sB + (c >> 4) * B_BOX_BYTES + sw128(r, c & 15)) = v;
                        }
                    }
                    mbar_arrive(&full[stage]);
                }
                if (++stage == STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
        }
        // Never leave the CTA with a tensor copy still writing its shared memory.
        if (USE_TMA && lane == 0) {
            for (int s = 0; s < STAGES; ++s)
                if (armed_parity[s] >= 0) mbar_wait_bounded(&full[s], (uint32_t)armed_parity[s], p.status, kDevTimeoutFull);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(CONSUMER_REGS));
    const int cw = warp - PRODUCER_WARPS;
    const int wm = cw >> 2;  // 0..1
    const int wn = cw & 3;   // 0..3
    const int g = lane >> 2;
    const int t = lane & 3;

    int stage = 0;
    uint32_t phase = 0;
    const uint32_t smem_base = smem_u32(smem);

    // Per-lane parts of the fragment addresses (see the header comment for the permutation).
    uint32_t a_row_off[MT][2];
    for (int mt = 0; mt < MT; ++mt)
        for (int h = 0; h < 2; ++h)
            a_row_off[mt][h] = (uint32_t)((wm * (TBM / 2) + mt * 16 + h * 8 + g) * 128 + ((t & 1) << 3));

    // dst (+)= acc for this lane's fragments, masked to the tile's bounds (dst = C, or a split-K
    // slice of the partial products).
    auto store_acc = [&](double (&acc)[MT][4][4], int m0, int n0, int m_end, int n_end, int n_lo, int beta_one,
                         double *dst_base, int ld, int vec_store) {
        if (PANELS) {
            // SUMMA panels: C += acc as fire-and-forget L2 reductions, so the consumers go on with
            // the next panel instead of waiting for C to load.  An FP64 atomic add rounds like
            // the load-add-store it replaces; one thread owns each element, and its adds to one
            // address stay in program order, so the panel order of the sums is kept.
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = m0 + wm * (TBM / 2) + mt * 16 + h * 8 + g;
                    if (row >= m_end) continue;
                    double *crow = dst_base + (size_t)row * ld;
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        const int col = n0 + wn * 32 + nt * 8 + 2 * t;
                        if (col < n_end && col >= n_lo)
                            asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(crow + col),
                                         "d"(acc[mt][nt][2 * h])
                                         : "memory");
                        if (col + 1 < n_end && col + 1 >= n_lo)
                            asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(crow + col + 1),
                                         "d"(acc[mt][nt][2 * h + 1])
                                         : "memory");
                    }
                }
            }
        } else {
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = m0 + wm * (TBM / 2) + mt * 16 + h * 8 + g;
                    if (row >= m_end) continue;
                    double *crow = dst_base + (size_t)row * ld;
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        const int col = n0 + wn * 32 + nt * 8 + 2 * t;
                        double v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
                        if (vec_store && col + 1 < n_end && col >= n_lo) {
                            double2 *dst = reinterpret_cast<double2 *>(crow + col);
                            if (beta_one) {
                                const double2 old = *dst;
                                v0 = old.x + v0;
                                v1 = old.y + v1;
                            }
                            *dst = make_double2(v0, v1);
                        } else {
                            if (col < n_end && col >= n_lo) crow[col] = beta_one ? crow[col] + v0 : v0;
                            if (col + 1 < n_end && col + 1 >= n_lo)
                                crow[col + 1] = beta_one ? crow[col + 1] + v1 : v1;
                        }
                    }
                }
            }
        }
    };

    Walk walk;
    walk_init(p, tiles, kblocks, walk);
    int tile, m0, n0, m_end, n_end, n_lo, kb_begin, kb_end, slice;
    while (walk_next<TBM>(p, tiles_m, tiles_n, kblocks, items, walk, tile, m0, n0, m_end, n_end, n_lo, kb_begin,
                          kb_end, slice)) {

        double acc[MT][4][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

        bool ok = true;
        for (int kb = kb_begin; kb < kb_end; ++kb) {
            bool got = true;
            if (lane == 0) got = mbar_wait_bounded(&full[stage], phase, p.status, kDevTimeoutFull);
            got = __shfl_sync(0xffffffffu, got ? 1 : 0, 0) != 0;
            if (!got) {
                ok = false;
                break;
            }
            const uint32_t sA = smem_base + stage * STAGE_BYTES;
            const uint32_t sB = sA + A_STAGE_BYTES;
#pragma unroll
            for (int kb8 = 0; kb8 < 4; ++kb8) {
                // One m16n8k8 per (mt, nt): logical k t -> physical k (t&1) + 4(t>>1), logical t+4 ->
                // the same plus 2, i.e. the permutation 0,1,4,5 | 2,3,6,7 of the group of 8.  B
                // fragments are loaded once per group; A fragments one 16-row tile at a time.
                double bf[4][2];
#pragma unroll
                for (int step = 0; step < 2; ++step) {
                    const int phys = (t & 1) + ((t >> 1) << 2) + 2 * step;
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) {
                        const int j = wn * 2 + (nt >> 1);
                        const int krow = kb8 * 8 + phys;
                        const uint32_t off = (uint32_t)(j * B_BOX_BYTES + krow * 128 +
                                                        (((((nt & 1) * 4) + (g >> 1)) ^ phys) << 4) + ((g & 1) << 3));
                        bf[nt][step] = lds_f64(sB + off);
                    }
                }
                const uint32_t abase = sA + (kb8 >> 1) * A_BOX_BYTES;
                const uint32_t c0 = (uint32_t)((((kb8 & 1) * 4 + (t >> 1) * 2) ^ g) << 4);
                const uint32_t c1 = (uint32_t)((((kb8 & 1) * 4 + (t >> 1) * 2 + 1) ^ g) << 4);
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    double af[4];
                    af[0] = lds_f64(abase + c0 + a_row_off[mt][0]);
                    af[1] = lds_f64(abase + c0 + a_row_off[mt][1]);
                    af[2] = lds_f64(abase + c1 + a_row_off[mt][0]);
                    af[3] = lds_f64(abase + c1 + a_row_off[mt][1]);
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt) dmma_16x8x8(acc[mt][nt], af, bf[nt]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1u;
            }
            if (PANELS && ((kb + 1) % p.panel_kb == 0) && kb + 1 < kblocks) {
                // end of a SUMMA panel: C_ij += panel product, one rounding, as the reference
                store_acc(acc, m0, n0, m_end, n_end, n_lo, 1, p.C, p.ldc, p.vec_store);
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
            }
        }
        if (!ok) return;
        if (p.streamk) {
            if constexpr (TBM == BM_SMALL && !PANELS) {
                // A tile whose K range spans several CTAs' shares is finished by the CTA that
                // arrives last at its ticket: every piece's accumulator goes to that CTA's partial
                // slot, and the last arrival adds the pieces in K order (p0 + p1) + p2 ... and
                // stores C.  No CTA waits for another.
                const long long U = (long long)tiles * kblocks, NG = gridDim.x;
                const long long t0 = (long long)tile * kblocks;
                const int c0 = sk_owner(t0, U, NG), pieces = sk_owner(t0 + kblocks - 1, U, NG) - c0 + 1;
                if (pieces == 1) {
                    store_acc(acc, m0, n0, m_end, n_end, n_lo, p.beta_one, p.C, p.ldc, p.vec_store);
                } else {
                    // Each consumer warp owns the same fragment of the tile in every piece, so it
                    // finishes that fragment on its own: a ticket per (tile, warp), and no barrier
                    // between the warps (a warp that gave up on a wait cannot block the others).
                    constexpr int NACC = MT * 16;
                    constexpr size_t PART = (size_t)CWARPS * 32 * NACC;  // doubles per partial slot
                    const int ct = threadIdx.x - PRODUCER_WARPS * 32;     // consumer thread 0..255
                    const int j = (int)blockIdx.x - c0;                    // this CTA's piece
                    const int slot = (t0 + kb_begin == sk_begin(blockIdx.x, U, NG)) ? 0 : 1;
                    double(&af)[NACC] = reinterpret_cast<double(&)[NACC]>(acc);
                    unsigned long long *ticket = p.sk_tickets + (size_t)tile * CWARPS + cw;
                    // The head piece is usually computed last (at the end of its CTA's share):
                    // when every later piece has taken its ticket, it finishes the tile without
                    // writing its own partial.
                    int last = 0;
                    if (j == 0) {
                        if (lane == 0) last = ticket_count(ticket, p.sk_epoch) == pieces - 1;
                        last = __shfl_sync(0xffffffffu, last, 0);
                    }
                    if (!last) {
                        double *mine = p.sk_partial + ((size_t)blockIdx.x * 2 + slot) * PART;
#pragma unroll
                        for (int i = 0; i < NACC; ++i) __stcg(mine + (size_t)i * (CWARPS * 32) + ct, af[i]);
                        __threadfence();
                        __syncwarp();
                        if (lane == 0) last = ticket_take(ticket, p.sk_epoch, p.status) == pieces - 1;
                        last = __shfl_sync(0xffffffffu, last, 0);
                    }
                    if (last) {
                        __threadfence();
                        double tot[NACC];
                        const int slot0 = (sk_begin(c0, U, NG) == t0) ? 0 : 1;
                        const double *p0 = p.sk_partial + ((size_t)c0 * 2 + slot0) * PART;
#pragma unroll
                        for (int i = 0; i < NACC; ++i)
                            tot[i] = j == 0 ? af[i] : __ldcg(p0 + (size_t)i * (CWARPS * 32) + ct);
                        for (int jj = 1; jj < pieces; ++jj) {
                            // pieces after the first start their CTA's share: slot 0
                            const double *pj = p.sk_partial + ((size_t)(c0 + jj) * 2) * PART;
#pragma unroll
                            for (int i = 0; i < NACC; ++i)
                                tot[i] = tot[i] + (jj == j ? af[i] : __ldcg(pj + (size_t)i * (CWARPS * 32) + ct));
                        }
#pragma unroll
                        for (int i = 0; i < NACC; ++i) af[i] = tot[i];
                        store_acc(acc, m0, n0, m_end, n_end, n_lo, p.beta_one, p.C, p.ldc, p.vec_store);
                    }
                }
            }
        } else if (p.ksplit > 1)
            store_acc(acc, m0, n0, m_end, n_end, n_lo, 0, p.partial + (size_t)slice * p.partial_stride, p.partial_ld, 1);
        else
            store_acc(acc, m0, n0, m_end, n_end, n_lo, PANELS ? 1 : p.beta_one, p.C, p.ldc, p.vec_store);
    }
}

// Split-K epilogue: C = (beta ? C : 0) + (slice 0 + slice 1 + ...), the slices summed in that
// fixed order, so the result does not depend on which CTA finished first.  Two columns per
// thread: the partial rows are 16-byte aligned (even ld, 256-byte aligned base; the pad column
// of an odd n is read and dropped).
__global__ void splitk_reduce(double *__restrict__ C, int ldc, int beta_one, const double *__restrict__ P, int ld,
                              size_t stride, int slices, int m, int n)
{
    const bool c_vec = ((ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    for (int row = blockIdx.x; row < m; row += gridDim.x) {
        const double *prow = P + (size_t)row * ld;
        double *crow = C + (size_t)row * ldc;
        for (int col = 2 * threadIdx.x; col < n; col += 2 * blockDim.x) {
            double2 v = *reinterpret_cast<const double2 *>(prow + col);
            int s = 1;
            for (; s + 3 < slices; s += 4) {  // four independent loads in flight, summed in order
                const double2 p1 = *reinterpret_cast<const double2 *>(prow + (size_t)s * stride + col);
                const double2 p2 = *reinterpret_cast<const double2 *>(prow + (size_t)(s + 1) * stride + col);
                const double2 p3 = *reinterpret_cast<const double2 *>(prow + (size_t)(s + 2) * stride + col);
                const double2 p4 = *reinterpret_cast<const double2 *>(prow + (size_t)(s + 3) * stride + col);
                v.x = (((v.x + p1.x) + p2.x) + p3.x) + p4.x;
                v.y = (((v.y + p1.y) + p2.y) + p3.y) + p4.y;
            }
            for (; s < slices; ++s) {
                const double2 p1 = *reinterpret_cast<const double2 *>(prow + (size_t)s * stride + col);
                v.x += p1.x;
                v.y += p1.y;
            }
            if (col + 1 < n) {
                if (c_vec) {
                    double2 *dst = reinterpret_cast<double2 *>(crow + col);
                    if (beta_one) {
                        const double2 o = *dst;
                        v.x = o.x + v.x;
                        v.y = o.y + v.y;
                    }
                    *dst = v;
                } else {
                    crow[col] = beta_one ? crow[col] + v.x : v.x;
                    crow[col + 1] = beta_one ? crow[col + 1] + v.y : v.y;
                }
            } else {
                crow[col] = beta_one ? crow[col] + v.x : v.x;
            }
        }
    }
}

// dst[r][c] = src[r][col0 + c] for c < live, 0 for live <= c < cols, r < rows (rows >= src_rows
// read as 0): an operand re-laid out with an even pitch and a 16-byte-aligned base for TMA.
__global__ void pack_kernel(const double *__restrict__ src, int src_rows, int ld_src, int col0, int live,
                            double *__restrict__ dst, int rows, int cols, int ld_dst)
{
    const size_t total = (size_t)rows * ld_dst;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / ld_dst), c = (int)(i % ld_dst);
        dst[i] = (r < src_rows && c < live && c < cols) ? src[(size_t)r * ld_src + col0 + c] : 0.0;
    }
}

}  // namespace fp64
}  // namespace mgx

using namespace mgx;

static int tiles_list_or(const int4 *tiles, int num_tiles, int m, int n, int bm)
{
    return tiles ? num_tiles : ((m + bm - 1) / bm) * ((n + fp64::BN - 1) / fp64::BN);
}

// Split-K geometry: K blocks per slice and the number of non-empty slices for `ksplit` asked.
static void splitk_geometry(int k_len, int ksplit, int *kb_split, int *slices)
{
    const int kblocks = (k_len + fp64::BK - 1) / fp64::BK;
    if (ksplit < 1) ksplit = 1;
    if (ksplit > kblocks) ksplit = kblocks > 0 ? kblocks : 1;
    *kb_split = (kblocks + ksplit - 1) / ksplit;
    *slices = *kb_split > 0 ? (kblocks + *kb_split - 1) / *kb_split : 1;
}

// Launches the split-K epilogue (also used by the Ozaki form's split-K).
int mgx_launch_splitk_reduce(double *C, int ldc, int beta_one, const double *P, int ld, size_t stride, int slices,
                             int m, int n, cudaStream_t stream)
{
    if (m <= 0 || n <= 0) return MGX_SUCCESS;
    int rgrid = mgx_sm_count() * 8;
    if (rgrid > m) rgrid = m;
    fp64::splitk_reduce<<<rgrid, 256, 0, stream>>>(C, ldc, beta_one, P, ld, stride, slices, m, n);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

size_t mgx_fp64_splitk_bytes(int m, int n, int k, int ksplit)
{
    int kbs, slices;
    splitk_geometry(k, ksplit, &kbs, &slices);
    if (slices <= 1 || m <= 0 || n <= 0) return 0;
    return (size_t)slices * (size_t)m * (size_t)((n + 1) & ~1) * sizeof(double) + 256;
}

static int launch_dgemm(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                        int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic,
                        const int4 *tiles, int num_tiles, int panel_kb, int ksplit, void *partial,
                        size_t partial_bytes, int bm = fp64::BM, int streamk = 0);

// Stream-K workspace: two partial accumulators (256 consumer threads x 32 doubles) per CTA of the
// grid, then one 8-byte ticket per 64 x 128 tile and consumer warp.
static size_t streamk_partial_bytes(int grid) { return (size_t)grid * 2 * fp64::CWARPS * 32 * 32 * sizeof(double); }
static int streamk_grid(int m, int n, int k)
{
    const long long units = (long long)((m + fp64::BM_SMALL - 1) / fp64::BM_SMALL) * ((n + fp64::BN - 1) / fp64::BN) *
                            ((k + fp64::BK - 1) / fp64::BK);
    const int sms = mgx_sm_count();
    return units < sms ? (int)units : sms;
}

size_t mgx_fp64_streamk_bytes(int m, int n, int k)
{
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    const size_t tiles = (size_t)((m + fp64::BM_SMALL - 1) / fp64::BM_SMALL) * ((n + fp64::BN - 1) / fp64::BN);
    return streamk_partial_bytes(streamk_grid(m, n, k)) +
           ((tiles * fp64::CWARPS * sizeof(unsigned long long) + 255) & ~size_t(255));
}

// Stream-K form over 64 x 128 tiles: every CTA takes an equal share of all tiles' K blocks.
int mgx_launch_dgemm_streamk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                             int ldc, int beta_one, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
    return launch_dgemm(A, B, C, m, n, k, 0, k, k, lda, ldb, ldc, beta_one, stream, 0, nullptr, 0, 0, 1, workspace,
                        workspace_bytes, fp64::BM_SMALL, 1);
}

// Launch C (+)= A[:, a_x0 : a_x0 + k_len] * B[0 : k_len, :] with the library's FP64 kernel.
// a_x_end: A columns at or beyond it read as zero; b_rows: rows of B that exist.
int mgx_launch_dgemm_ex(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                        int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic,
                        const int4 *tiles, int num_tiles, int panel_kb)
{
    return launch_dgemm(A, B, C, m, n, k_len, a_x0, a_x_end, b_rows, lda, ldb, ldc, beta_one, stream, force_generic,
                        tiles, num_tiles, panel_kb, 1, nullptr, 0);
}

// Split-K form of the above (regular tiling only): the K range is cut into `ksplit` slices whose
// products land in `partial` (mgx_fp64_splitk_bytes bytes, 256-byte aligned) and are summed
// into C in slice order by a second kernel.
int mgx_launch_dgemm_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                            int ldc, int beta_one, int ksplit, void *partial, size_t partial_bytes,
                            cudaStream_t stream, int tile_m)
{
    return launch_dgemm(A, B, C, m, n, k, 0, k, k, lda, ldb, ldc, beta_one, stream, 0, nullptr, 0, 0, ksplit,
                        partial, partial_bytes, tile_m == fp64::BM_SMALL ? fp64::BM_SMALL : fp64::BM);
}

static int launch_dgemm(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                        int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic,
                        const int4 *tiles, int num_tiles, int panel_kb, int ksplit, void *partial,
                        size_t partial_bytes, int bm, int streamk)
{
    // SUMMA work lists and panel accumulation are laid out for 128-row tiles
    if (tiles || panel_kb > 0) bm = fp64::BM;
    // stream-K runs the 64-row tile over a regular tiling only
    if (streamk && (tiles || panel_kb > 0 || ksplit > 1 || bm != fp64::BM_SMALL)) {
        mgx_set_last_message("FP64 stream-K: 64-row tiles over a regular tiling only");
        return MGX_E_INVALID;
    }
    if (m <= 0 || n <= 0) return MGX_SUCCESS;
    if (k_len <= 0) {
        if (beta_one) return MGX_SUCCESS;
        // C = A*B with an empty reduction is zero
        MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)n * sizeof(double), m, stream));
        return MGX_SUCCESS;
    }
    fp64::Params p;
    p.A = A;
    p.B = B;
    p.C = C;
    p.m = m;
    p.n = n;
    p.k_len = k_len;
    p.a_x0 = a_x0;
    p.a_x_end = a_x_end;
    p.b_rows = b_rows;
    p.lda = lda;
    p.ldb = ldb;
    p.ldc = ldc;
    p.beta_one = beta_one;
    p.vec_store = ((ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    p.status = mgx_device_status_ptr();
    p.tiles = tiles;
    p.num_tiles = num_tiles;
    p.panel_kb = panel_kb;
    p.streamk = 0;
    p.sk_tickets = nullptr;
    p.sk_partial = nullptr;
    int kb_split = 0, slices = 1;
    splitk_geometry(k_len, (tiles || panel_kb > 0) ? 1 : ksplit, &kb_split, &slices);
    p.ksplit = slices;
    p.kb_split = kb_split;
    p.partial = nullptr;
    p.partial_ld = (n + 1) & ~1;
    p.partial_stride = (size_t)m * (size_t)p.partial_ld;
    if (slices > 1) {
        const size_t need = (size_t)slices * p.partial_stride * sizeof(double);
        if (!partial || partial_bytes < need || (reinterpret_cast<uintptr_t>(partial) & 255)) {
            mgx_set_last_message("FP64 split-K: workspace of %zu bytes (aligned to 256) needed, %zu given", need,
                                 partial_bytes);
            return MGX_E_WORKSPACE;
        }
        p.partial = reinterpret_cast<double *>(partial);
    }

    const bool a_ok = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 2 == 0) && (a_x0 % 2 == 0);
    const bool b_ok = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % 2 == 0);
    if (!force_generic && a_x_end > a_x0 && b_rows > 0 && (!a_ok || !b_ok)) {
        // Re-lay the operands TMA cannot describe into stream-ordered scratch with an even pitch,
        // then run the TMA kernel on the copies (an HBM-bound pass, small beside the product).
        const int lda2 = (k_len + 1) & ~1, ldb2 = (n + 1) & ~1;
        const size_t abytes = a_ok ? 0 : (size_t)m * lda2 * sizeof(double);
        const size_t bbytes = b_ok ? 0 : (size_t)k_len * ldb2 * sizeof(double);
        char *scratch = nullptr;
        {
            const int arc = mgx_scratch_alloc(reinterpret_cast<void **>(&scratch), abytes + bbytes + 256, stream);
            if (arc != MGX_SUCCESS) return arc;
        }
        double *A2 = a_ok ? nullptr : reinterpret_cast<double *>(scratch);
        double *B2 = b_ok ? nullptr : reinterpret_cast<double *>(scratch + ((abytes + 255) & ~size_t(255)));
        const int blocks = mgx_sm_count() * 8;
        if (A2) fp64::pack_kernel<<<blocks, 256, 0, stream>>>(A, m, lda, a_x0, a_x_end - a_x0, A2, m, k_len, lda2);
        if (B2) fp64::pack_kernel<<<blocks, 256, 0, stream>>>(B, b_rows, ldb, 0, n, B2, k_len, n, ldb2);
        int rc = MGX_SUCCESS;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            mgx_set_last_cuda_error(e, "operand packing", __FILE__, __LINE__);
            rc = MGX_E_CUDA;
        } else {
            rc = launch_dgemm(A2 ? A2 : A, B2 ? B2 : B, C, m, n, k_len, A2 ? 0 : a_x0, A2 ? k_len : a_x_end,
                              B2 ? k_len : b_rows, A2 ? lda2 : lda, B2 ? ldb2 : ldb, ldc, beta_one, stream, 0, tiles,
                              num_tiles, panel_kb, ksplit, partial, partial_bytes, bm, streamk);
        }
        cudaFreeAsync(scratch, stream);
        return rc;
    }
    const bool tma_ok = !force_generic && a_ok && b_ok && a_x_end > 0 && b_rows > 0;
    CUtensorMap tmA, tmB;
    memset(&tmA, 0, sizeof tmA);
    memset(&tmB, 0, sizeof tmB);
    bool use_tma = false;
    if (tma_ok) {
        const int ea = mgx_encode_tmap_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, (uint64_t)a_x_end, (uint64_t)m,
                                          (uint64_t)lda * 8, 16, (uint32_t)bm, CU_TENSOR_MAP_SWIZZLE_128B);
        const int eb = mgx_encode_tmap_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, B, (uint64_t)n, (uint64_t)b_rows,
                                          (uint64_t)ldb * 8, 16, fp64::BK, CU_TENSOR_MAP_SWIZZLE_128B);
        use_tma = (ea == MGX_SUCCESS && eb == MGX_SUCCESS);
    }
    const int total_items = tiles_list_or(tiles, num_tiles, m, n, bm) * slices;
    int grid = mgx_sm_count();
    if (grid > total_items) grid = total_items;
    if (streamk) {
        grid = streamk_grid(m, n, k_len);
        if (grid > 255) {  // arrivals per tile must fit a ticket's 8-bit count
            mgx_set_last_message("FP64 stream-K: grid of %d CTAs exceeds 255", grid);
            return MGX_E_UNSUPPORTED;
        }
        const size_t pbytes = streamk_partial_bytes(grid);
        const size_t ntickets = (size_t)total_items * fp64::CWARPS;
        const size_t tbytes = ntickets * sizeof(unsigned long long);
        if (!partial || partial_bytes < pbytes + tbytes || (reinterpret_cast<uintptr_t>(partial) & 255)) {
            mgx_set_last_message("FP64 stream-K: workspace of %zu bytes (aligned to 256) needed, %zu given",
                                 pbytes + tbytes, partial_bytes);
            return MGX_E_WORKSPACE;
        }
        p.streamk = 1;
        p.sk_partial = reinterpret_cast<double *>(partial);
        p.sk_tickets = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(partial) + pbytes);
        // a fresh tag per launch (56 bits, never 0: zeroed memory reads as no arrivals)
        static std::atomic<unsigned long long> epochs{0};
        p.sk_epoch = ((epochs.fetch_add(1, std::memory_order_relaxed) + 1) & ((1ull << 56) - 1));
    }
    auto launch = [&](auto kernel, int smem_bytes) -> int {
        cudaFuncAttributes fa;
        MGX_HOST_CHECK(cudaFuncGetAttributes(&fa, kernel));
        if (fa.numRegs != fp64::LAUNCH_REGS) {
            mgx_set_last_message("FP64 kernel compiled with %d registers/thread, expected %d for its register split",
                                 fa.numRegs, fp64::LAUNCH_REGS);
            return MGX_E_UNSUPPORTED;
        }
        MGX_HOST_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
        // programmatic dependent launch: the set-up above griddepcontrol.wait overlaps the end of
        // the previous kernel in the stream
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof cfg);
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(fp64::THREADS);
        cfg.dynamicSmemBytes = (size_t)smem_bytes;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        MGX_HOST_CHECK(cudaLaunchKernelEx(&cfg, kernel, tmA, tmB, p));
        return MGX_SUCCESS;
    };
    constexpr int S128 = fp64::Geo<fp64::BM>::SMEM_BYTES, S64 = fp64::Geo<fp64::BM_SMALL>::SMEM_BYTES;
    int rc;
    if (bm == fp64::BM_SMALL)
        rc = use_tma ? launch(fp64::dgemm_kernel<fp64::BM_SMALL, true, false>, S64)
                     : launch(fp64::dgemm_kernel<fp64::BM_SMALL, false, false>, S64);
    else if (use_tma)
        rc = panel_kb > 0 ? launch(fp64::dgemm_kernel<fp64::BM, true, true>, S128)
                          : launch(fp64::dgemm_kernel<fp64::BM, true, false>, S128);
    else
        rc = panel_kb > 0 ? launch(fp64::dgemm_kernel<fp64::BM, false, true>, S128)
                          : launch(fp64::dgemm_kernel<fp64::BM, false, false>, S128);
    if (rc != MGX_SUCCESS) return rc;
    MGX_HOST_CHECK(cudaGetLastError());
    if (slices > 1) {
        int rgrid = mgx_sm_count() * 8;
        if (rgrid > m) rgrid = m;
        fp64::splitk_reduce<<<rgrid, 256, 0, stream>>>(C, ldc, beta_one, p.partial, p.partial_ld, p.partial_stride,
                                                       slices, m, n);
        MGX_HOST_CHECK(cudaGetLastError());
    }
    return MGX_SUCCESS;
}

int mgx_launch_dgemm(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                     int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic)
{
    return mgx_launch_dgemm_ex(A, B, C, m, n, k_len, a_x0, a_x_end, b_rows, lda, ldb, ldc, beta_one, stream,
                               force_generic, nullptr, 0, 0);
}
