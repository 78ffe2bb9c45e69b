// mgx_common.cuh -- shared device helpers for the sm_100a kernels of libmgxgemm.
//
// Every wait on an mbarrier is bounded by wall time (the %globaltimer register): a wait that
// runs out records an error code in the library's device status word and returns false, so a
// kernel that loses a producer or consumer ends instead of hanging the GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mgxgemm.h"

#define MGX_HOST_CHECK(call)                                         \
    do {                                                             \
        cudaError_t mgx_e_ = (call);                                 \
        if (mgx_e_ != cudaSuccess) {                                 \
            mgx_set_last_cuda_error(mgx_e_, #call, __FILE__, __LINE__); \
            return MGX_E_CUDA;                                       \
        }                                                            \
    } while (0)

// Host-side bookkeeping shared by the translation units (defined in capi.cu).
void mgx_set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);
void mgx_set_last_message(const char *fmt, ...);
int *mgx_device_status_ptr();  // device address of this device's status word (no allocation)
// The library's file-scope device arrays whose addresses host code looks up.
enum MgxSymbolSlot : int { kMgxSymStatus = 0, kMgxSymOzSync = 1, kMgxSymOzakiNoalloc = 2, kMgxSymbolSlots = 3 };
void *mgx_symbol_address(const void *symbol, int slot, cudaError_t *err = nullptr);
int mgx_sm_count();
// Stream-ordered scratch from the library's pool on the current device (free with cudaFreeAsync).
int mgx_scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream);
int mgx_encode_tmap_2d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base,
                       uint64_t inner, uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                       uint32_t box_outer, CUtensorMapSwizzle swizzle);
int mgx_encode_tmap_3d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base,
                       uint64_t d0, uint64_t d1, uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes,
                       uint32_t b0, uint32_t b1, uint32_t b2, CUtensorMapSwizzle swizzle);

namespace mgx {

// Device status codes (first error wins).
enum DeviceStatus : int {
    kDevOk = 0,
    kDevTimeoutFull = 1,     // consumer waited too long for a filled stage
    kDevTimeoutEmpty = 2,    // producer waited too long for a free stage
    kDevTimeoutAcc = 3,      // accumulator hand-off wait ran out
    kDevNonFinite = 4,       // non-finite input where the form cannot represent it
    kDevBadLaunch = 5,       // launch geometry does not match the kernel's assumptions
    kDevTicket = 6,          // a stream-K ticket could not be taken
};

constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void record_status(int *status, int code)
{
    if (status) atomicCAS(status, 0, code);
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar` for at most `limit_ns`.  Returns false (and records `code`)
// when the wait ran out; the caller then abandons its loop.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, uint32_t parity, int *status, int code,
                                              unsigned long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    uint32_t spins = 0;
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((++spins & 255u) == 0u) {
            if (global_ns() - t0 > limit_ns) {
                record_status(status, code);
                return false;
            }
        }
    }
}

// Bounded wait with the library's limit (kWaitLimitNs).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status, int code)
{
    return mbar_wait_for(bar, parity, status, code, kWaitLimitNs);
}

// Bounded wait for waits expected to be long (a warp idling through a whole phase of another
// role's work): polls with a growing nanosleep so the waiting warp leaves the issue slots to
// the warps doing the work.
__device__ __forceinline__ bool mbar_wait_sleepy(uint64_t *bar, uint32_t parity, int *status, int code)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    unsigned ns = 64;
    while (true) {
        __nanosleep(ns);
        if (mbar_try_wait(bar, parity)) return true;
        if (ns < 2048) ns <<= 1;
        if (global_ns() - t0 > kWaitLimitNs) {
            record_status(status, code);
            return false;
        }
    }
}

// ---------------------------------------------------------------- TMA (no multicast anywhere)
__device__ __forceinline__ void tma_load_2d(void *smem_dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *smem_dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Plain bulk copy global -> shared (16-byte aligned, size a multiple of 16), completing on `bar`.
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Asks L2 to fetch [gsrc, gsrc + bytes) ahead of use (no completion signal).
__device__ __forceinline__ void bulk_prefetch_l2(const void *gsrc, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gsrc), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------- FP64 tensor-core MMA (DMMA)
// D(16x8) += A(16x4) * B(4x8); fragment ownership for lane = 4*g + t:
//   a0 = A[g][t], a1 = A[g+8][t];  b0 = B[t][g];  c = {(g,2t), (g,2t+1), (g+8,2t), (g+8,2t+1)}
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// D(16x8) += A(16x8) * B(8x8): a = {(g,t), (g+8,t), (g,t+4), (g+8,t+4)}, b = {(t,g), (t+4,g)}
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// D(16x8) += A(16x16) * B(16x8): a[v0 + 2 v1] = (g + 8 v0, t + 4 v1), b[v] = (t + 4 v, g)
__device__ __forceinline__ void dmma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// D(8x8) += A(8x4) * B(4x8): a0 = A[g][t], b0 = B[t][g], c = {(g,2t), (g,2t+1)}
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a0, double b0)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a0), "d"(b0));
}

__device__ __forceinline__ double lds_f64(uint32_t addr)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
    return v;
}

}  // namespace mgx
