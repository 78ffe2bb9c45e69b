// peaks.cu -- FP64 throughput microbenchmarks: the roofline denominators for the native FP64
// GEMM are measured on the running GPU with these loops rather than taken from a datasheet.
#include <cstdio>

#include "mgx_common.cuh"

namespace mgx {
namespace peaks {

constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256) dfma_loop(double *out, int iters)
{
    double x[CHAINS];
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 1e-7 * (blockIdx.x + 1);
#pragma unroll
    for (int i = 0; i < CHAINS; ++i) x[i] = 1e-3 * (i + 1);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < CHAINS; ++i) x[i] = fma(x[i], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < CHAINS; ++i) s += x[i];
    if (s == 12345.678) out[0] = s;  // keeps the loop alive
}

template <int KIND>
__global__ void __launch_bounds__(256) dmma_loop(double *out, int iters)
{
    const int lane = threadIdx.x & 31;
    const double av = 1e-3 * (1 + (lane & 7)), bv = 1e-3 * (1 + (lane >> 3));
    double acc[CHAINS][4];
#pragma unroll
    for (int i = 0; i < CHAINS; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[i][v] = 0.0;
    double a8[8], b4[4];
#pragma unroll
    for (int v = 0; v < 8; ++v) a8[v] = av * (v + 1);
#pragma unroll
    for (int v = 0; v < 4; ++v) b4[v] = bv * (v + 1);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < CHAINS; ++i) {
            if (KIND == 1) {
                double c2[2] = {acc[i][0], acc[i][1]};
                dmma_8x8x4(c2, a8[0], b4[0]);
                acc[i][0] = c2[0];
                acc[i][1] = c2[1];
            } else if (KIND == 2) {
                dmma_16x8x4(acc[i], a8[0], a8[1], b4[0]);
            } else if (KIND == 3) {
                const double a[4] = {a8[0], a8[1], a8[2], a8[3]};
                const double b[2] = {b4[0], b4[1]};
                dmma_16x8x8(acc[i], a, b);
            } else {
                dmma_16x8x16(acc[i], a8, b4);
            }
        }
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < CHAINS; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) s += acc[i][v];
    if (s == 12345.678) out[0] = s;
}

}  // namespace peaks
}  // namespace mgx

using namespace mgx;

extern "C" MGX_API int mgx_peak_fp64(int kind, int iterations, double *tflops_out)
{
    if (kind < 0 || kind > 4 || iterations <= 0 || !tflops_out) {
        mgx_set_last_message("mgx_peak_fp64: invalid arguments");
        return MGX_E_INVALID;
    }
    double *d_out = nullptr;
    MGX_HOST_CHECK(cudaMalloc(&d_out, sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = mgx_sm_count() * 4, threads = 256;
    double flops_per_iter_thread;  // FLOPs per thread per loop iteration
    auto launch = [&](int it) {
        switch (kind) {
        case 0: peaks::dfma_loop<<<blocks, threads>>>(d_out, it); break;
        case 1: peaks::dmma_loop<1><<<blocks, threads>>>(d_out, it); break;
        case 2: peaks::dmma_loop<2><<<blocks, threads>>>(d_out, it); break;
        case 3: peaks::dmma_loop<3><<<blocks, threads>>>(d_out, it); break;
        default: peaks::dmma_loop<4><<<blocks, threads>>>(d_out, it); break;
        }
    };
    switch (kind) {
    case 0: flops_per_iter_thread = 2.0 * peaks::CHAINS; break;
    case 1: flops_per_iter_thread = peaks::CHAINS * 2.0 * 8 * 8 * 4 / 32; break;
    case 2: flops_per_iter_thread = peaks::CHAINS * 2.0 * 16 * 8 * 4 / 32; break;
    case 3: flops_per_iter_thread = peaks::CHAINS * 2.0 * 16 * 8 * 8 / 32; break;
    default: flops_per_iter_thread = peaks::CHAINS * 2.0 * 16 * 8 * 16 / 32; break;
    }
    launch(iterations / 10 + 1);  // warm-up
    cudaEventRecord(e0);
    launch(iterations);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    if (err != cudaSuccess) {
        mgx_set_last_cuda_error(err, "peak loop", __FILE__, __LINE__);
        return MGX_E_CUDA;
    }
    *tflops_out = flops_per_iter_thread * (double)iterations * blocks * threads / (ms * 1e-3) / 1e12;
    return MGX_SUCCESS;
}

// ------------------------------------------------------------------------------------------
// INT8 tensor-core throughput of one tcgen05.mma.cta_group::1.kind::i8 shape (M = 128, K = 32,
// N = 64 / 128 / 256), operands resident in shared memory, accumulators alternating between two
// TMEM regions.  One CTA per SM, one issuing thread; every wait is bounded.
namespace mgx {
namespace peaks {

__device__ __forceinline__ uint64_t i8_desc(uint32_t smem_addr)
{
    uint64_t d = (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(256 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)6 << 61;
    return d;
}

template <int N>
__global__ void __launch_bounds__(128, 1) i8_mma_loop(int iters, int *status)
{
    __shared__ __align__(1024) uint8_t sA[128 * 32];
    __shared__ __align__(1024) uint8_t sB[N * 32];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    for (int i = threadIdx.x; i < 128 * 32; i += blockDim.x) sA[i] = (uint8_t)((i * 7) & 0x3f);
    for (int i = threadIdx.x; i < N * 32; i += blockDim.x) sB[i] = (uint8_t)((i * 13) & 0x3f);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tslot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        const uint64_t ad = i8_desc(smem_u32(sA)), bd = i8_desc(smem_u32(sB));
        const uint32_t stride = (N <= 256 / 2) ? 256 : N;  // two accumulators within 512 columns
        for (int it = 0; it < iters; ++it) {
            const uint32_t acc = (uint32_t)(it & 1);
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tbase + acc * stride),
                "l"(ad), "l"(bd), "r"(idesc), "r"((uint32_t)(it > 1))
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&bar))
                     : "memory");
        mbar_wait_bounded(&bar, 0, status, kDevTimeoutAcc);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(512) : "memory");
}

}  // namespace peaks
}  // namespace mgx

namespace mgx {
namespace peaks {

// Same MMA (M = N = 128, K = 32) cycling over 8 distinct A and 8 distinct B tiles in the pair
// pattern of the Ozaki kernel's high-weight set (t + u in 6..9), optionally while a second warp
// streams 64 KiB per round from global memory into another part of shared memory (the traffic
// a producer adds).  Measures what operand variety and concurrent copies cost the tensor core.
template <bool COPY>
__global__ void __launch_bounds__(128, 1) i8_mma_mix(int iters, const uint8_t *gsrc, int *status)
{
    extern __shared__ __align__(1024) uint8_t dsm[];
    uint8_t *tiles = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
    uint8_t *sink = tiles + 16 * 4096;
    __shared__ __align__(8) uint64_t bar, cbar;
    __shared__ uint32_t tslot;
    for (int i = threadIdx.x; i < 16 * 4096; i += blockDim.x) tiles[i] = (uint8_t)((i * 7) & 0x3f);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init(&cbar, 1);
        fence_barrier_init();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tslot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | (16u << 17) | (8u << 24);
        const uint32_t base = smem_u32(tiles);
        int n = 0;
        for (int it = 0; it < iters; ++it) {
            for (int t = 1; t <= 8; ++t)
                for (int u = (6 - t > 1 ? 6 - t : 1); u <= 8 && t + u <= 9; ++u) {
                    const uint32_t slot = 9 - (t + u);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tbase + slot * 128),
                        "l"(i8_desc(base + (t - 1) * 4096)), "l"(i8_desc(base + (7 + u) * 4096)), "r"(idesc),
                        "r"((uint32_t)(n >= 4))
                        : "memory");
                    ++n;
                }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&bar))
                     : "memory");
        mbar_wait_bounded(&bar, 0, status, kDevTimeoutAcc);
    } else if (COPY && threadIdx.x == 32) {
        // about as many bytes per round as the kernel's producer moves per 26 MMAs
        uint32_t ph = 0;
        for (int it = 0; it < iters; ++it) {
            mbar_arrive_expect_tx(&cbar, 65536);
            for (int j = 0; j < 2; ++j) bulk_load(sink + j * 32768, gsrc + (size_t)((it + j) & 63) * 32768, 32768, &cbar);
            if (!mbar_wait_bounded(&cbar, ph, status, kDevTimeoutFull)) break;
            ph ^= 1u;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(512) : "memory");
}

}  // namespace peaks
}  // namespace mgx

// kind 0: N = 64, 1: N = 128, 2: N = 256 (one A, one B tile); 3: N = 128 over 8 x 8 tiles in
// the Ozaki pair pattern; 4: as 3 with a concurrent 64 KiB/round bulk-copy stream into shared
// memory.  Writes INT8 TOP/s (2 M N K per MMA).
extern "C" MGX_API int mgx_peak_int8(int kind, int iterations, double *tops_out)
{
    if (kind < 0 || kind > 4 || iterations <= 0 || !tops_out) {
        mgx_set_last_message("mgx_peak_int8: invalid arguments");
        return MGX_E_INVALID;
    }
    const int n = kind <= 2 ? 64 << kind : 128;
    int *status = mgx_device_status_ptr();
    const int blocks = mgx_sm_count();
    const int mix_smem = 32 * 4096 + 1024;
    uint8_t *gsrc = nullptr;
    if (kind >= 3) {
        MGX_HOST_CHECK(cudaMalloc(&gsrc, 64 * 32768 + 32768));
        MGX_HOST_CHECK(cudaMemset(gsrc, 1, 64 * 32768 + 32768));
        MGX_HOST_CHECK(cudaFuncSetAttribute(peaks::i8_mma_mix<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mix_smem));
        MGX_HOST_CHECK(cudaFuncSetAttribute(peaks::i8_mma_mix<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mix_smem));
    }
    // mix kernels do 26 MMAs per iteration
    const int mix_iters = iterations / 26 > 0 ? iterations / 26 : 1;
    auto launch = [&](int it) {
        if (kind == 0) peaks::i8_mma_loop<64><<<blocks, 128>>>(it, status);
        else if (kind == 1) peaks::i8_mma_loop<128><<<blocks, 128>>>(it, status);
        else if (kind == 2) peaks::i8_mma_loop<256><<<blocks, 128>>>(it, status);
        else if (kind == 3) peaks::i8_mma_mix<false><<<blocks, 128, mix_smem>>>(it == iterations ? mix_iters : 2, gsrc, status);
        else peaks::i8_mma_mix<true><<<blocks, 128, mix_smem>>>(it == iterations ? mix_iters : 2, gsrc, status);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch(iterations / 10 + 2);
    cudaEventRecord(e0);
    launch(iterations);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (gsrc) cudaFree(gsrc);
    if (err != cudaSuccess) {
        mgx_set_last_cuda_error(err, "int8 peak loop", __FILE__, __LINE__);
        return MGX_E_CUDA;
    }
    const double mmas = kind <= 2 ? (double)iterations : 26.0 * mix_iters;
    *tops_out = 2.0 * 128.0 * n * 32.0 * mmas * blocks / (ms * 1e-3) / 1e12;
    return MGX_SUCCESS;
}
