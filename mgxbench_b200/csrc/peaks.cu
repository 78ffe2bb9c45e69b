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
