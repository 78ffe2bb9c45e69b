// mlp.cu -- the autotuner's learned cost model: a 3-layer FP32 MLP (6 -> 64 -> 64 -> 2, tanh),
// trained and run on the GPU by these kernels.
//
// Inputs (standardised by the caller): log2 M, log2 N, log2 K, input exponent range, tile shape
// id, split count.  Outputs: predicted (standardised) log runtime and log10 normwise error.
// Loss: sum_o w_o (out_o - y_o)^2 / batch.  Optimiser: Adam.
//
// Parameter vector layout (floats):
//   W1[64][6] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2]     (4738 values)
#include <cmath>

#include "mgx_common.cuh"

namespace mgx {
namespace mlp {

constexpr int NI = 6, NH = 64, NO = 2;
constexpr int OW1 = 0, OB1 = OW1 + NH * NI, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NO * NH, NPARAM = OB3 + NO;
constexpr int SPB = 16;        // samples per block in the gradient kernel (static smem < 48 KB)
constexpr int THREADS = 256;

__device__ __forceinline__ void forward_sample(const float *P, const float *x, float *h1, float *h2, float *out)
{
    for (int j = 0; j < NH; ++j) {
        float a = P[OB1 + j];
        for (int i = 0; i < NI; ++i) a = fmaf(P[OW1 + j * NI + i], x[i], a);
        h1[j] = tanhf(a);
    }
    for (int j = 0; j < NH; ++j) {
        float a = P[OB2 + j];
        for (int k = 0; k < NH; ++k) a = fmaf(P[OW2 + j * NH + k], h1[k], a);
        h2[j] = tanhf(a);
    }
    for (int o = 0; o < NO; ++o) {
        float a = P[OB3 + o];
        for (int k = 0; k < NH; ++k) a = fmaf(P[OW3 + o * NH + k], h2[k], a);
        out[o] = a;
    }
}

// Inference: one thread per sample, parameters staged in shared memory.
__global__ void __launch_bounds__(THREADS) forward_kernel(const float *__restrict__ X, int batch,
                                                          const float *__restrict__ params, float *__restrict__ out)
{
    __shared__ float P[NPARAM];
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= batch) return;
    float x[NI], h1[NH], h2[NH], o[NO];
    for (int i = 0; i < NI; ++i) x[i] = X[s * NI + i];
    forward_sample(P, x, h1, h2, o);
    for (int k = 0; k < NO; ++k) out[s * NO + k] = o[k];
}

// Gradients of the loss over `batch` samples; each block handles SPB samples and adds its share
// into grads (which the caller zeroes) and loss.
__global__ void __launch_bounds__(THREADS) grad_kernel(const float *__restrict__ X, const float *__restrict__ Y,
                                                       const float *__restrict__ wout, int batch,
                                                       const float *__restrict__ params, float *__restrict__ grads,
                                                       float *__restrict__ loss)
{
    __shared__ float P[NPARAM];
    __shared__ float xs[SPB][NI], h1[SPB][NH], h2[SPB][NH], d2[SPB][NH], d1[SPB][NH], dout[SPB][NO];
    __shared__ float lsum[THREADS / 32];
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) P[i] = params[i];
    const int s0 = blockIdx.x * SPB;
    const int ns = min(SPB, batch - s0);
    for (int i = threadIdx.x; i < SPB * NI; i += blockDim.x) {
        const int s = i / NI;
        xs[s][i % NI] = (s < ns) ? X[(s0 + s) * NI + i % NI] : 0.f;
    }
    __syncthreads();
    // layer 1
    for (int i = threadIdx.x; i < SPB * NH; i += blockDim.x) {
        const int s = i / NH, j = i % NH;
        float a = P[OB1 + j];
        for (int q = 0; q < NI; ++q) a = fmaf(P[OW1 + j * NI + q], xs[s][q], a);
        h1[s][j] = tanhf(a);
    }
    __syncthreads();
    // layer 2
    for (int i = threadIdx.x; i < SPB * NH; i += blockDim.x) {
        const int s = i / NH, j = i % NH;
        float a = P[OB2 + j];
        for (int k = 0; k < NH; ++k) a = fmaf(P[OW2 + j * NH + k], h1[s][k], a);
        h2[s][j] = tanhf(a);
    }
    __syncthreads();
    // output, loss and its gradient
    float lpart = 0.f;
    for (int i = threadIdx.x; i < SPB * NO; i += blockDim.x) {
        const int s = i / NO, o = i % NO;
        float g = 0.f;
        if (s < ns) {
            float a = P[OB3 + o];
            for (int k = 0; k < NH; ++k) a = fmaf(P[OW3 + o * NH + k], h2[s][k], a);
            const float diff = a - Y[(s0 + s) * NO + o];
            lpart += wout[o] * diff * diff / batch;
            g = 2.f * wout[o] * diff / batch;
        }
        dout[s][o] = g;
    }
    for (int o = 16; o > 0; o >>= 1) lpart += __shfl_xor_sync(0xffffffffu, lpart, o);
    if ((threadIdx.x & 31) == 0) lsum[threadIdx.x >> 5] = lpart;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < THREADS / 32; ++w) t += lsum[w];
        atomicAdd(loss, t);
    }
    // dW3, db3
    for (int i = threadIdx.x; i < NO * NH + NO; i += blockDim.x) {
        float g = 0.f;
        if (i < NO * NH) {
            const int o = i / NH, k = i % NH;
            for (int s = 0; s < SPB; ++s) g = fmaf(dout[s][o], h2[s][k], g);
            atomicAdd(&grads[OW3 + i], g);
        } else {
            const int o = i - NO * NH;
            for (int s = 0; s < SPB; ++s) g += dout[s][o];
            atomicAdd(&grads[OB3 + o], g);
        }
    }
    // dH2 = (dout W3) * (1 - h2^2)
    for (int i = threadIdx.x; i < SPB * NH; i += blockDim.x) {
        const int s = i / NH, k = i % NH;
        float a = 0.f;
        for (int o = 0; o < NO; ++o) a = fmaf(dout[s][o], P[OW3 + o * NH + k], a);
        d2[s][k] = a * (1.f - h2[s][k] * h2[s][k]);
    }
    __syncthreads();
    // dW2, db2
    for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) {
        const int j = i / NH, k = i % NH;
        float g = 0.f;
        for (int s = 0; s < SPB; ++s) g = fmaf(d2[s][j], h1[s][k], g);
        atomicAdd(&grads[OW2 + i], g);
    }
    for (int j = threadIdx.x; j < NH; j += blockDim.x) {
        float g = 0.f;
        for (int s = 0; s < SPB; ++s) g += d2[s][j];
        atomicAdd(&grads[OB2 + j], g);
    }
    // dH1 = (dH2 W2) * (1 - h1^2)
    for (int i = threadIdx.x; i < SPB * NH; i += blockDim.x) {
        const int s = i / NH, k = i % NH;
        float a = 0.f;
        for (int j = 0; j < NH; ++j) a = fmaf(d2[s][j], P[OW2 + j * NH + k], a);
        d1[s][k] = a * (1.f - h1[s][k] * h1[s][k]);
    }
    __syncthreads();
    // dW1, db1
    for (int i = threadIdx.x; i < NH * NI + NH; i += blockDim.x) {
        float g = 0.f;
        if (i < NH * NI) {
            const int j = i / NI, q = i % NI;
            for (int s = 0; s < SPB; ++s) g = fmaf(d1[s][j], xs[s][q], g);
            atomicAdd(&grads[OW1 + i], g);
        } else {
            const int j = i - NH * NI;
            for (int s = 0; s < SPB; ++s) g += d1[s][j];
            atomicAdd(&grads[OB1 + j], g);
        }
    }
}

__global__ void adam_kernel(float *__restrict__ params, const float *__restrict__ grads, float *__restrict__ m,
                            float *__restrict__ v, int step, float lr, float beta1, float beta2, float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    const float g = grads[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float mhat = mi / (1.f - powf(beta1, (float)step));
    const float vhat = vi / (1.f - powf(beta2, (float)step));
    params[i] -= lr * mhat / (sqrtf(vhat) + eps);
}

// Glorot-uniform weights from a counter-based hash, zero biases.
__global__ void init_kernel(float *__restrict__ params, unsigned long long seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const float u = 2.f * ((float)(z >> 40) * (1.f / 16777216.f)) - 1.f;
    float limit = 0.f;
    if (i < OB1) limit = sqrtf(6.f / (NI + NH));
    else if (i >= OW2 && i < OB2) limit = sqrtf(6.f / (NH + NH));
    else if (i >= OW3 && i < OB3) limit = sqrtf(6.f / (NH + NO));
    params[i] = u * limit;
}

}  // namespace mlp
}  // namespace mgx

using namespace mgx;

extern "C" {

MGX_API int mgx_mlp_param_count(void) { return mlp::NPARAM; }

MGX_API int mgx_mlp_init(float *params, uint64_t seed, void *stream)
{
    if (!params) return MGX_E_INVALID;
    mlp::init_kernel<<<(mlp::NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, seed);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

MGX_API int mgx_mlp_forward(const float *X, int batch, const float *params, float *out, void *stream)
{
    if (batch < 0 || (batch > 0 && (!X || !params || !out))) return MGX_E_INVALID;
    if (batch == 0) return MGX_SUCCESS;
    mlp::forward_kernel<<<(batch + mlp::THREADS - 1) / mlp::THREADS, mlp::THREADS, 0, (cudaStream_t)stream>>>(
        X, batch, params, out);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

MGX_API int mgx_mlp_gradients(const float *X, const float *Y, const float *out_weights, int batch,
                              const float *params, float *grads, float *loss, void *stream)
{
    if (batch <= 0 || !X || !Y || !out_weights || !params || !grads || !loss) return MGX_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    MGX_HOST_CHECK(cudaMemsetAsync(grads, 0, sizeof(float) * mlp::NPARAM, s));
    MGX_HOST_CHECK(cudaMemsetAsync(loss, 0, sizeof(float), s));
    mlp::grad_kernel<<<(batch + mlp::SPB - 1) / mlp::SPB, mlp::THREADS, 0, s>>>(X, Y, out_weights, batch, params,
                                                                                grads, loss);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

MGX_API int mgx_mlp_adam_step(float *params, const float *grads, float *m, float *v, int step, float lr,
                              void *stream)
{
    if (!params || !grads || !m || !v || step < 1 || !(lr > 0.f)) return MGX_E_INVALID;
    mlp::adam_kernel<<<(mlp::NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, step, lr,
                                                                                  0.9f, 0.999f, 1e-8f);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}

}  // extern "C"
