// fill.cu -- seeded synthetic matrices generated on the device (counter-based, so any element
// can be regenerated on the host from (seed, row, col) alone).
#include "mgx_common.cuh"

namespace mgx {
namespace fill {

// splitmix64 finaliser of (seed, linear index): a stateless per-element random stream.
__host__ __device__ __forceinline__ uint64_t mix(uint64_t seed, uint64_t idx)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (idx + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void fill_kernel(double *X, int rows, int cols, int ld, int kind, double value, int e_range,
                            uint64_t seed)
{
    const size_t total = (size_t)rows * cols;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / cols, c = i % cols;
        double v = value;
        if (kind != 0) {
            const uint64_t h = mix(seed, i);
            v = 2.0 * ((double)(h >> 11) * 0x1.0p-53) - 1.0;  // uniform [-1, 1), exact
            if (kind == 2 && e_range > 0) {
                const uint64_t h2 = mix(seed ^ 0x5851F42D4C957F2Dull, i);
                const int e = (int)(h2 % (uint64_t)(2 * e_range + 1)) - e_range;
                v = ldexp(v, e);
            }
        }
        X[r * ld + c] = v;
    }
}

}  // namespace fill
}  // namespace mgx

using namespace mgx;

extern "C" MGX_API int mgx_fill_matrix(double *X, int rows, int cols, int ld, int kind, double value, int e_range,
                                       uint64_t seed, void *stream)
{
    if (rows < 0 || cols < 0 || ld < cols || kind < 0 || kind > 2 || e_range < 0 || e_range > 500 ||
        (rows > 0 && cols > 0 && !X)) {
        mgx_set_last_message("mgx_fill_matrix: invalid arguments");
        return MGX_E_INVALID;
    }
    if (rows == 0 || cols == 0) return MGX_SUCCESS;
    const int blocks = mgx_sm_count() * 8;
    fill::fill_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(X, rows, cols, ld, kind, value, e_range, seed);
    MGX_HOST_CHECK(cudaGetLastError());
    return MGX_SUCCESS;
}
