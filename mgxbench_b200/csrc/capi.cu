// capi.cu -- extern "C" entry points of libmgxgemm (declared in include/mgxgemm.h) and the host
// bookkeeping shared by the kernels' translation units.
#include <cudaTypedefs.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "mgx_common.cuh"

// ------------------------------------------------------------------------------- host state
namespace {
thread_local char g_msg[512] = "";
constexpr int kMaxDevices = 64;
std::mutex g_mu;
int g_sm_count[kMaxDevices];
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
}  // namespace

// One status word per device; kernels record the first device-side error here.
__device__ int mgx_status_word;

void mgx_set_last_message(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
}

void mgx_set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line)
{
    mgx_set_last_message("%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
}

static int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    return dev;
}

// Id of the context current on this thread (cuCtxGetId), 0 when there is none yet or the driver
// lacks the call.  A context that cudaDeviceReset ended and the runtime later re-created gets a
// new id, so an address cached under the old id is known to be stale.
static unsigned long long current_context_id()
{
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 4000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(fn);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of one of this library's __device__ arrays on the current device.  Host code
// only knows the array's name, a host-side stand-in; the address a kernel needs is taken with
// cudaGetSymbolAddress in the device's context.  It is cached per device together with the
// context's id and taken again when the context has changed (after a cudaDeviceReset).  A failed
// lookup returns nullptr with CUDA's last-error state cleared, so the next launch check does not
// report it as its own failure; *err (if given) receives the lookup's error.
void *mgx_symbol_address(const void *symbol, int slot, cudaError_t *err)
{
    struct Entry {
        unsigned long long ctx;
        void *ptr;
    };
    static Entry cache[kMgxSymbolSlots][kMaxDevices];
    if (err) *err = cudaSuccess;
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices || slot < 0 || slot >= kMgxSymbolSlots) {
        cudaGetLastError();
        if (err) *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    Entry &e = cache[slot][dev];
    unsigned long long ctx = current_context_id();
    if (e.ptr && ctx != 0 && ctx == e.ctx) return e.ptr;
    void *p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, symbol);
    if (rc != cudaSuccess || !p) {
        cudaGetLastError();
        if (err) *err = rc != cudaSuccess ? rc : cudaErrorInvalidSymbol;
        e.ptr = nullptr;
        return nullptr;
    }
    // The lookup itself creates the primary context when none was current yet.
    if (ctx == 0) ctx = current_context_id();
    e.ctx = ctx;
    e.ptr = p;
    return p;
}

int *mgx_device_status_ptr()
{
    return static_cast<int *>(mgx_symbol_address(reinterpret_cast<const void *>(&mgx_status_word), kMgxSymStatus));
}

int mgx_sm_count()
{
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices) return 148;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_sm_count[dev]) {
        int c = 0;
        if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
        g_sm_count[dev] = c;
    }
    return g_sm_count[dev];
}

// The library's own stream-ordered memory pool on each device, for short-lived scratch (operand
// packing, the host-buffer pipeline, validation accumulators).  It keeps up to 32 GiB across
// synchronisations, so repeated calls reuse their scratch instead of mapping fresh memory each
// time (a process's default pool returns everything at every synchronisation), and it leaves
// the process's default pool settings alone.  mgx_scratch_trim() hands the cached memory back.
static cudaMemPool_t g_pool[kMaxDevices];

int mgx_scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream)
{
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices) return MGX_E_CUDA;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_pool[dev]) {
            cudaMemPoolProps props;
            memset(&props, 0, sizeof props);
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t pool = nullptr;
            cudaError_t e = cudaMemPoolCreate(&pool, &props);
            if (e != cudaSuccess) {
                mgx_set_last_cuda_error(e, "cudaMemPoolCreate", __FILE__, __LINE__);
                return MGX_E_CUDA;
            }
            uint64_t keep = 32ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pool[dev] = pool;
        }
    }
    const cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, g_pool[dev], stream);
    if (e != cudaSuccess) {
        mgx_set_last_cuda_error(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
        return MGX_E_CUDA;
    }
    return MGX_SUCCESS;
}

MGX_API int mgx_scratch_trim(void)
{
    const int dev = current_device();
    if (dev < 0 || dev >= kMaxDevices) return MGX_E_CUDA;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        pool = g_pool[dev];
    }
    if (!pool) return MGX_SUCCESS;
    MGX_HOST_CHECK(cudaDeviceSynchronize());
    MGX_HOST_CHECK(cudaMemPoolTrimTo(pool, 0));
    return MGX_SUCCESS;
}

static int get_encoder()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_encode) return MGX_SUCCESS;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
        mgx_set_last_message("cuTensorMapEncodeTiled unavailable (%s)", cudaGetErrorString(e));
        return MGX_E_UNSUPPORTED;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return MGX_SUCCESS;
}

int mgx_encode_tmap_2d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base, uint64_t inner,
                       uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer,
                       CUtensorMapSwizzle swizzle)
{
    (void)elem_bytes;
    const int rc = get_encoder();
    if (rc != MGX_SUCCESS) return rc;
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, dtype, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        mgx_set_last_message("cuTensorMapEncodeTiled(2d) failed with %d", (int)r);
        return MGX_E_CUDA;
    }
    return MGX_SUCCESS;
}

int mgx_encode_tmap_3d(CUtensorMap *map, CUtensorMapDataType dtype, int elem_bytes, const void *base, uint64_t d0,
                       uint64_t d1, uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t b0,
                       uint32_t b1, uint32_t b2, CUtensorMapSwizzle swizzle)
{
    (void)elem_bytes;
    const int rc = get_encoder();
    if (rc != MGX_SUCCESS) return rc;
    cuuint64_t dims[3] = {d0, d1, d2};
    cuuint64_t strides[2] = {stride1_bytes, stride2_bytes};
    cuuint32_t box[3] = {b0, b1, b2};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = g_encode(map, dtype, 3, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        mgx_set_last_message("cuTensorMapEncodeTiled(3d) failed with %d", (int)r);
        return MGX_E_CUDA;
    }
    return MGX_SUCCESS;
}

// Defined in the kernels' translation units.
size_t mgx_fp64_splitk_bytes(int m, int n, int k, int ksplit);
size_t mgx_fp64_streamk_bytes(int m, int n, int k);
int mgx_launch_dgemm_streamk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                             int ldc, int beta_one, void *workspace, size_t workspace_bytes, cudaStream_t stream);
int mgx_launch_dgemm_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                            int ldc, int beta_one, int ksplit, void *partial, size_t partial_bytes,
                            cudaStream_t stream, int tile_m = 128);

int mgx_launch_dgemm(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                     int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic);
int mgx_validate_impl(const double *d_c, size_t count, double expected, double abs_tol, double rel_tol,
                      mgx_validation_t *out, cudaStream_t stream);

static bool dims_ok(int m, int n, int k, int lda, int ldb, int ldc)
{
    if (m < 0 || n < 0 || k < 0) return false;
    if (lda < (k > 0 ? k : 1) && m > 0 && k > 0) return false;
    if (ldb < (n > 0 ? n : 1) && k > 0 && n > 0) return false;
    if (ldc < (n > 0 ? n : 1) && m > 0 && n > 0) return false;
    return true;
}

extern "C" {

MGX_API const char *mgx_last_error_message(void) { return g_msg; }

MGX_API const char *mgx_status_string(int status)
{
    switch (status) {
    case MGX_SUCCESS: return "success";
    case MGX_E_INVALID: return "invalid argument";
    case MGX_E_CUDA: return "CUDA error";
    case MGX_E_NONFINITE: return "non-finite input";
    case MGX_E_TIMEOUT: return "device-side wait timed out";
    case MGX_E_WORKSPACE: return "workspace missing or too small";
    case MGX_E_UNSUPPORTED: return "unsupported configuration";
    case MGX_E_DEVICE: return "device-side error";
    default: return "unknown status";
    }
}

namespace mgx {
// One thread waits on an mbarrier that nothing ever completes: its bounded wait runs out after
// limit_ns and records the timeout in the status word, and the kernel returns normally.
__global__ void wait_probe_kernel(int *status, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait_for(&bar, 0, status, kDevTimeoutFull, limit_ns);
}
}  // namespace mgx

MGX_API int mgx_wait_probe(int limit_us)
{
    if (limit_us < 1 || limit_us > 2000000) {
        mgx_set_last_message("mgx_wait_probe: limit %d us outside 1 .. 2000000", limit_us);
        return MGX_E_INVALID;
    }
    int *status = mgx_device_status_ptr();
    if (!status) {
        mgx_set_last_message("no device status word (no CUDA device?)");
        return MGX_E_CUDA;
    }
    mgx::wait_probe_kernel<<<1, 32>>>(status, (unsigned long long)limit_us * 1000ull);
    MGX_HOST_CHECK(cudaGetLastError());
    MGX_HOST_CHECK(cudaDeviceSynchronize());
    return MGX_SUCCESS;
}

MGX_API int mgx_device_status(int *code_out)
{
    int *p = mgx_device_status_ptr();
    if (!p) {
        mgx_set_last_message("no device status word (no CUDA device?)");
        return MGX_E_CUDA;
    }
    MGX_HOST_CHECK(cudaDeviceSynchronize());
    int code = 0;
    MGX_HOST_CHECK(cudaMemcpy(&code, p, sizeof(int), cudaMemcpyDeviceToHost));
    if (code != 0) {
        const int zero = 0;
        MGX_HOST_CHECK(cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice));
    }
    if (code_out) *code_out = code;
    return MGX_SUCCESS;
}

MGX_API int mgx_gemm_fp64(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                          int ldc, int beta_one, void *stream)
{
    if (!dims_ok(m, n, k, lda, ldb, ldc) || (m > 0 && n > 0 && (!C || (k > 0 && (!A || !B))))) {
        mgx_set_last_message("mgx_gemm_fp64: invalid arguments m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k, lda,
                             ldb, ldc);
        return MGX_E_INVALID;
    }
    return mgx_launch_dgemm(A, B, C, m, n, k, 0, k, k, lda, ldb, ldc, beta_one ? 1 : 0, (cudaStream_t)stream, 0);
}

MGX_API size_t mgx_fp64_splitk_workspace_size(int m, int n, int k, int ksplit)
{
    if (m < 0 || n < 0 || k < 0) return 0;
    return mgx_fp64_splitk_bytes(m, n, k, ksplit);
}

MGX_API int mgx_gemm_fp64_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                 int ldb, int ldc, int beta_one, int ksplit, void *workspace,
                                 size_t workspace_bytes, void *stream)
{
    if (!dims_ok(m, n, k, lda, ldb, ldc) || ksplit < 1 || (m > 0 && n > 0 && (!C || (k > 0 && (!A || !B))))) {
        mgx_set_last_message("mgx_gemm_fp64_splitk: invalid arguments m=%d n=%d k=%d lda=%d ldb=%d ldc=%d ksplit=%d",
                             m, n, k, lda, ldb, ldc, ksplit);
        return MGX_E_INVALID;
    }
    return mgx_launch_dgemm_splitk(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, ksplit, workspace,
                                   workspace_bytes, (cudaStream_t)stream);
}

MGX_API size_t mgx_fp64_streamk_workspace_size(int m, int n, int k)
{
    if (m < 0 || n < 0 || k < 0) return 0;
    return mgx_fp64_streamk_bytes(m, n, k);
}

MGX_API int mgx_gemm_fp64_streamk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                                  int ldc, int beta_one, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!dims_ok(m, n, k, lda, ldb, ldc) || (m > 0 && n > 0 && (!C || (k > 0 && (!A || !B))))) {
        mgx_set_last_message("mgx_gemm_fp64_streamk: invalid arguments m=%d n=%d k=%d lda=%d ldb=%d ldc=%d", m, n, k,
                             lda, ldb, ldc);
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0 || k == 0)
        return mgx_launch_dgemm(A, B, C, m, n, k, 0, k, k, lda, ldb, ldc, beta_one ? 1 : 0, (cudaStream_t)stream, 0);
    return mgx_launch_dgemm_streamk(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, workspace, workspace_bytes,
                                    (cudaStream_t)stream);
}

MGX_API int mgx_gemm_fp64_tiled(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                                int ldc, int beta_one, int tile_m, int ksplit, void *workspace,
                                size_t workspace_bytes, void *stream)
{
    if (!dims_ok(m, n, k, lda, ldb, ldc) || ksplit < 1 || (tile_m != 64 && tile_m != 128) ||
        (m > 0 && n > 0 && (!C || (k > 0 && (!A || !B))))) {
        mgx_set_last_message("mgx_gemm_fp64_tiled: invalid arguments m=%d n=%d k=%d lda=%d ldb=%d ldc=%d tile_m=%d "
                             "(64 or 128) ksplit=%d",
                             m, n, k, lda, ldb, ldc, tile_m, ksplit);
        return MGX_E_INVALID;
    }
    return mgx_launch_dgemm_splitk(A, B, C, m, n, k, lda, ldb, ldc, beta_one ? 1 : 0, ksplit, workspace,
                                   workspace_bytes, (cudaStream_t)stream, tile_m);
}

MGX_API int mgx_ab_multiply(double *a, double *b, double *c, int m, int n, int k, int lda, int ldb, int ldc, int w)
{
    if (w <= 0) {
        mgx_set_last_message("mgx_ab_multiply: tile width w=%d must be positive", w);
        return MGX_E_INVALID;
    }
    return mgx_gemm_fp64(a, b, c, m, n, k, lda, ldb, ldc, 0, nullptr);
}

MGX_API int mgx_ab_multiply_accumulate_async(const double *a, const double *b_chunk, double *c, int m, int n,
                                             int k_total, int k_offset, int k_chunk, int lda, int ldb, int ldc,
                                             int w, void *stream)
{
    if (w <= 0 || m < 0 || n < 0 || k_chunk < 0 || k_offset < 0 || k_total < 0 ||
        (m > 0 && n > 0 && k_chunk > 0 && (!a || !b_chunk || !c || lda < 1 || ldb < n || ldc < n))) {
        mgx_set_last_message("mgx_ab_multiply_accumulate_async: invalid arguments");
        return MGX_E_INVALID;
    }
    if (m == 0 || n == 0 || k_chunk == 0) return MGX_SUCCESS;
    int a_x_end = k_offset + k_chunk;
    if (a_x_end > k_total) a_x_end = k_total;
    if (a_x_end <= k_offset) {
        // Every A column of the chunk is outside k_total: the reference multiplies zeros.
        // Route it through the generic kernel so 0 * B keeps the reference's NaN behaviour.
        return mgx_launch_dgemm(a, b_chunk, c, m, n, k_chunk, k_offset, k_offset, k_chunk, lda, ldb, ldc, 1,
                                (cudaStream_t)stream, 1);
    }
    return mgx_launch_dgemm(a, b_chunk, c, m, n, k_chunk, k_offset, a_x_end, k_chunk, lda, ldb, ldc, 1,
                            (cudaStream_t)stream, 0);
}

MGX_API int mgx_validate_matrix_c(const double *d_c, int rows, int cols, double expected, double abs_tol,
                                  double rel_tol, int rank, int print, mgx_validation_t *out)
{
    if (rows < 0 || cols < 0 || (rows > 0 && cols > 0 && !d_c)) {
        mgx_set_last_message("mgx_validate_matrix_c: invalid arguments");
        return MGX_E_INVALID;
    }
    mgx_validation_t v;
    const size_t count = (size_t)rows * (size_t)cols;
    const int rc = mgx_validate_impl(d_c, count, expected, abs_tol, rel_tol, &v, nullptr);
    if (rc != MGX_SUCCESS) return rc;
    if (out) *out = v;
    if (rank == 0 && print) {
        // Same block and formats as validate_matrix_C (1D-row-block/mulmat_kernel.cu:298-319).
        printf("\n");
        printf("============================================================\n");
        printf("NUMERICAL VALIDATION\n");
        printf("============================================================\n");
        printf("Matrix dimensions  : %d x %d\n", rows, cols);
        printf("Expected C[i,j]    : %.12f\n", expected);
        printf("Elements checked   : %llu\n", (unsigned long long)count);
        printf("Invalid elements   : %llu\n", (unsigned long long)v.invalid);
        printf("Max absolute error : %.6e\n", v.max_abs_error);
        printf("Max relative error : %.6e\n", v.max_rel_error);
        printf("Absolute tolerance : %.6e\n", abs_tol);
        printf("Relative tolerance : %.6e\n", rel_tol);
        printf("Result             : %s\n", v.invalid == 0 ? "PASS" : "FAIL");
        printf("============================================================\n");
        fflush(stdout);
    }
    return v.invalid == 0 ? 1 : 0;
}

}  // extern "C"
