/*
 * mgxgemm.h -- C ABI of libmgxgemm, the B200 (sm_100a) per-rank FP64 block-multiply path of
 * MGXBench.
 *
 * MGXBench's GPU work is three host functions in mulmat_kernel.cu, declared by its drivers at
 * 1D-row-block/mmb.cu:162-164 and 2D-block-matrix/mmb.cu:20-22:
 *     void ABMultiply(double*, double*, double*, int m, int n, int k, int lda, int ldb, int ldc, int w);
 *     void ABMultiplyAccumulateAsync(const double*, const double*, double*, int m, int n, int k_total,
 *                                    int k_offset, int k_chunk, int lda, int ldb, int ldc, int w,
 *                                    cudaStream_t);
 *     int  validate_matrix_C(const double*, int rows, int cols, double expected, double abs_tol,
 *                            double rel_tol, int rank);
 * The mgx_ab_* / mgx_validate_* entry points below replace them one for one, with the same
 * argument meaning (row-major matrices, leading dimensions in elements, device pointers owned
 * by the caller).  Where the reference aborts or ignores errors, these return a status code.
 *
 * Conventions
 *   - Every pointer argument named a, b, c, A, B, C is a device pointer.
 *   - Matrices are row-major: element (i, j) of X is X[i * ldx + j].
 *   - Functions taking a `stream` (a cudaStream_t passed as void*, NULL = legacy default stream)
 *     are stream-ordered and return after launching.  The others synchronise.
 *   - Return value: MGX_SUCCESS (0) or a negative mgx_status_t; mgx_last_error_message() says more.
 *   - No function exits or aborts the process.
 *   - Thread safety: calls on different host threads are safe; device work that overlaps on the
 *     GPU shares nothing unless a comment says otherwise.
 */
#ifndef MGXGEMM_H
#define MGXGEMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MGX_API __attribute__((visibility("default")))
#else
#define MGX_API
#endif

/* Arithmetic forms of the product. */
typedef enum { MGX_FORM_FP64 = 0, MGX_FORM_OZAKI = 1, MGX_FORM_CRT = 2 } mgx_form_t;

typedef enum {
    MGX_SUCCESS = 0,
    MGX_E_INVALID = -1,      /* an argument is out of range (sizes, leading dimensions, null pointer) */
    MGX_E_CUDA = -2,         /* a CUDA runtime or driver call failed */
    MGX_E_NONFINITE = -3,    /* the Ozaki form met a NaN or infinity in A or B */
    MGX_E_TIMEOUT = -4,      /* a bounded device-side wait ran out (kernel abandoned its work) */
    MGX_E_WORKSPACE = -5,    /* workspace pointer null or smaller than required */
    MGX_E_UNSUPPORTED = -6,  /* no kernel for this device / configuration */
    MGX_E_DEVICE = -7        /* the kernel reported another device-side error */
} mgx_status_t;

/* Result of a constant-value validation (validate_C_kernel semantics). */
typedef struct {
    uint64_t elements;       /* rows * cols */
    uint64_t invalid;        /* elements with abs err > abs_tol AND rel err > rel_tol, or non-finite */
    double max_abs_error;
    double max_rel_error;
} mgx_validation_t;

/* Error of a computed C against a double-double reference product of the same A and B. */
typedef struct {
    double normwise;         /* ||C - AB||_F / ||AB||_F */
    double max_rel;          /* max |C - AB| / |AB| over elements with |AB| >= floor_rel * max|AB| */
    double max_componentwise;/* max |C - AB| / (|A||B|) */
    double max_abs;          /* max |C - AB| */
    uint64_t rows_checked;
} mgx_error_t;

/* ------------------------------------------------------------------------------------------
 * Drop-in replacements for MGXBench's launchers
 * ------------------------------------------------------------------------------------------ */

/* Replaces ABMultiply (1D-row-block/mulmat_kernel.cu:86-92; 2D-block-matrix/mulmat_kernel.cu:81-87):
 * C[m x n] = A[m x k] * B[k x n] on the legacy default stream, asynchronously.  `w` is the
 * reference's tile width (TILE_DIM = 32); it must be positive and does not change the result or
 * the tiling this library uses. */
MGX_API int mgx_ab_multiply(double *a, double *b, double *c, int m, int n, int k, int lda, int ldb, int ldc,
                            int w);

/* Replaces ABMultiplyAccumulateAsync (1D-row-block/mulmat_kernel.cu:148-158;
 * 2D-block-matrix/mulmat_kernel.cu:142-151):
 * C[m x n] += A[:, k_offset : k_offset + k_chunk] * B_chunk[k_chunk x n], the chunk's product
 * summed first and then added to C with one rounding, as the reference does.  Columns of A at
 * or beyond k_total read as zero. */
MGX_API int mgx_ab_multiply_accumulate_async(const double *a, const double *b_chunk, double *c, int m, int n,
                                             int k_total, int k_offset, int k_chunk, int lda, int ldb, int ldc,
                                             int w, void *stream);

/* Replaces validate_matrix_C (1D-row-block/mulmat_kernel.cu:228-326; 2D copy :221-304):
 * checks every element of the rows x cols device matrix against `expected`, prints the
 * reference's NUMERICAL VALIDATION block on stdout when rank == 0 and print != 0, fills *out
 * when out != NULL, and returns 1 (pass), 0 (fail) or a negative mgx_status_t.  Unlike the
 * reference it also counts NaN and infinite elements as invalid. Synchronous. */
MGX_API int mgx_validate_matrix_c(const double *d_c, int rows, int cols, double expected, double abs_tol,
                                  double rel_tol, int rank, int print, mgx_validation_t *out);

/* ------------------------------------------------------------------------------------------
 * Native FP64 GEMM (FP64 tensor-core MMA, TMA-fed warp-specialised pipeline)
 * ------------------------------------------------------------------------------------------ */

/* C = A B (beta_one == 0) or C += A B (beta_one != 0), A m x k, B k x n, all FP64. */
MGX_API int mgx_gemm_fp64(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                          int ldc, int beta_one, void *stream);

/* Split-K form for products with too few 128 x 128 output tiles to fill the GPU: the K range is
 * cut into `ksplit` slices (at most one per 32-wide K block) computed by separate CTAs, and the
 * slice products are summed into C in slice order (deterministic).  The rounding differs from
 * mgx_gemm_fp64 by the slice sums.  No counterpart in MGXBench; the autotuner picks ksplit.
 * `workspace` (256-byte aligned) holds mgx_fp64_splitk_workspace_size(m, n, k, ksplit) bytes;
 * 0 bytes means ksplit resolved to one slice and the call is mgx_gemm_fp64. */
MGX_API size_t mgx_fp64_splitk_workspace_size(int m, int n, int k, int ksplit);
MGX_API int mgx_gemm_fp64_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                 int ldb, int ldc, int beta_one, int ksplit, void *workspace,
                                 size_t workspace_bytes, void *stream);

/* mgx_gemm_fp64_splitk with a choice of output tile: tile_m = 128 (128 x 128 tiles, the default
 * of every other FP64 entry point) or 64 (64 x 128 tiles: twice the work items, for products with
 * few 128 x 128 tiles on the 148 SMs).  No counterpart in MGXBench; the autotuner's tile
 * candidates pick it.  Both tiles reduce every element over K in the same order, so the result
 * does not depend on tile_m.  ksplit and workspace as for mgx_gemm_fp64_splitk. */
MGX_API int mgx_gemm_fp64_tiled(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                                int ldc, int beta_one, int tile_m, int ksplit, void *workspace,
                                size_t workspace_bytes, void *stream);

/* Stream-K form of the FP64 product over 64 x 128 tiles, for products with too few tiles to fill
 * the GPU (no counterpart in MGXBench; the autotuner offers it).  Every CTA takes an equal
 * share of all tiles' 32-wide K blocks, so every SM has the same work; a tile whose K range is
 * split between CTAs is finished by the last of them to arrive, which adds the pieces in K order.
 * No CTA waits for another.  Deterministic for a given GPU (the shares depend on its SM count),
 * and within the same any-order bound as the other FP64 entry points.  `workspace` (256-byte
 * aligned) holds mgx_fp64_streamk_workspace_size(m, n, k) bytes on the current device; its
 * contents need no initialisation (the arrival tickets carry a per-launch tag). */
MGX_API size_t mgx_fp64_streamk_workspace_size(int m, int n, int k);
MGX_API int mgx_gemm_fp64_streamk(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                                  int ldc, int beta_one, void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------------------------------
 * Ozaki-scheme FP64 GEMM on the INT8 tensor cores (tcgen05, exact int32 TMEM accumulation)
 * ------------------------------------------------------------------------------------------ */

/* Bytes of device workspace mgx_gemm_ozaki needs for this shape and split count. */
MGX_API size_t mgx_ozaki_workspace_size(int m, int n, int k, int splits);

/* C = A B or C += A B computed as the exact integer products of `splits` signed 7-bit digit
 * slices per operand (per-row / per-column power-of-two scaling), recombined in FP64.
 * splits in [2, 12].  Returns MGX_E_NONFINITE if A or B holds NaN or infinity. */
MGX_API int mgx_gemm_ozaki(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb,
                           int ldc, int beta_one, int splits, void *workspace, size_t workspace_bytes,
                           void *stream);

/* Split-K form of mgx_gemm_ozaki for products with few 128 x 128 output tiles (small m n, long
 * k): the 32-wide K blocks are cut into `ksplit` slices computed by separate CTAs; each slice's
 * group sums are recombined and scaled on their own, and the slice results are added into C in
 * slice order (deterministic).  The exponents and digits are those of the whole K range, so only
 * the final additions differ from mgx_gemm_ozaki.  Needs k <= mgx_ozaki_kmax(splits) and
 * mgx_ozaki_splitk_workspace_size(m, n, k, splits, ksplit) bytes of 256-byte aligned workspace
 * (0 when k is too long).  No counterpart in MGXBench; the autotuner picks ksplit. */
MGX_API size_t mgx_ozaki_splitk_workspace_size(int m, int n, int k, int splits, int ksplit);
MGX_API int mgx_gemm_ozaki_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                  int ldb, int ldc, int beta_one, int splits, int ksplit, void *workspace,
                                  size_t workspace_bytes, void *stream);

/* The two phases of mgx_gemm_ozaki for one K range of at most mgx_ozaki_kmax(splits):
 * mgx_ozaki_split writes the exponents and digit slices of A and B into the workspace;
 * mgx_ozaki_multiply runs the INT8 tensor-core products and the FP64 recombination into C.
 * Calling split once and multiply several times reuses the slices. */
MGX_API int mgx_ozaki_split(const double *A, const double *B, int m, int n, int k, int lda, int ldb, int splits,
                            void *workspace, size_t workspace_bytes, void *stream);
MGX_API int mgx_ozaki_multiply(double *C, int m, int n, int k, int ldc, int beta_one, int splits,
                               const void *workspace, size_t workspace_bytes, void *stream);

/* Largest K one int32 accumulation of `splits`-digit slices can take (mgx_gemm_ozaki splits K
 * into chunks of this size and adds them in order). */
MGX_API int mgx_ozaki_kmax(int splits);

/* ------------------------------------------------------------------------------------------
 * CRT form (Ozaki scheme II): one INT8 tensor-core product per modulus
 * ------------------------------------------------------------------------------------------ */

/* Bytes of device workspace mgx_gemm_ozaki_crt needs for this shape and modulus count. */
MGX_API size_t mgx_crt_workspace_size(int m, int n, int k, int moduli);

/* C = A B or C += A B computed as `moduli` (8..16) INT8 products of residues: each row of A and
 * column of B is scaled by a power of two to integers whose norms leave every exact integer
 * product below a quarter of the moduli's product, the integers are reduced modulo pairwise-coprime
 * p_l <= 256, each residue product runs on the tensor cores (exact int32) and is reduced mod p_l,
 * and C is rebuilt in FP64 by the Chinese remainder theorem.  15 moduli reach FP64 accuracy at
 * K = 16384 with 15 products, where the slice form needs 36 for 8 slices.  Rows or columns
 * holding NaN or infinity give NaN results and set the device status (mgx_device_status).
 * No counterpart in MGXBench. */
MGX_API int mgx_gemm_ozaki_crt(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                               int ldb, int ldc, int beta_one, int moduli, void *workspace,
                               size_t workspace_bytes, void *stream);

/* The three phases of mgx_gemm_ozaki_crt for one K range of at most mgx_crt_kmax(), each
 * stream-ordered on the same workspace: mgx_crt_split writes the scales and residues of A and B;
 * mgx_crt_products runs the residue products on the tensor cores (one persistent launch);
 * mgx_crt_combine rebuilds C (+)= A B from the product residues.  Splitting once and
 * multiplying several times reuses the residues. */
MGX_API int mgx_crt_split(const double *A, const double *B, int m, int n, int k, int lda, int ldb, int moduli,
                          void *workspace, size_t workspace_bytes, void *stream);
MGX_API int mgx_crt_products(int m, int n, int k, int moduli, void *workspace, size_t workspace_bytes,
                             void *stream);
MGX_API int mgx_crt_combine(double *C, int m, int n, int k, int ldc, int beta_one, int moduli, void *workspace,
                            size_t workspace_bytes, void *stream);

/* Split-K form of mgx_gemm_ozaki_crt for products with few 256 x 256 output tiles (small m n,
 * long k): the 32-wide K blocks are cut into `ksplit` slices whose residue products run as
 * separate work items; the slices' residues are added modulo each p before the CRT rebuild, so
 * the result is bit-identical to mgx_gemm_ozaki_crt.  Needs k <= mgx_crt_kmax() and
 * mgx_crt_splitk_workspace_size(m, n, k, moduli, ksplit) bytes of 256-byte aligned workspace
 * (0 when k is too long).  No counterpart in MGXBench; the autotuner picks ksplit. */
MGX_API size_t mgx_crt_splitk_workspace_size(int m, int n, int k, int moduli, int ksplit);
MGX_API int mgx_gemm_ozaki_crt_splitk(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                      int ldb, int ldc, int beta_one, int moduli, int ksplit, void *workspace,
                                      size_t workspace_bytes, void *stream);

/* Smallest modulus count whose a-priori normwise error bound meets `target` for reduction
 * length k (8..16). */
MGX_API int mgx_crt_choose_moduli(int k, double target);

/* Largest K of one int32 residue accumulation (longer K is processed in chunks of this size). */
MGX_API int mgx_crt_kmax(void);

/* C = A B from HOST buffers (hA m x k, hB k x n, hC m x n, row-major, leading dimensions in
 * elements) with form MGX_FORM_FP64, MGX_FORM_OZAKI (`splits` slices) or MGX_FORM_CRT (`splits` =
 * moduli, 8..16).  A is cut into `panels` (1..64) row panels and B into `panels` column panels
 * (multiples of 128; 256 for the CRT form); the panels are copied in the order A_0, B_0,
 * A_1, B_1, ....  Once A_t and B_t are on the device, the blocks (i, j) with max(i, j) = t are
 * computed as two products (the row strip (t, 0..t) and the column strip (0..t-1, t)) and each
 * strip is copied back while the rest computes, so PCIe copies in both directions overlap the
 * product.  At N = 16384, 32 panels keep the last strips short (the end-to-end time is set by
 * the copies in plus the work the last panels unlock).
 * The result is bit-identical to the device-buffer entry points'.  Device memory (A, B, C and
 * the Ozaki workspace) is taken stream-ordered from the library's pool on the current device
 * and returned before the call's work completes.  Page-locked host memory gives full
 * copy/compute overlap.  Stream-ordered; the Ozaki form needs k <= mgx_ozaki_kmax(splits). */
MGX_API int mgx_gemm_host(const double *hA, const double *hB, double *hC, int m, int n, int k, int lda, int ldb,
                          int ldc, int form, int splits, int panels, void *stream);

/* Size of the fixed workspace of mgx_gemm_ozaki_noalloc (32 MiB). */
#define MGX_OZAKI_NOALLOC_BYTES (32u << 20)

/* mgx_gemm_ozaki for callers that cannot allocate device memory at call time (inside a stream
 * capture that must not gain allocation nodes, under an allocator that owns the device memory,
 * after a no-allocation start-up phase).  No counterpart in MGXBench.  It allocates nothing: its
 * workspace is a fixed device array of MGX_OZAKI_NOALLOC_BYTES that every GPU loading the library
 * holds until exit, so it takes only products whose mgx_ozaki_workspace_size fits (for example
 * m = n = k = 1024 with 8 splits) and returns MGX_E_WORKSPACE otherwise.  The first call on a
 * device looks up the array's device address and should come before any stream capture; the
 * address is looked up again only when the device's context has changed (after a
 * cudaDeviceReset), and that call too should come before any capture.  All calls share the
 * array, and the products' lockstep counters with mgx_gemm_ozaki: calls whose work overlaps on
 * the GPU race on the array.  Stream-ordered. */
MGX_API int mgx_gemm_ozaki_noalloc(const double *A, const double *B, double *C, int m, int n, int k, int lda,
                                   int ldb, int ldc, int beta_one, int splits, void *stream);

/* Split count the library picks to reach a normwise relative error <= target for inputs whose
 * per-row / per-column dynamic range is `exp_range` binades (a-priori model; 3..9). */
MGX_API int mgx_ozaki_choose_splits(int k, double exp_range, double target);

/* ------------------------------------------------------------------------------------------
 * 2D SUMMA over a process grid, all blocks and panels on this GPU
 *
 * Replaces the panel loop of 2D-block-matrix/mmb.cu:239-361 for every rank of a grid_rows x
 * grid_cols process grid at once: block (i, j) owns rows [row_cuts[i], row_cuts[i+1]) and
 * columns [col_cuts[j], col_cuts[j+1]) of C, and C = 0 followed by C_ij += A_i[:, k0:k0+kc]
 * B_j[k0:k0+kc, :] for every panel of width panel_k.  The plan runs all (block, tile, panel)
 * work in ONE persistent kernel launch (plus the split kernels of the Ozaki form), so a run can
 * be captured in a CUDA graph.  Blocks need not be equal (uneven splits, remainders).  With the
 * CRT form (MGX_FORM_CRT) a run is one CRT product of the whole C; its results do not depend on
 * the block cuts or the panel width.
 * ------------------------------------------------------------------------------------------ */

typedef struct {
    int m, n, k;               /* C is m x n, the reduction is k */
    int grid_rows, grid_cols;  /* Pr x Pc process grid (2D-block-matrix/mmb.cu:45-58) */
    const int *row_cuts;       /* grid_rows + 1 ascending row boundaries; NULL = split evenly, the
                                  first (m mod Pr) blocks one row taller */
    const int *col_cuts;       /* likewise for columns */
    int panel_k;               /* panel width BK (MGXBENCH_SUMMA_BK, 2D-block-matrix/mmb.cu:107) */
    int form;                  /* mgx_form_t */
    int splits;                /* slices of the Ozaki form (2..12), moduli of the CRT form (8..16) */
} mgx_summa_desc_t;

typedef struct mgx_summa_plan mgx_summa_plan_t;

/* The FP64 plan's work list, computed on the host: returns the number of work tiles and writes up
 * to `capacity` of them to out as {m0, n_lo, m_end, n_end} (columns [n_lo, n_end) of rows
 * [m0, m_end)).  Needs no device. */
MGX_API int mgx_summa_tiles(const mgx_summa_desc_t *desc, int *out, int capacity);

/* Builds the work list on the current device and allocates the Ozaki workspace if needed. */
MGX_API int mgx_summa_plan_create(const mgx_summa_desc_t *desc, mgx_summa_plan_t **plan);

/* C = SUMMA product of A (m x k, lda) and B (k x n, ldb); stream-ordered, allocates nothing. */
MGX_API int mgx_summa_run(mgx_summa_plan_t *plan, const double *A, int lda, const double *B, int ldb, double *C,
                          int ldc, void *stream);

/* Work tiles, K steps and workspace bytes of a plan.  FP64 form: the persistent kernel's 128 x 128
 * tiles clipped to their blocks, and the panels it accumulates in order.  The Ozaki and CRT forms
 * use no panel list: their integer sums are exact and their scales belong to whole rows and
 * columns, so neither the block cuts nor the panel order change a bit of C, and the plan runs one
 * product of all of C.  For them work_tiles is that product's work items (128 x 128 tiles for the
 * slice form; moduli x 256 x 256 tiles for the CRT form) and panels the number of K chunks of
 * one exact int32 accumulation (1 unless k > mgx_ozaki_kmax / mgx_crt_kmax). */
MGX_API int mgx_summa_plan_info(const mgx_summa_plan_t *plan, int *work_tiles, int *panels, size_t *workspace_bytes);

MGX_API int mgx_summa_plan_destroy(mgx_summa_plan_t *plan);

/* ------------------------------------------------------------------------------------------
 * Accuracy checking on the GPU (double-double reference product)
 * ------------------------------------------------------------------------------------------ */

/* Error of C (m x n) against A B computed in double-double, over `row_count` rows starting at
 * `row_start` (all rows when row_count <= 0).  Synchronous. */
MGX_API int mgx_error_vs_dd(const double *A, const double *B, const double *C, int m, int n, int k, int lda,
                            int ldb, int ldc, int row_start, int row_count, double floor_rel, mgx_error_t *out);

/* ------------------------------------------------------------------------------------------
 * Synthetic inputs
 * ------------------------------------------------------------------------------------------ */

/* Fills rows x cols of X (leading dimension ld) on the device: kind 0 = the constant `value`
 * (MGXBench's A = 1, B = 2 initialisation, 1D-row-block/mmb.cu:586-591), 1 = uniform [-1, 1),
 * 2 = u * 2^e with u uniform [-1, 1) and e a uniform integer in [-e_range, e_range].  Element
 * (r, c) depends only on (seed, r * cols + c).  Stream-ordered. */
MGX_API int mgx_fill_matrix(double *X, int rows, int cols, int ld, int kind, double value, int e_range,
                            uint64_t seed, void *stream);

/* ------------------------------------------------------------------------------------------
 * Learned cost model of the autotuner: a 3-layer FP32 MLP (6 -> 64 -> 64 -> 2, tanh) trained
 * and evaluated on the GPU.  Inputs per sample (standardised by the caller): log2 M, log2 N,
 * log2 K, input exponent range, tile shape id, split count.  Outputs: standardised log
 * runtime and log10 normwise error.  No counterpart in MGXBench: it replaces the regression of
 * autotuning/predictive.py:100-165.  All pointers are device pointers; stream-ordered.
 * ------------------------------------------------------------------------------------------ */

/* Number of floats in the parameter vector (W1 | b1 | W2 | b2 | W3 | b3). */
MGX_API int mgx_mlp_param_count(void);
/* Glorot-uniform weights from `seed`, zero biases. */
MGX_API int mgx_mlp_init(float *params, uint64_t seed, void *stream);
/* out[batch x 2] = MLP(X[batch x 6]). */
MGX_API int mgx_mlp_forward(const float *X, int batch, const float *params, float *out, void *stream);
/* grads = d loss / d params and *loss = sum_o w_o (out_o - Y_o)^2 / batch over the batch. */
MGX_API int mgx_mlp_gradients(const float *X, const float *Y, const float *out_weights, int batch,
                              const float *params, float *grads, float *loss, void *stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8); `step` counts from 1. */
MGX_API int mgx_mlp_adam_step(float *params, const float *grads, float *m, float *v, int step, float lr,
                              void *stream);

/* ------------------------------------------------------------------------------------------
 * Library state
 * ------------------------------------------------------------------------------------------ */

/* Returns the device memory the library keeps cached for its scratch (operand packing, the
 * host-buffer pipeline) on the current device: it synchronises the device, then releases the
 * cache.  Later calls allocate again.  No counterpart in MGXBench. */
MGX_API int mgx_scratch_trim(void);

/* Exercises the timeout path of the library's bounded device-side waits: a kernel waits on a
 * barrier that nothing completes, gives up after `limit_us` microseconds (1 .. 2e6), records
 * the timeout in the device status word (read it with mgx_device_status) and returns; the
 * context stays usable.  Synchronises the device.  No counterpart in MGXBench. */
MGX_API int mgx_wait_probe(int limit_us);

/* Reads and clears the current device's status word written by bounded device-side waits
 * (0 = none).  Synchronises the device. */
MGX_API int mgx_device_status(int *code_out);

MGX_API const char *mgx_last_error_message(void);
MGX_API const char *mgx_status_string(int status);

/* Measured peaks of this GPU's FP64 paths: kind 0 = DFMA on the FP64 units, 1 = DMMA m8n8k4,
 * 2 = DMMA m16n8k4, 3 = DMMA m16n8k8, 4 = DMMA m16n8k16.  Synchronous; writes TFLOP/s. */
MGX_API int mgx_peak_fp64(int kind, int iterations, double *tflops_out);

/* Measured INT8 tensor-core rate of tcgen05.mma.cta_group::1.kind::i8 with M = 128, K = 32 and
 * N = 64 (kind 0), 128 (kind 1) or 256 (kind 2), operands resident in shared memory.
 * Synchronous; writes TOP/s. */
MGX_API int mgx_peak_int8(int kind, int iterations, double *tops_out);

#ifdef __cplusplus
}
#endif
#endif /* MGXGEMM_H */
