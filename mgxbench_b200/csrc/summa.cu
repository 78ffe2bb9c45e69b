// summa.cu -- 2D SUMMA over an uneven process grid, every rank's blocks on this GPU.
//
// The reference runs one process per block (2D-block-matrix/mmb.cu:94-109) and, for every panel
// k0 of width BK, broadcasts A_i[:, k0:k0+kc] along its process row and B_j[k0:k0+kc, :] along
// its process column before C_ij += A_panel B_panel (mmb.cu:239-361).  Here A and B are resident,
// so a plan turns the grid into a list of 128 x 128 work tiles clipped to their blocks, and one
// persistent kernel walks (tile, panel) in order: the FP64 form adds each panel's product into
// C_ij with one rounding, as the reference does.  The Ozaki form accumulates the panels exactly
// in int32 and recombines once; because its element values do not depend on how the output is
// tiled, it covers every block with one uniform 128 x 128 raster of the whole C.  The CRT form
// likewise: its scales belong to whole rows of A and columns of B and its residue sums are exact,
// so all blocks run as one CRT product of the whole C.
#include <cstring>
#include <vector>

#include "mgx_common.cuh"

int mgx_launch_dgemm_ex(const double *A, const double *B, double *C, int m, int n, int k_len, int a_x0, int a_x_end,
                        int b_rows, int lda, int ldb, int ldc, int beta_one, cudaStream_t stream, int force_generic,
                        const int4 *tiles, int num_tiles, int panel_kb);
int mgx_ozaki_run(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb, int ldc,
                  int beta_one, int splits, void *workspace, size_t workspace_bytes, cudaStream_t stream);
int mgx_crt_run(const double *A, const double *B, double *C, int m, int n, int k, int lda, int ldb, int ldc,
                int beta_one, int moduli, void *workspace, size_t workspace_bytes, cudaStream_t stream);

struct mgx_summa_plan {
    mgx_summa_desc_t desc;
    std::vector<int> rcut, ccut;
    int4 *d_tiles = nullptr;
    int num_tiles = 0;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    int device = 0;
};

static std::vector<int> even_cuts(int extent, int parts)
{
    std::vector<int> c(parts + 1, 0);
    const int base = extent / parts, rem = extent % parts;
    for (int i = 0; i < parts; ++i) c[i + 1] = c[i] + base + (i < rem ? 1 : 0);
    return c;
}

static bool cuts_ok(const std::vector<int> &c, int extent)
{
    if (c.front() != 0 || c.back() != extent) return false;
    for (size_t i = 1; i < c.size(); ++i)
        if (c[i] <= c[i - 1]) return false;
    return true;
}

// Work tiles, block by block in rank order: {m0, n_lo, m_end, n_end}.  Rows start at the block's
// first row.  Column tiles start at the block's first column rounded down to even (the kernel's
// B boxes need an even column); n_lo keeps the block's exact first column so the kernel never
// stores into the neighbouring block.
static std::vector<int4> summa_tiles(const std::vector<int> &rcut, const std::vector<int> &ccut)
{
    std::vector<int4> tiles;
    for (size_t bi = 0; bi + 1 < rcut.size(); ++bi)
        for (size_t bj = 0; bj + 1 < ccut.size(); ++bj) {
            const int c_lo = ccut[bj], c_hi = ccut[bj + 1], base = c_lo & ~1;
            for (int r = rcut[bi]; r < rcut[bi + 1]; r += 128)
                for (int c = base; c < c_hi; c += 128)
                    tiles.push_back(make_int4(r, c < c_lo ? c_lo : c, rcut[bi + 1] < r + 128 ? rcut[bi + 1] : r + 128,
                                              c_hi < c + 128 ? c_hi : c + 128));
        }
    return tiles;
}

extern "C" {

MGX_API int mgx_summa_tiles(const mgx_summa_desc_t *desc, int *out, int capacity)
{
    if (!desc || desc->m <= 0 || desc->n <= 0 || desc->grid_rows <= 0 || desc->grid_cols <= 0 ||
        desc->grid_rows > desc->m || desc->grid_cols > desc->n) {
        mgx_set_last_message("mgx_summa_tiles: invalid descriptor");
        return MGX_E_INVALID;
    }
    const std::vector<int> rc = desc->row_cuts ? std::vector<int>(desc->row_cuts, desc->row_cuts + desc->grid_rows + 1)
                                               : even_cuts(desc->m, desc->grid_rows);
    const std::vector<int> cc = desc->col_cuts ? std::vector<int>(desc->col_cuts, desc->col_cuts + desc->grid_cols + 1)
                                               : even_cuts(desc->n, desc->grid_cols);
    if (!cuts_ok(rc, desc->m) || !cuts_ok(cc, desc->n)) {
        mgx_set_last_message("mgx_summa_tiles: block cuts must rise strictly from 0 to the extent");
        return MGX_E_INVALID;
    }
    const std::vector<int4> t = summa_tiles(rc, cc);
    if (out)
        for (int i = 0; i < (int)t.size() && i < capacity; ++i) {
            out[4 * i] = t[i].x;
            out[4 * i + 1] = t[i].y;
            out[4 * i + 2] = t[i].z;
            out[4 * i + 3] = t[i].w;
        }
    return (int)t.size();
}

MGX_API int mgx_summa_plan_create(const mgx_summa_desc_t *desc, mgx_summa_plan_t **plan)
{
    if (!desc || !plan || desc->m <= 0 || desc->n <= 0 || desc->k <= 0 || desc->grid_rows <= 0 ||
        desc->grid_cols <= 0 || desc->grid_rows > desc->m || desc->grid_cols > desc->n || desc->panel_k <= 0 ||
        (desc->form != MGX_FORM_FP64 && desc->form != MGX_FORM_OZAKI && desc->form != MGX_FORM_CRT) ||
        (desc->form == MGX_FORM_OZAKI && (desc->splits < 2 || desc->splits > 12)) ||
        (desc->form == MGX_FORM_CRT && (desc->splits < 8 || desc->splits > 16))) {
        mgx_set_last_message("mgx_summa_plan_create: invalid descriptor");
        return MGX_E_INVALID;
    }
    mgx_summa_plan *P = new mgx_summa_plan;
    P->desc = *desc;
    P->rcut = desc->row_cuts ? std::vector<int>(desc->row_cuts, desc->row_cuts + desc->grid_rows + 1)
                             : even_cuts(desc->m, desc->grid_rows);
    P->ccut = desc->col_cuts ? std::vector<int>(desc->col_cuts, desc->col_cuts + desc->grid_cols + 1)
                             : even_cuts(desc->n, desc->grid_cols);
    P->desc.row_cuts = nullptr;
    P->desc.col_cuts = nullptr;
    if (!cuts_ok(P->rcut, desc->m) || !cuts_ok(P->ccut, desc->n)) {
        delete P;
        mgx_set_last_message("mgx_summa_plan_create: block cuts must rise strictly from 0 to the extent");
        return MGX_E_INVALID;
    }
    std::vector<int4> tiles = summa_tiles(P->rcut, P->ccut);
    P->num_tiles = (int)tiles.size();
    cudaGetDevice(&P->device);
    if (cudaMalloc(&P->d_tiles, tiles.size() * sizeof(int4)) != cudaSuccess ||
        cudaMemcpy(P->d_tiles, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) {
        mgx_set_last_message("mgx_summa_plan_create: could not store the work list on the device");
        if (P->d_tiles) cudaFree(P->d_tiles);
        delete P;
        return MGX_E_CUDA;
    }
    if (desc->form == MGX_FORM_OZAKI || desc->form == MGX_FORM_CRT) {
        P->ws_bytes = desc->form == MGX_FORM_OZAKI ? mgx_ozaki_workspace_size(desc->m, desc->n, desc->k, desc->splits)
                                                   : mgx_crt_workspace_size(desc->m, desc->n, desc->k, desc->splits);
        if (cudaMalloc(&P->ws, P->ws_bytes) != cudaSuccess) {
            mgx_set_last_message("mgx_summa_plan_create: workspace of %zu bytes", P->ws_bytes);
            cudaFree(P->d_tiles);
            delete P;
            return MGX_E_CUDA;
        }
    }
    *plan = P;
    return MGX_SUCCESS;
}

MGX_API int mgx_summa_run(mgx_summa_plan_t *P, const double *A, int lda, const double *B, int ldb, double *C, int ldc,
                          void *stream)
{
    if (!P || !A || !B || !C || lda < P->desc.k || ldb < P->desc.n || ldc < P->desc.n) {
        mgx_set_last_message("mgx_summa_run: invalid arguments");
        return MGX_E_INVALID;
    }
    const mgx_summa_desc_t &d = P->desc;
    cudaStream_t s = (cudaStream_t)stream;
    if (d.form == MGX_FORM_OZAKI)  // element values do not depend on the tiling: one uniform 128 x 128 raster
        return mgx_ozaki_run(A, B, C, d.m, d.n, d.k, lda, ldb, ldc, 0, d.splits, P->ws, P->ws_bytes, s);
    if (d.form == MGX_FORM_CRT)  // likewise: one CRT product of the whole C
        return mgx_crt_run(A, B, C, d.m, d.n, d.k, lda, ldb, ldc, 0, d.splits, P->ws, P->ws_bytes, s);
    // C = 0 (2D-block-matrix/mmb.cu:186), then every panel adds into it.
    MGX_HOST_CHECK(cudaMemset2DAsync(C, (size_t)ldc * sizeof(double), 0, (size_t)d.n * sizeof(double), d.m, s));
    const int bk = d.panel_k < d.k ? d.panel_k : d.k;
    if (bk % 32 == 0)
        return mgx_launch_dgemm_ex(A, B, C, d.m, d.n, d.k, 0, d.k, d.k, lda, ldb, ldc, 1, s, 0, P->d_tiles,
                                   P->num_tiles, bk / 32);
    // Panels that do not align with the kernel's 32-wide K blocks: one launch per panel.
    for (int k0 = 0; k0 < d.k; k0 += bk) {
        const int kc = (d.k - k0 < bk) ? d.k - k0 : bk;
        const int rc = mgx_launch_dgemm_ex(A, B + (size_t)k0 * ldb, C, d.m, d.n, kc, k0, k0 + kc, kc, lda, ldb, ldc, 1,
                                           s, 0, P->d_tiles, P->num_tiles, 0);
        if (rc != MGX_SUCCESS) return rc;
    }
    return MGX_SUCCESS;
}

MGX_API int mgx_summa_plan_info(const mgx_summa_plan_t *P, int *work_tiles, int *panels, size_t *workspace_bytes)
{
    if (!P) return MGX_E_INVALID;
    const mgx_summa_desc_t &d = P->desc;
    int tiles = P->num_tiles, steps = (d.k + d.panel_k - 1) / d.panel_k;
    if (d.form == MGX_FORM_OZAKI) {
        // one whole product of C: 128 x 128 output tiles, one K chunk per int32 accumulation
        const int kmax = mgx_ozaki_kmax(d.splits);
        tiles = ((d.m + 127) / 128) * ((d.n + 127) / 128);
        steps = kmax > 0 ? (d.k + kmax - 1) / kmax : 1;
    } else if (d.form == MGX_FORM_CRT) {
        // one whole product of C: (modulus, 256 x 256 tile) work items, K chunks likewise
        const int kmax = mgx_crt_kmax();
        tiles = d.splits * ((d.m + 255) / 256) * ((d.n + 255) / 256);
        steps = (d.k + kmax - 1) / kmax;
    }
    if (work_tiles) *work_tiles = tiles;
    if (panels) *panels = steps;
    if (workspace_bytes) *workspace_bytes = P->ws_bytes;
    return MGX_SUCCESS;
}

MGX_API int mgx_summa_plan_destroy(mgx_summa_plan_t *P)
{
    if (!P) return MGX_SUCCESS;
    if (P->d_tiles) cudaFree(P->d_tiles);
    if (P->ws) cudaFree(P->ws);
    delete P;
    return MGX_SUCCESS;
}

}  // extern "C"
