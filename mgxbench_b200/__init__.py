"""mgxbench_b200 -- Python host mirror of libmgxgemm's C ABI (include/mgxgemm.h).

The names follow MGXBench's own GPU entry points (mulmat_kernel.cu): ``ab_multiply`` is
``ABMultiply``, ``ab_multiply_accumulate_async`` is ``ABMultiplyAccumulateAsync`` and
``validate_matrix_c`` is ``validate_matrix_C``, with the same argument meaning.  Matrices are
torch CUDA tensors (FP64, row-major); leading dimensions default to the tensors' row strides.

Every call goes through the compiled library ``mgxbench_b200/lib/libmgxgemm.so``; there is no
Python or CPU fallback.  A missing library, or a failing call, raises ``MgxError``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libmgxgemm.so"
REPO = PKG.parent
BUILD_DIR = REPO / "build"
LAUNCHER = PKG / "mgx-onegpu-launch"

MGX_SUCCESS = 0
STATUS_NAMES = {0: "success", -1: "invalid argument", -2: "CUDA error", -3: "non-finite input",
                -4: "device-side wait timed out", -5: "workspace missing or too small",
                -6: "unsupported configuration", -7: "device-side error"}
FORM_FP64, FORM_OZAKI, FORM_CRT = 0, 1, 2


class MgxError(RuntimeError):
    def __init__(self, status: int, what: str, message: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)} ({message})")


class Validation(ctypes.Structure):
    _fields_ = [("elements", ctypes.c_uint64), ("invalid", ctypes.c_uint64),
                ("max_abs_error", ctypes.c_double), ("max_rel_error", ctypes.c_double)]


class ErrorReport(ctypes.Structure):
    _fields_ = [("normwise", ctypes.c_double), ("max_rel", ctypes.c_double),
                ("max_componentwise", ctypes.c_double), ("max_abs", ctypes.c_double),
                ("rows_checked", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SummaDesc(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("k", ctypes.c_int),
                ("grid_rows", ctypes.c_int), ("grid_cols", ctypes.c_int),
                ("row_cuts", ctypes.POINTER(ctypes.c_int)), ("col_cuts", ctypes.POINTER(ctypes.c_int)),
                ("panel_k", ctypes.c_int), ("form", ctypes.c_int), ("splits", ctypes.c_int)]


# (name, restype, argtypes) of every exported entry point declared in include/mgxgemm.h
_i, _d, _vp, _sz, _u64 = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64
EXPORTS = [
    ("mgx_ab_multiply", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i]),
    ("mgx_ab_multiply_accumulate_async", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp]),
    ("mgx_validate_matrix_c", _i, [_vp, _i, _i, _d, _d, _d, _i, _i, ctypes.POINTER(Validation)]),
    ("mgx_gemm_fp64", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _vp]),
    ("mgx_fp64_splitk_workspace_size", _sz, [_i, _i, _i, _i]),
    ("mgx_gemm_fp64_splitk", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_gemm_fp64_tiled", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_fp64_streamk_workspace_size", _sz, [_i, _i, _i]),
    ("mgx_gemm_fp64_streamk", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_ozaki_workspace_size", _sz, [_i, _i, _i, _i]),
    ("mgx_gemm_ozaki", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_ozaki_splitk_workspace_size", _sz, [_i, _i, _i, _i, _i]),
    ("mgx_gemm_ozaki_splitk", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_ozaki_choose_splits", _i, [_i, _d, _d]),
    ("mgx_ozaki_split", _i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_ozaki_multiply", _i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_ozaki_kmax", _i, [_i]),
    ("mgx_crt_workspace_size", _sz, [_i, _i, _i, _i]),
    ("mgx_gemm_ozaki_crt", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_crt_splitk_workspace_size", _sz, [_i, _i, _i, _i, _i]),
    ("mgx_gemm_ozaki_crt_splitk", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_crt_split", _i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_crt_products", _i, [_i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_crt_combine", _i, [_vp, _i, _i, _i, _i, _i, _i, _vp, _sz, _vp]),
    ("mgx_crt_choose_moduli", _i, [_i, _d]),
    ("mgx_crt_kmax", _i, []),
    ("mgx_gemm_ozaki_noalloc", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp]),
    ("mgx_gemm_host", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _vp]),
    ("mgx_summa_tiles", _i, [ctypes.POINTER(SummaDesc), ctypes.POINTER(_i), _i]),
    ("mgx_summa_plan_create", _i, [ctypes.POINTER(SummaDesc), ctypes.POINTER(_vp)]),
    ("mgx_summa_run", _i, [_vp, _vp, _i, _vp, _i, _vp, _i, _vp]),
    ("mgx_summa_plan_info", _i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_sz)]),
    ("mgx_summa_plan_destroy", _i, [_vp]),
    ("mgx_error_vs_dd", _i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _d, ctypes.POINTER(ErrorReport)]),
    ("mgx_fill_matrix", _i, [_vp, _i, _i, _i, _i, _d, _i, _u64, _vp]),
    ("mgx_device_status", _i, [ctypes.POINTER(_i)]),
    ("mgx_scratch_trim", _i, []),
    ("mgx_wait_probe", _i, [_i]),
    ("mgx_last_error_message", ctypes.c_char_p, []),
    ("mgx_status_string", ctypes.c_char_p, [_i]),
    ("mgx_peak_fp64", _i, [_i, _i, ctypes.POINTER(_d)]),
    ("mgx_peak_int8", _i, [_i, _i, ctypes.POINTER(_d)]),
    ("mgx_mlp_param_count", _i, []),
    ("mgx_mlp_init", _i, [_vp, _u64, _vp]),
    ("mgx_mlp_forward", _i, [_vp, _i, _vp, _vp, _vp]),
    ("mgx_mlp_gradients", _i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _vp]),
    ("mgx_mlp_adam_step", _i, [_vp, _vp, _vp, _vp, _i, ctypes.c_float, _vp]),
]

_lib = None


def lib():
    """Loads the compiled library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise MgxError(-6, "load", f"{LIB_PATH} is missing: build with `make -C mgxbench_b200`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in EXPORTS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str) -> int:
    if rc < 0:
        raise MgxError(rc, what, lib().mgx_last_error_message().decode(errors="replace"))
    return rc


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _ld(t) -> int:
    assert t.dim() == 2 and t.stride(1) == 1, "row-major matrices with unit column stride"
    return t.stride(0)


def _check_f64(*ts):
    import torch
    for t in ts:
        if t.dtype != torch.float64 or not t.is_cuda:
            raise MgxError(-1, "argument", "matrices must be float64 CUDA tensors")


# ------------------------------------------------------------------ reference-named entry points
def ab_multiply(a, b, c, m=None, n=None, k=None, lda=None, ldb=None, ldc=None, w: int = 32):
    """ABMultiply: c[m x n] = a[m x k] @ b[k x n] on the legacy default stream."""
    _check_f64(a, b, c)
    m = a.shape[0] if m is None else m
    k = a.shape[1] if k is None else k
    n = b.shape[1] if n is None else n
    return _check(lib().mgx_ab_multiply(_ptr(a), _ptr(b), _ptr(c), m, n, k, lda or _ld(a), ldb or _ld(b),
                                         ldc or _ld(c), w), "mgx_ab_multiply")


def ab_multiply_accumulate_async(a, b_chunk, c, m, n, k_total, k_offset, k_chunk, lda, ldb, ldc, w=32,
                                 stream=None):
    """ABMultiplyAccumulateAsync: c += a[:, k_offset:k_offset+k_chunk] @ b_chunk (chunk summed first)."""
    _check_f64(a, b_chunk, c)
    return _check(lib().mgx_ab_multiply_accumulate_async(_ptr(a), _ptr(b_chunk), _ptr(c), m, n, k_total,
                                                          k_offset, k_chunk, lda, ldb, ldc, w,
                                                          _stream(stream)),
                  "mgx_ab_multiply_accumulate_async")


def validate_matrix_c(d_c, rows, cols, expected, abs_tol=1e-9, rel_tol=1e-12, rank=0, print_block=False):
    """validate_matrix_C: returns (passed, Validation)."""
    _check_f64(d_c)
    v = Validation()
    rc = _check(lib().mgx_validate_matrix_c(_ptr(d_c), rows, cols, expected, abs_tol, rel_tol, rank,
                                            int(print_block), ctypes.byref(v)), "mgx_validate_matrix_c")
    return rc == 1, v


# ------------------------------------------------------------------ library forms
def fp64_splitk_workspace_size(m, n, k, ksplit) -> int:
    return int(lib().mgx_fp64_splitk_workspace_size(m, n, k, ksplit))


def gemm_fp64(A, B, C, beta_one: bool = False, stream=None, ksplit: int = 1, workspace=None, tile_m: int = 128):
    """C (+)= A B on the FP64 tensor cores; ksplit > 1 cuts K into slices computed by separate
    CTAs (for products with few output tiles) and needs a workspace (grown on demand); tile_m = 64
    runs 64 x 128 output tiles instead of 128 x 128 (same result, bit for bit); ksplit = 0 is the
    stream-K form over 64 x 128 tiles (equal K shares per CTA, workspace grown on demand)."""
    _check_f64(A, B, C)
    m, k = A.shape
    n = B.shape[1]
    if ksplit == 0:
        # stream-K over 64 x 128 tiles
        need = lib().mgx_fp64_streamk_workspace_size(m, n, k)
        ws = (workspace or _default_ws).get(need) if need else None
        return _check(lib().mgx_gemm_fp64_streamk(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                                  int(beta_one), _ptr(ws), ws.numel() if ws is not None else 0,
                                                  _stream(stream)), "mgx_gemm_fp64_streamk")
    if tile_m != 128:
        need = fp64_splitk_workspace_size(m, n, k, ksplit) if ksplit > 1 else 0
        ws = (workspace or _default_ws).get(need) if need else None
        return _check(lib().mgx_gemm_fp64_tiled(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                                int(beta_one), tile_m, ksplit, _ptr(ws) if ws is not None else None,
                                                ws.numel() if ws is not None else 0, _stream(stream)),
                      "mgx_gemm_fp64_tiled")
    if ksplit > 1:
        need = fp64_splitk_workspace_size(m, n, k, ksplit)
        ws = (workspace or _default_ws).get(need)
        return _check(lib().mgx_gemm_fp64_splitk(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                                 int(beta_one), ksplit, _ptr(ws), ws.numel(), _stream(stream)),
                      "mgx_gemm_fp64_splitk")
    return _check(lib().mgx_gemm_fp64(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                      int(beta_one), _stream(stream)), "mgx_gemm_fp64")


def ozaki_workspace_size(m, n, k, splits) -> int:
    return int(lib().mgx_ozaki_workspace_size(m, n, k, splits))


class OzakiWorkspace:
    """Device workspace for gemm_ozaki, grown on demand (256-byte aligned torch allocation)."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes: int):
        import torch
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device="cuda")
        return self.buf


# Shared by calls that pass no workspace.  Calls that may run concurrently on different streams
# must each pass their own OzakiWorkspace (a shared one would be overwritten in flight).
_default_ws = OzakiWorkspace()


def ozaki_splitk_workspace_size(m, n, k, splits, ksplit) -> int:
    return int(lib().mgx_ozaki_splitk_workspace_size(m, n, k, splits, ksplit))


def gemm_ozaki(A, B, C, splits: int = 8, beta_one: bool = False, workspace=None, stream=None, ksplit: int = 1):
    """C (+)= A B by the Ozaki form; ksplit > 1 cuts K into slices computed by separate CTAs
    (mgx_gemm_ozaki_splitk, for products with few output tiles)."""
    _check_f64(A, B, C)
    m, k = A.shape
    n = B.shape[1]
    if ksplit > 1:
        need = ozaki_splitk_workspace_size(m, n, k, splits, ksplit)
        ws = (workspace or _default_ws).get(need)
        return _check(lib().mgx_gemm_ozaki_splitk(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                                  int(beta_one), splits, ksplit, _ptr(ws), ws.numel(),
                                                  _stream(stream)), "mgx_gemm_ozaki_splitk")
    need = ozaki_workspace_size(m, n, k, splits)
    ws = (workspace or _default_ws).get(need)
    return _check(lib().mgx_gemm_ozaki(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                       int(beta_one), splits, _ptr(ws), ws.numel(), _stream(stream)),
                  "mgx_gemm_ozaki")


def crt_workspace_size(m, n, k, moduli) -> int:
    return int(lib().mgx_crt_workspace_size(m, n, k, moduli))


def crt_splitk_workspace_size(m, n, k, moduli, ksplit) -> int:
    return int(lib().mgx_crt_splitk_workspace_size(m, n, k, moduli, ksplit))


def gemm_ozaki_crt(A, B, C, moduli: int = 15, beta_one: bool = False, workspace=None, stream=None, ksplit: int = 1):
    """C (+)= A B by the CRT form (Ozaki scheme II): one INT8 tensor-core product per modulus,
    FP64 result rebuilt by the Chinese remainder theorem (mgx_gemm_ozaki_crt); ksplit > 1 cuts K
    into slices computed as separate work items (mgx_gemm_ozaki_crt_splitk, same result)."""
    _check_f64(A, B, C)
    m, k = A.shape
    n = B.shape[1]
    if ksplit > 1:
        need = crt_splitk_workspace_size(m, n, k, moduli, ksplit)
        ws = (workspace or _default_ws).get(need)
        return _check(lib().mgx_gemm_ozaki_crt_splitk(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                                      int(beta_one), moduli, ksplit, _ptr(ws), ws.numel(),
                                                      _stream(stream)), "mgx_gemm_ozaki_crt_splitk")
    need = crt_workspace_size(m, n, k, moduli)
    ws = (workspace or _default_ws).get(need)
    return _check(lib().mgx_gemm_ozaki_crt(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C),
                                           int(beta_one), moduli, _ptr(ws), ws.numel(), _stream(stream)),
                  "mgx_gemm_ozaki_crt")


def crt_split(A, B, moduli: int, workspace, stream=None):
    """Phase 1 of gemm_ozaki_crt (k <= crt_kmax()): scales and residues of A and B into `workspace`."""
    _check_f64(A, B)
    m, k = A.shape
    n = B.shape[1]
    return _check(lib().mgx_crt_split(_ptr(A), _ptr(B), m, n, k, _ld(A), _ld(B), moduli, _ptr(workspace),
                                      workspace.numel(), _stream(stream)), "mgx_crt_split")


def crt_products(m: int, n: int, k: int, moduli: int, workspace, stream=None):
    """Phase 2: the residue products on the tensor cores (one persistent launch)."""
    return _check(lib().mgx_crt_products(m, n, k, moduli, _ptr(workspace), workspace.numel(), _stream(stream)),
                  "mgx_crt_products")


def crt_combine(C, k: int, moduli: int, workspace, beta_one: bool = False, stream=None):
    """Phase 3: C (+)= the CRT recombination of the product residues in `workspace`."""
    _check_f64(C)
    m, n = C.shape
    return _check(lib().mgx_crt_combine(_ptr(C), m, n, k, _ld(C), int(beta_one), moduli, _ptr(workspace),
                                        workspace.numel(), _stream(stream)), "mgx_crt_combine")


def crt_choose_moduli(k: int, target: float = 1e-15) -> int:
    return int(lib().mgx_crt_choose_moduli(k, target))


def crt_kmax() -> int:
    return int(lib().mgx_crt_kmax())


def ozaki_split(A, B, splits: int, workspace, stream=None):
    """Phase 1 of gemm_ozaki (k <= ozaki_kmax(splits)): slices of A and B into `workspace`."""
    _check_f64(A, B)
    m, k = A.shape
    n = B.shape[1]
    return _check(lib().mgx_ozaki_split(_ptr(A), _ptr(B), m, n, k, _ld(A), _ld(B), splits, _ptr(workspace),
                                        workspace.numel(), _stream(stream)), "mgx_ozaki_split")


def ozaki_multiply(C, k: int, splits: int, workspace, beta_one: bool = False, stream=None):
    """Phase 2 of gemm_ozaki: C (+)= product of the slices held in `workspace`."""
    _check_f64(C)
    m, n = C.shape
    return _check(lib().mgx_ozaki_multiply(_ptr(C), m, n, k, _ld(C), int(beta_one), splits, _ptr(workspace),
                                           workspace.numel(), _stream(stream)), "mgx_ozaki_multiply")


def scratch_trim():
    """Release the device memory the library keeps cached for its scratch on this device."""
    return _check(lib().mgx_scratch_trim(), "mgx_scratch_trim")


def gemm_host(hA, hB, hC, form=FORM_OZAKI, splits=8, panels=32, stream=None):
    """C = A B from host (CPU, ideally pinned) float64 tensors, copies overlapped with compute."""
    import torch
    for t in (hA, hB, hC):
        if t.dtype != torch.float64 or t.is_cuda or t.stride(-1) != 1:
            raise MgxError(-1, "argument", "host matrices must be row-major float64 CPU tensors")
    m, k = hA.shape
    n = hB.shape[1]
    return _check(lib().mgx_gemm_host(_ptr(hA), _ptr(hB), _ptr(hC), m, n, k, hA.stride(0), hB.stride(0),
                                      hC.stride(0), form, splits, panels, _stream(stream)), "mgx_gemm_host")


# Kernel launches of one product per K chunk of one exact int32 accumulation: the FP64 SUMMA
# plan's persistent kernel; the slice form's exponent, digit and product kernels; the CRT form's
# scale, residue, product and recombination kernels.
_LAUNCHES_PER_CHUNK = {FORM_FP64: 1, FORM_OZAKI: 6, FORM_CRT: 8}


def launches_per_product(form: int, k: int, splits: int = 0) -> int:
    """Kernel launches of one SUMMA-plan product of inner dimension k in the given form."""
    if form == FORM_FP64:
        return 1
    kmax = ozaki_kmax(splits) if form == FORM_OZAKI else crt_kmax()
    return _LAUNCHES_PER_CHUNK[form] * ((k + kmax - 1) // kmax)


def ozaki_kmax(splits: int) -> int:
    return int(lib().mgx_ozaki_kmax(splits))


def ozaki_choose_splits(k: int, exp_range: float, target: float = 1e-15) -> int:
    return int(lib().mgx_ozaki_choose_splits(k, exp_range, target))


def summa_tiles(m, n, grid_rows, grid_cols, row_cuts=None, col_cuts=None):
    """Host-side work list of a SUMMA plan: list of (m0, n_lo, m_end, n_end)."""
    d = SummaDesc(m, n, 1, grid_rows, grid_cols, None, None, 1, FORM_FP64, 0)
    keep = []
    if row_cuts is not None:
        keep.append((ctypes.c_int * len(row_cuts))(*row_cuts))
        d.row_cuts = ctypes.cast(keep[-1], ctypes.POINTER(ctypes.c_int))
    if col_cuts is not None:
        keep.append((ctypes.c_int * len(col_cuts))(*col_cuts))
        d.col_cuts = ctypes.cast(keep[-1], ctypes.POINTER(ctypes.c_int))
    count = _check(lib().mgx_summa_tiles(ctypes.byref(d), None, 0), "mgx_summa_tiles")
    buf = (ctypes.c_int * (4 * count))()
    _check(lib().mgx_summa_tiles(ctypes.byref(d), buf, count), "mgx_summa_tiles")
    return [tuple(buf[4 * i:4 * i + 4]) for i in range(count)]


class SummaPlan:
    """mgx_summa_plan_t: every block and panel of a process grid in one persistent kernel."""

    def __init__(self, m, n, k, grid_rows, grid_cols, panel_k, form=FORM_FP64, splits=8,
                 row_cuts=None, col_cuts=None):
        d = SummaDesc(m, n, k, grid_rows, grid_cols, None, None, panel_k, form, splits)
        self._keep = []
        if row_cuts is not None:
            arr = (ctypes.c_int * len(row_cuts))(*row_cuts)
            self._keep.append(arr)
            d.row_cuts = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int))
        if col_cuts is not None:
            arr = (ctypes.c_int * len(col_cuts))(*col_cuts)
            self._keep.append(arr)
            d.col_cuts = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int))
        self.handle = ctypes.c_void_p()
        _check(lib().mgx_summa_plan_create(ctypes.byref(d), ctypes.byref(self.handle)), "mgx_summa_plan_create")

    def run(self, A, B, C, stream=None):
        _check_f64(A, B, C)
        return _check(lib().mgx_summa_run(self.handle, _ptr(A), _ld(A), _ptr(B), _ld(B), _ptr(C), _ld(C),
                                          _stream(stream)), "mgx_summa_run")

    def info(self):
        t, p, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        _check(lib().mgx_summa_plan_info(self.handle, ctypes.byref(t), ctypes.byref(p), ctypes.byref(w)),
               "mgx_summa_plan_info")
        return {"work_tiles": t.value, "panels": p.value, "workspace_bytes": w.value}

    def close(self):
        if self.handle:
            lib().mgx_summa_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def error_vs_dd(A, B, C, row_start=0, row_count=0, floor_rel=2.0 ** -40) -> dict:
    _check_f64(A, B, C)
    m, k = A.shape
    n = B.shape[1]
    e = ErrorReport()
    _check(lib().mgx_error_vs_dd(_ptr(A), _ptr(B), _ptr(C), m, n, k, _ld(A), _ld(B), _ld(C), row_start,
                                 row_count, floor_rel, ctypes.byref(e)), "mgx_error_vs_dd")
    return e.as_dict()


def fill_matrix(X, kind: int, value: float = 0.0, e_range: int = 0, seed: int = 0, stream=None):
    """kind 0 constant, 1 uniform [-1,1), 2 u * 2^e with e uniform in [-e_range, e_range]."""
    _check_f64(X)
    r, c = X.shape
    return _check(lib().mgx_fill_matrix(_ptr(X), r, c, _ld(X), kind, value, e_range, seed, _stream(stream)),
                  "mgx_fill_matrix")


def device_status() -> int:
    code = ctypes.c_int()
    _check(lib().mgx_device_status(ctypes.byref(code)), "mgx_device_status")
    return code.value


def peak_int8(kind: int, iterations: int = 200000) -> float:
    out = ctypes.c_double()
    _check(lib().mgx_peak_int8(kind, iterations, ctypes.byref(out)), "mgx_peak_int8")
    return out.value


def peak_fp64(kind: int, iterations: int = 20000) -> float:
    out = ctypes.c_double()
    _check(lib().mgx_peak_fp64(kind, iterations, ctypes.byref(out)), "mgx_peak_fp64")
    return out.value


# ------------------------------------------------------------------ learned cost model kernels
def _check_f32(*ts):
    import torch
    for t in ts:
        if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
            raise MgxError(-1, "argument", "MLP tensors must be contiguous float32 CUDA tensors")


def mlp_param_count() -> int:
    return int(lib().mgx_mlp_param_count())


def mlp_init(params, seed: int = 0, stream=None):
    _check_f32(params)
    return _check(lib().mgx_mlp_init(_ptr(params), seed, _stream(stream)), "mgx_mlp_init")


def mlp_forward(X, params, out=None, stream=None):
    import torch
    _check_f32(X, params)
    out = torch.empty((X.shape[0], 2), dtype=torch.float32, device="cuda") if out is None else out
    _check(lib().mgx_mlp_forward(_ptr(X), X.shape[0], _ptr(params), _ptr(out), _stream(stream)), "mgx_mlp_forward")
    return out


def mlp_gradients(X, Y, weights, params, grads, loss, stream=None):
    _check_f32(X, Y, weights, params, grads, loss)
    return _check(lib().mgx_mlp_gradients(_ptr(X), _ptr(Y), _ptr(weights), X.shape[0], _ptr(params), _ptr(grads),
                                          _ptr(loss), _stream(stream)), "mgx_mlp_gradients")


def mlp_adam_step(params, grads, m, v, step: int, lr: float, stream=None):
    _check_f32(params, grads, m, v)
    return _check(lib().mgx_mlp_adam_step(_ptr(params), _ptr(grads), _ptr(m), _ptr(v), step, lr, _stream(stream)),
                  "mgx_mlp_adam_step")
