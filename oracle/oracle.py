"""ctypes wrapper over the CPU oracle (oracle/libmgx_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline /
reference legs of bench.py, never by the product package.  Every function mirrors one C entry
point of oracle/mgx_oracle.c, which cites the MGXBench source it restates.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmgx_oracle.so"
REF_LIB_PATH = HERE / "_ref" / "libref_mulmat.so"

_dp = ctypes.POINTER(ctypes.c_double)
_i8p = ctypes.POINTER(ctypes.c_int8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(str(LIB_PATH))
        i, d, sz = ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        L.oracle_ab_multiply.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i, i]
        L.oracle_ab_multiply_naive.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i]
        L.oracle_ab_multiply_accumulate.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i, i, i, i]
        L.oracle_pipeline_k_chunk.argtypes = [i, i]
        L.oracle_pipeline_k_chunk.restype = i
        L.oracle_mm1d.argtypes = [_dp, _dp, _dp, i, i, i, i, i]
        L.oracle_summa2d.argtypes = [_dp, _dp, _dp, i, i, i, i, i]
        L.oracle_validate_constant.argtypes = [_dp, sz, d, d, d, i, ctypes.POINTER(ctypes.c_uint64), _dp, _dp]
        L.oracle_validate_2d.argtypes = [_dp, sz, d]
        L.oracle_validate_2d.restype = ctypes.c_int64
        L.oracle_gemm_dd.argtypes = [_dp, _dp, _dp, _dp, _dp, i, i, i, i, i, i, i]
        L.oracle_error_metrics.argtypes = [_dp, i, _dp, _dp, _dp, i, i, i, d, _dp]
        L.oracle_ozaki_exponents.argtypes = [_dp, _dp, i, i, i, i, i, _i32p, _i32p]
        L.oracle_ozaki_exponents.restype = i
        L.oracle_ozaki_split.argtypes = [_dp, _dp, i, i, i, i, i, i, i, _i32p, _i32p, _i8p, _i8p]
        L.oracle_ozaki_kmax.argtypes = [i]
        L.oracle_ozaki_kmax.restype = i
        L.oracle_ozaki_gemm.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i, i, i, i]
        L.oracle_ozaki_gemm.restype = i
        L.oracle_ozaki_gemm_splitk.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i, i, i, i, i]
        L.oracle_ozaki_gemm_splitk.restype = i
        L.oracle_crt_scales.argtypes = [_dp, _dp, i, i, i, i, i, i, _i32p, _i32p]
        L.oracle_crt_scales.restype = i
        L.oracle_crt_residues.argtypes = [_dp, _dp, i, i, i, i, i, i, i, _i32p, _i32p, _i8p, _i8p]
        L.oracle_crt_kmax.restype = i
        L.oracle_crt_gemm.argtypes = [_dp, _dp, _dp, i, i, i, i, i, i, i, i, i]
        L.oracle_crt_gemm.restype = i
        L.oracle_max_threads.restype = i
        _lib = L
    return _lib


def _p(a: np.ndarray, ty=_dp):
    return a.ctypes.data_as(ty)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ab_multiply(A, B, threads: int = 0, naive: bool = False) -> np.ndarray:
    """C = A @ B as sharedABMultiply computes it (one FMA chain per output)."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    k2, n = B.shape
    assert k == k2
    C = np.empty((m, n), np.float64)
    if naive:
        lib().oracle_ab_multiply_naive(_p(A), _p(B), _p(C), m, n, k, k, n, n)
    else:
        lib().oracle_ab_multiply(_p(A), _p(B), _p(C), m, n, k, k, n, n, threads)
    return C


def ab_multiply_accumulate(A, Bchunk, C, k_offset: int, k_chunk: int, threads: int = 0) -> np.ndarray:
    """C += A[:, k_offset:k_offset+k_chunk] @ Bchunk, in place (sharedABMultiplyAccumulate)."""
    A, Bchunk = _f64(A), _f64(Bchunk)
    assert C.dtype == np.float64 and C.flags.c_contiguous
    m, k_total = A.shape
    n = C.shape[1]
    lib().oracle_ab_multiply_accumulate(_p(A), _p(Bchunk), _p(C), m, n, k_total, k_offset, k_chunk,
                                        k_total, n, n, threads)
    return C


def pipeline_k_chunk(k: int, requested: int = 0) -> int:
    return lib().oracle_pipeline_k_chunk(k, requested)


def mm1d(A, B, ranks: int, chunked: bool, k_chunk: int, threads: int = 0) -> np.ndarray:
    A, B = _f64(A), _f64(B)
    N = A.shape[0]
    C = np.empty((N, N), np.float64)
    lib().oracle_mm1d(_p(A), _p(B), _p(C), N, ranks, int(chunked), k_chunk, threads)
    return C


def summa2d(A, B, bk: int, threads: int = 0) -> np.ndarray:
    A, B = _f64(A), _f64(B)
    M, K = A.shape
    N = B.shape[1]
    C = np.empty((M, N), np.float64)
    lib().oracle_summa2d(_p(A), _p(B), _p(C), M, N, K, bk, threads)
    return C


def validate_constant(C, expected, abs_tol=1e-9, rel_tol=1e-12, count_nonfinite=False):
    C = _f64(C)
    nb = ctypes.c_uint64()
    ma = ctypes.c_double()
    mr = ctypes.c_double()
    lib().oracle_validate_constant(_p(C), C.size, expected, abs_tol, rel_tol, int(count_nonfinite),
                                   ctypes.byref(nb), ctypes.byref(ma), ctypes.byref(mr))
    return int(nb.value), ma.value, mr.value


def validate_2d(C, expected) -> int:
    C = _f64(C)
    return int(lib().oracle_validate_2d(_p(C), C.size, expected))


def gemm_dd(A, B, threads: int = 0):
    """Double-double reference: returns (hi, lo, absprod)."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    hi = np.empty((m, n)); lo = np.empty((m, n)); ab = np.empty((m, n))
    lib().oracle_gemm_dd(_p(A), _p(B), _p(hi), _p(lo), _p(ab), m, n, k, k, n, n, threads)
    return hi, lo, ab


def error_metrics(C, ref, floor_rel: float = 2.0 ** -40) -> dict:
    """normwise, max elementwise relative (|R| >= floor_rel*max|R|), max componentwise, max abs."""
    hi, lo, ab = ref
    C = _f64(C)
    m, n = C.shape
    out = (ctypes.c_double * 4)()
    lib().oracle_error_metrics(_p(C), n, _p(hi), _p(lo), _p(ab), n, m, n, floor_rel, out)
    return {"normwise": out[0], "max_rel": out[1], "max_componentwise": out[2], "max_abs": out[3]}


def ozaki_exponents(A, B):
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    ea = np.empty(m, np.int32); eb = np.empty(n, np.int32)
    bad = lib().oracle_ozaki_exponents(_p(A), _p(B), m, n, k, k, n, _p(ea, _i32p), _p(eb, _i32p))
    return ea, eb, bool(bad)


def ozaki_split(A, B, s: int):
    """Digits (da [s,m,kp], db [s,n,kp]) and exponents of the Ozaki form."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    ea, eb, bad = ozaki_exponents(A, B)
    kp = (k + 15) & ~15
    da = np.empty((s, m, kp), np.int8); db = np.empty((s, n, kp), np.int8)
    lib().oracle_ozaki_split(_p(A), _p(B), m, n, k, k, n, s, kp, _p(ea, _i32p), _p(eb, _i32p),
                             _p(da, _i8p), _p(db, _i8p))
    return da, db, ea, eb


def ozaki_kmax(s: int) -> int:
    return lib().oracle_ozaki_kmax(s)


def ozaki_gemm(A, B, s: int, C=None, beta_one: bool = False, threads: int = 0) -> np.ndarray:
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    if C is None:
        C = np.zeros((m, n), np.float64)
    rc = lib().oracle_ozaki_gemm(_p(A), _p(B), _p(C), m, n, k, k, n, n, s, int(beta_one), threads)
    if rc:
        raise ValueError("non-finite input to the Ozaki form")
    return C


def ozaki_gemm_splitk(A, B, s: int, ksplit: int, C=None, beta_one: bool = False, threads: int = 0) -> np.ndarray:
    """The Ozaki product with the K range cut into ksplit slices, each recombined on its own and
    the slice results added in order (the GPU's split-K form; k <= ozaki kmax)."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    if C is None:
        C = np.zeros((m, n), np.float64)
    rc = lib().oracle_ozaki_gemm_splitk(_p(A), _p(B), _p(C), m, n, k, k, n, n, s, ksplit, int(beta_one), threads)
    if rc == 1:
        raise ValueError("non-finite input to the Ozaki form")
    if rc == 2:
        raise ValueError("k above one int32 accumulation for this split count")
    return C


CRT_MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193)


def crt_scales(A, B, q: int):
    """Power-of-two scale exponents of the CRT form: sigma per row of A, tau per column of B."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    sg = np.empty(m, np.int32); tu = np.empty(n, np.int32)
    rc = lib().oracle_crt_scales(_p(A), _p(B), m, n, k, k, n, q, _p(sg, _i32p), _p(tu, _i32p))
    return sg, tu, rc


def crt_residues(A, B, q: int):
    """Residues of the scaled operands: ra [q, m, kp] and rb [q, n, kp] (B transposed), int8."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    sg, tu, rc = crt_scales(A, B, q)
    kp = (k + 15) & ~15
    ra = np.empty((q, m, kp), np.int8); rb = np.empty((q, n, kp), np.int8)
    lib().oracle_crt_residues(_p(A), _p(B), m, n, k, k, n, q, kp, _p(sg, _i32p), _p(tu, _i32p),
                              _p(ra, _i8p), _p(rb, _i8p))
    return ra, rb, sg, tu


def crt_kmax() -> int:
    return lib().oracle_crt_kmax()


def crt_gemm(A, B, q: int, C=None, beta_one: bool = False, threads: int = 0) -> np.ndarray:
    """A B by the CRT form (Ozaki scheme II) with q moduli, as the GPU computes it."""
    A, B = _f64(A), _f64(B)
    m, k = A.shape
    n = B.shape[1]
    if C is None:
        C = np.zeros((m, n), np.float64)
    rc = lib().oracle_crt_gemm(_p(A), _p(B), _p(C), m, n, k, k, n, n, q, int(beta_one), threads)
    if rc == 1:
        raise ValueError("non-finite input to the CRT form")
    if rc == 2:
        raise ValueError(f"{q} moduli: the CRT form takes 8..16")
    return C


def max_threads() -> int:
    return lib().oracle_max_threads()


def ref_lib():
    """MGXBench's own kernels (oracle/_ref/libref_mulmat.so), or None when not built."""
    if not REF_LIB_PATH.exists():
        return None
    L = ctypes.CDLL(str(REF_LIB_PATH))
    i, d, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.ref_ab_multiply.argtypes = [vp, vp, vp, i, i, i, i, i, i]
    L.ref_ab_multiply.restype = i
    L.ref_ab_multiply_accumulate.argtypes = [vp, vp, vp, i, i, i, i, i, i, i, i, vp]
    L.ref_ab_multiply_accumulate.restype = i
    L.ref_validate_matrix_C.argtypes = [vp, i, i, d, d, d]
    L.ref_validate_matrix_C.restype = i
    return L
