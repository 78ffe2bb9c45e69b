"""The C ABI library loads and exports every entry point include/mgxgemm.h declares (no GPU)."""
import ctypes
import re
import subprocess

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "mgxgemm.h").read_text()
    return sorted(set(re.findall(r"MGX_API\s+[^;(]*?\b(mgx_\w+)\s*\(", text, flags=re.S)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("mgx_ab_multiply", "mgx_ab_multiply_accumulate_async", "mgx_validate_matrix_c",
                     "mgx_gemm_fp64", "mgx_gemm_ozaki", "mgx_summa_run", "mgx_error_vs_dd"):
        assert required in names


def test_library_exports_every_declared_symbol(mgx):
    lib = ctypes.CDLL(str(mgx.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(mgx.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (mgx_\w+)", out))
    assert set(declared_symbols()) <= exported
    # the Python mirror binds every declared entry point
    assert set(declared_symbols()) == {n for n, _, _ in mgx.EXPORTS}


def test_host_only_calls(mgx):
    L = mgx.lib()
    assert L.mgx_status_string(-3) == b"non-finite input"
    assert mgx.ozaki_workspace_size(0, 0, 0, 1) == 0          # splits out of range
    assert mgx.ozaki_workspace_size(1000, 500, 300, 8) >= 8 * 1500 * 320
    assert mgx.ozaki_kmax(8) == 65408
    assert mgx.ozaki_choose_splits(16384, 20.0, 1e-15) == 8
    assert mgx.ozaki_choose_splits(16384, 0.0, 1e-12) < 8
    # argument checks return before touching a device
    assert L.mgx_ab_multiply(None, None, None, 4, 4, 4, 4, 4, 4, 0) == -1          # w must be positive
    assert L.mgx_gemm_fp64(None, None, None, -1, 4, 4, 4, 4, 4, 0, None) == -1
    assert L.mgx_gemm_ozaki(None, None, None, 4, 4, 4, 4, 4, 4, 0, 1, None, 0, None) == -1


def test_summa_work_list_covers_blocks_once_with_even_tma_columns(mgx):
    import numpy as np
    for (m, n, pr, pc, rc, cc) in [(389, 613, 3, 5, None, None), (12288, 20480, 3, 5, None, None),
                                   (300, 300, 2, 2, [0, 100, 300], [0, 251, 300]), (7, 9, 7, 9, None, None)]:
        tiles = mgx.summa_tiles(m, n, pr, pc, rc, cc)
        cover = np.zeros((m, n), np.int32)
        for (m0, n_lo, m_end, n_end) in tiles:
            assert m_end - m0 <= 128 and 0 < n_end - n_lo <= 128
            assert (n_lo & ~1) + 128 >= n_end      # the tile's even TMA base reaches every stored column
            cover[m0:m_end, n_lo:n_end] += 1
        assert cover.min() == 1 and cover.max() == 1
    assert len(mgx.summa_tiles(12288, 20480, 3, 5)) == 96 * 160
