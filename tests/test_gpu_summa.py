"""Persistent SUMMA plans on the GPU: every block and panel in one kernel, matching the per-panel
reference structure (2D-block-matrix/mmb.cu:239-361)."""
import numpy as np
import pytest

from conftest import gamma, rng_matrix
from gpu_util import bits, dev, host

pytestmark = pytest.mark.gpu


def per_panel(mgx, dA, dB, M, N, K, bk, rcut, ccut):
    """The reference's structure: C = 0, then one accumulate launch per (panel, block)."""
    import torch
    C = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    for k0 in range(0, K, bk):
        kc = min(bk, K - k0)
        for bi in range(len(rcut) - 1):
            for bj in range(len(ccut) - 1):
                r0, c0 = rcut[bi], ccut[bj]
                mgx.ab_multiply_accumulate_async(dA[r0:], dB[k0:, c0:], C[r0:, c0:], rcut[bi + 1] - r0,
                                                 ccut[bj + 1] - c0, K, k0, kc, K, N, N)
    return C


@pytest.mark.parametrize("M,N,K,pr,pc,bk,cuts", [
    (384, 640, 512, 3, 5, 64, None),          # even blocks
    (389, 613, 530, 3, 5, 64, None),          # remainders on both axes and in K
    (300, 300, 256, 2, 2, 96, ([0, 100, 300], [0, 250, 300])),  # explicit uneven cuts
    (256, 256, 300, 2, 2, 100, None),         # panel width not a multiple of 32
])
def test_summa_fp64_matches_per_panel_and_oracle(mgx, oracle, M, N, K, pr, pc, bk, cuts):
    import torch
    rng = np.random.default_rng(M + N + K)
    A, B = rng_matrix(rng, (M, K)), rng_matrix(rng, (K, N))
    dA, dB = dev(A), dev(B)
    rc, cc = cuts if cuts else (None, None)
    plan = mgx.SummaPlan(M, N, K, pr, pc, bk, row_cuts=rc, col_cuts=cc)
    C = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
    plan.run(dA, dB, C)
    got = host(C)
    if rc is None:
        rc = [sum(M // pr + (1 if i < M % pr else 0) for i in range(b)) for b in range(pr + 1)]
        cc = [sum(N // pc + (1 if j < N % pc else 0) for j in range(b)) for b in range(pc + 1)]
    ref_gpu = host(per_panel(mgx, dA, dB, M, N, K, bk, rc, cc))
    assert np.array_equal(bits(got), bits(ref_gpu))
    ref = oracle.summa2d(A, B, bk)
    _, _, ab = oracle.gemm_dd(A, B)
    assert np.all(np.abs(got - ref) <= 2 * gamma(K) * ab + 4 * 2.0 ** -53 * np.abs(ref) * (K // bk + 1))
    info = plan.info()
    assert info["panels"] == (K + bk - 1) // bk
    plan.close()


def test_summa_constant_known_answer(mgx):
    import torch
    M, N, K = 12 * 32, 20 * 32, 16 * 32
    plan = mgx.SummaPlan(M, N, K, 3, 5, 64)
    A = torch.ones((M, K), dtype=torch.float64, device="cuda")
    B = torch.full((K, N), 2.0, dtype=torch.float64, device="cuda")
    C = torch.empty((M, N), dtype=torch.float64, device="cuda")
    plan.run(A, B, C)
    assert torch.all(C == 2.0 * K)


def test_summa_ozaki_form(mgx, oracle):
    import torch
    rng = np.random.default_rng(9)
    M, N, K = 389, 613, 530
    A, B = rng_matrix(rng, (M, K), "wide"), rng_matrix(rng, (K, N), "wide")
    plan = mgx.SummaPlan(M, N, K, 3, 5, 64, form=mgx.FORM_OZAKI, splits=8)
    C = torch.empty((M, N), dtype=torch.float64, device="cuda")
    plan.run(dev(A), dev(B), C)
    assert np.array_equal(bits(host(C)), bits(oracle.ozaki_gemm(A, B, 8)))


def test_summa_graph_capture_replays(mgx):
    import torch
    M, N, K = 256, 384, 512
    rng = np.random.default_rng(10)
    dA, dB = dev(rng_matrix(rng, (M, K))), dev(rng_matrix(rng, (K, N)))
    plan = mgx.SummaPlan(M, N, K, 2, 3, 128)
    C1 = torch.empty((M, N), dtype=torch.float64, device="cuda")
    plan.run(dA, dB, C1)
    C2 = torch.empty((M, N), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.run(dA, dB, C2, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)


def test_summa_crt_form_and_graph_replay(mgx, oracle):
    """A plan with the CRT form runs the grid as one CRT product: bit-identical to the oracle's
    restatement, uneven cuts included, and the same again when replayed from a CUDA graph."""
    import torch
    rng = np.random.default_rng(11)
    M, N, K = 389, 613, 530
    A, B = rng_matrix(rng, (M, K), "wide"), rng_matrix(rng, (K, N), "wide")
    dA, dB = dev(A), dev(B)
    plan = mgx.SummaPlan(M, N, K, 3, 5, 64, form=mgx.FORM_CRT, splits=15,
                         row_cuts=[0, 100, 250, M], col_cuts=[0, 7, 200, 400, 401, N])
    C1 = torch.empty((M, N), dtype=torch.float64, device="cuda")
    plan.run(dA, dB, C1)
    assert np.array_equal(bits(host(C1)), bits(oracle.crt_gemm(A, B, 15)))
    C2 = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.run(dA, dB, C2, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(C1.view(torch.int64), C2.view(torch.int64))
    with pytest.raises(mgx.MgxError):
        mgx.SummaPlan(M, N, K, 3, 5, 64, form=mgx.FORM_CRT, splits=7)
