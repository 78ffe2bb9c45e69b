"""The cost model's hand-written CUDA forward / backward / Adam kernels against the CPU oracle:
forward outputs, and gradients against central finite differences of the loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def tensors(mgx, n=200, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 6)).astype(np.float32)
    Y = rng.normal(size=(n, 2)).astype(np.float32)
    w = np.array([1.0, 0.5], np.float32)
    P = torch.empty(mgx.mlp_param_count(), dtype=torch.float32, device="cuda")
    mgx.mlp_init(P, seed=7)
    return X, Y, w, P


def test_forward_matches_oracle(mgx):
    import torch
    from oracle import mlp_oracle as MO
    X, Y, w, P = tensors(mgx)
    assert mgx.mlp_param_count() == MO.NPARAM
    out = mgx.mlp_forward(torch.from_numpy(X).cuda(), P).cpu().numpy()
    ref = MO.forward(P.cpu().numpy().astype(np.float64), X.astype(np.float64))
    assert np.max(np.abs(out - ref)) < 1e-5


def test_gradients_match_finite_differences(mgx):
    import torch
    from oracle import mlp_oracle as MO
    X, Y, w, P = tensors(mgx, n=64, seed=1)
    p = P.cpu().numpy().astype(np.float64)
    G = torch.empty_like(P)
    L = torch.empty(1, dtype=torch.float32, device="cuda")
    mgx.mlp_gradients(torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda(), torch.from_numpy(w).cuda(), P, G, L)
    g = G.cpu().numpy().astype(np.float64)
    assert abs(L.item() - MO.loss(p, X.astype(np.float64), Y.astype(np.float64), w)) < 1e-5
    rng = np.random.default_rng(2)
    # every bias and a sample of each weight matrix
    idx = list(rng.choice(384, 40, replace=False)) + list(range(384, 448)) + \
          list(448 + rng.choice(4096, 60, replace=False)) + list(range(4544, 4608)) + list(range(4608, 4738))
    fd = MO.fd_gradient(p, X.astype(np.float64), Y.astype(np.float64), w, idx=idx)
    for i in idx:
        assert abs(g[i] - fd[i]) <= 2e-4 * max(1.0, abs(fd[i])), (i, g[i], fd[i])


def test_adam_training_fits_a_smooth_function(mgx):
    import torch
    rng = np.random.default_rng(3)
    X = rng.uniform(-1, 1, (1024, 6)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2], X[:, 3] ** 2 - X[:, 4]], axis=1).astype(np.float32)
    dX, dY = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    w = torch.tensor([1.0, 1.0], device="cuda")
    P = torch.empty(mgx.mlp_param_count(), dtype=torch.float32, device="cuda")
    mgx.mlp_init(P, seed=11)
    G, M, V = torch.empty_like(P), torch.zeros_like(P), torch.zeros_like(P)
    L = torch.empty(1, dtype=torch.float32, device="cuda")
    mgx.mlp_gradients(dX, dY, w, P, G, L)
    first = L.item()
    step = 0
    for epoch in range(150):
        perm = torch.randperm(1024, device="cuda")
        for b in range(0, 1024, 128):
            i = perm[b:b + 128]
            mgx.mlp_gradients(dX[i].contiguous(), dY[i].contiguous(), w, P, G, L)
            step += 1
            mgx.mlp_adam_step(P, G, M, V, step, 3e-3)
    mgx.mlp_gradients(dX, dY, w, P, G, L)
    assert L.item() < 0.05 * first
