#!/usr/bin/env python3
"""Generates tests/golden/ref_kernels.npz: outputs of MGXBench's OWN FP64 kernels
(sharedABMultiply via ABMultiply, sharedABMultiplyAccumulate via ABMultiplyAccumulateAsync,
1D-row-block/mulmat_kernel.cu), compiled unmodified from its sources into oracle/_ref/ by
`make -C oracle ref`, run on a GPU with seeded inputs.  tests/test_golden.py checks on the CPU
that the oracle reproduces every output bit for bit.

Run on a CUDA machine from the repository root:  python tests/golden/make_golden.py
"""
import ctypes
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

CASES_MUL = [(17, 19, 23), (33, 47, 65), (64, 96, 130), (129, 65, 257)]
CASES_ACC = [  # (m, n, k_total, k_offset, k_chunk)
    (40, 36, 200, 64, 96), (31, 50, 128, 96, 64), (64, 64, 100, 0, 100)]


def main():
    import torch
    from oracle import oracle as O
    R = O.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref_mulmat.so is missing: run `make -C oracle ref` where the sources are")
    rng = np.random.default_rng(20240901)
    out = {}
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    for i, (m, n, k) in enumerate(CASES_MUL):
        A = rng.uniform(-1, 1, (m, k))
        B = rng.uniform(-1, 1, (k, n)) * np.exp2(rng.integers(-8, 9, (k, n)))
        dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
        assert R.ref_ab_multiply(vp(dA), vp(dB), vp(dC), m, n, k, k, n, n) == 0
        out[f"mul{i}_A"], out[f"mul{i}_B"], out[f"mul{i}_C"] = A, B, dC.cpu().numpy()
    for i, (m, n, kt, ko, kc) in enumerate(CASES_ACC):
        A = rng.uniform(-1, 1, (m, kt))
        Bc = rng.uniform(-1, 1, (kc, n))
        C0 = rng.uniform(-1, 1, (m, n))
        dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, Bc, C0.copy()))
        assert R.ref_ab_multiply_accumulate(vp(dA), vp(dB), vp(dC), m, n, kt, ko, kc, kt, n, n, None) == 0
        out[f"acc{i}_A"], out[f"acc{i}_B"], out[f"acc{i}_C0"], out[f"acc{i}_C"] = A, Bc, C0, dC.cpu().numpy()
        out[f"acc{i}_args"] = np.array([m, n, kt, ko, kc])
    # the reference's NUMERICAL VALIDATION block for one failing and one passing matrix
    code = ("import ctypes,sys,torch;sys.path.insert(0,%r);from oracle import oracle as O;R=O.ref_lib();"
            "C=torch.full((40,50),100.0,dtype=torch.float64,device='cuda');C[1,1]=100.5;"
            "R.ref_validate_matrix_C(ctypes.c_void_p(C.data_ptr()),40,50,100.0,1e-9,1e-12);"
            "C[1,1]=100.0;R.ref_validate_matrix_C(ctypes.c_void_p(C.data_ptr()),40,50,100.0,1e-9,1e-12)" % str(ROOT))
    text = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    out["validation_text"] = np.array(text)
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_kernels.npz", **out)
    print("wrote tests/golden/ref_kernels.npz with", len(CASES_MUL), "multiply and", len(CASES_ACC), "accumulate cases")


if __name__ == "__main__":
    main()
