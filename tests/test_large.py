"""Full-size workloads, checked through size-independent properties.

C4: 96^3 27-point stencil, lognormal(0, 2) edge weights (high contrast),
diagonal 1.05 x the row's absolute off-diagonal sum, 16 right-hand sides:
FP32 tensor-core fronts with FP64 refinement must reach a backward error
<= 1e-10 in every column (falling back to FP64 factors only if refinement
stagnates), checked on the host against the original CSR.
"""
import time

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import rel_resid


@pytest.mark.gpu
def test_c4_27pt96_fp32_ir(gpu):
    rp, ci, v, B = generators.config("c4_27pt96")
    t0 = time.perf_counter()
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    t1 = time.perf_counter()
    X = s.factorize().solve(B)
    st = s.stats()
    worst = max(rel_resid(rp, ci, v, X[:, r], B[:, r]) for r in range(B.shape[1]))
    print(f"c4: n={len(rp) - 1} nnz={len(ci)} construct {t1 - t0:.1f}s "
          f"factor {st['factor_s'] * 1e3:.1f}ms solve {st['solve_s'] * 1e3:.1f}ms "
          f"({st['factor_flops'] * 1e-12:.2f} TFLOP, "
          f"{st['factor_flops'] / st['factor_s'] * 1e-12:.1f} TFLOP/s) ir {st['ir_iters']} "
          f"fallback {st['fp64_fallback']} backward error {worst:.2e} "
          f"device {st['device_bytes'] / 1e9:.1f} GB")
    assert worst <= 1e-10
