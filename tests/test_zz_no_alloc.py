"""snu_solve_device_noalloc: the solve for callers that must not allocate.

Code that runs while a stream is being captured into a CUDA graph, or inside
a process whose memory manager owns the whole device, cannot call cudaMalloc;
snu_solve_device_noalloc solves with its work vectors in a static device
array instead.  These tests call it through the C-ABI and check that it
returns what snu_solve_device returns (two calls in a row, fresh right-hand
sides each time), and that it refuses work that does not fit its array.
"""
import ctypes as C

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators

pytestmark = pytest.mark.gpu


def _entry(lib):
    f = lib.snu_solve_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                  C.c_void_p]
    return f


@pytest.mark.parametrize("precision,tol,be", [(snu.FP64, 1e-12, 1e-12),
                                              (snu.FP32_IR, 1e-8, 1e-10)])
def test_noalloc_matches_solve_device(gpu, precision, tol, be):
    import torch
    rp, ci, v = generators.laplace2d_perturbed(96, 96, seed=21)
    n = len(rp) - 1
    s = snu.Solver(nleaves=8, precision=precision).construct(rp, ci, v)
    s.factorize()
    noalloc = _entry(s._lib)
    for call in range(2):
        B = generators.rhs(n, 3, seed=30 + call)
        dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
        ref = torch.empty_like(dB)
        out = torch.full_like(dB, float("nan"))
        s.solve_device(dB.data_ptr(), ref.data_ptr(), 3, n)
        torch.cuda.synchronize()
        st = noalloc(s._h, dB.data_ptr(), out.data_ptr(), 3, n, None)
        assert st == 0, s._lib.snu_last_error(s._h).decode()
        torch.cuda.synchronize()
        got, want = out.cpu().numpy(), ref.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= tol, f"call {call}: relative difference {err:.3e}"
        assert s.stats()["backward_error"] <= be


def test_noalloc_refuses_oversized_work(gpu):
    import torch
    rp, ci, v = generators.laplace2d_perturbed(96, 96, seed=21)
    n = len(rp) - 1
    s = snu.Solver(nleaves=8).construct(rp, ci, v).factorize()
    nrhs = 400  # work vectors far beyond the 32 MiB static array
    dB = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    dX = torch.zeros_like(dB)
    st = _entry(s._lib)(s._h, dB.data_ptr(), dX.data_ptr(), nrhs, n, None)
    assert st == 1  # SNU_EINVAL
    assert "bytes" in s._lib.snu_last_error(s._h).decode()
