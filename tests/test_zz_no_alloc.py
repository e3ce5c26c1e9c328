"""snu_solve_device_noalloc: the solve for callers that may not allocate.

A process whose memory manager (a framework's caching allocator, a fixed
pool) owns the device memory, or a latency-bound caller that cannot let
cudaMalloc synchronize the device, cannot have the library allocate work
vectors; snu_solve_device_noalloc solves with its work vectors in a static
device array instead.  These tests call it through the C-ABI and check that
it returns what snu_solve_device returns: two calls in a row with fresh
right-hand sides, the first of them on a handle that has never solved
before; a batch handle; more than 64 right-hand sides (the backward error
covers every column); refinement stopped early (SNU_ENOTCONV, since this
path has no FP64 fallback); and that it refuses work that does not fit its
array.
"""
import ctypes as C

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import rel_resid

pytestmark = pytest.mark.gpu


def _entry(lib):
    f = lib.snu_solve_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                  C.c_void_p]
    return f


def _err(s):
    return s._lib.snu_last_error(s._h).decode()


def _compare_two_calls(s, n, nrhs, tol, be, seed):
    """Two no-alloc solves, each before the solve_device it is checked
    against (so the first runs on a handle that has not solved yet)."""
    import torch
    noalloc = _entry(s._lib)
    for call in range(2):
        B = generators.rhs(n, nrhs, seed=seed + call)
        dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
        out = torch.full_like(dB, float("nan"))
        ref = torch.empty_like(dB)
        st = noalloc(s._h, dB.data_ptr(), out.data_ptr(), nrhs, n, None)
        assert st == 0, _err(s)
        torch.cuda.synchronize()
        got_be = s.stats()["backward_error"]
        assert s.stats()["fp64_fallback"] == 0
        assert s.stats()["solve_launches"] > 0
        s.solve_device(dB.data_ptr(), ref.data_ptr(), nrhs, n)
        torch.cuda.synchronize()
        got, want = out.cpu().numpy(), ref.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= tol, f"call {call}: relative difference {err:.3e}"
        assert got_be <= be, got_be
    return got, B


@pytest.mark.parametrize("precision,tol,be", [(snu.FP64, 1e-12, 1e-12),
                                              (snu.FP32_IR, 1e-8, 1e-10)])
def test_noalloc_matches_solve_device(gpu, precision, tol, be):
    rp, ci, v = generators.laplace2d_perturbed(96, 96, seed=21)
    n = len(rp) - 1
    s = snu.Solver(nleaves=8, precision=precision).construct(rp, ci, v)
    s.factorize()
    _compare_two_calls(s, n, 3, tol, be, seed=30)


def test_noalloc_batch_handle(gpu):
    mats = [generators.laplace2d_perturbed(40 + 8 * k, 36, seed=50 + k)
            for k in range(3)]
    s = snu.Solver(nleaves=4, precision=snu.FP32_IR).construct_batch(mats)
    s.factorize()
    X, B = _compare_two_calls(s, s.n, 2, 1e-8, 1e-10, seed=60)
    rs = s.row_start
    for k, (rp, ci, v) in enumerate(mats):
        for c in range(2):
            sl = slice(rs[k], rs[k + 1])
            assert rel_resid(rp, ci, v, X[c, sl], B[sl, c]) <= 1e-10


def test_noalloc_more_than_64_columns(gpu):
    # 80 columns, the first 64 zero (solved exactly at once): refinement
    # must go on until the last 16 columns, too, reach the tolerance
    import torch
    rp, ci, v = generators.laplace2d_perturbed(32, 32, seed=23)
    n = len(rp) - 1
    s = snu.Solver(nleaves=4, precision=snu.FP32_IR).construct(rp, ci, v)
    s.factorize()
    B = generators.rhs(n, 80, seed=70)
    B[:, :64] = 0.0
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    out = torch.empty_like(dB)
    st = _entry(s._lib)(s._h, dB.data_ptr(), out.data_ptr(), 80, n, None)
    assert st == 0, _err(s)
    torch.cuda.synchronize()
    X = out.cpu().numpy().T
    assert np.all(X[:, :64] == 0.0)
    worst = max(rel_resid(rp, ci, v, X[:, c], B[:, c]) for c in range(64, 80))
    assert worst <= 1e-10, worst
    assert s.stats()["ir_iters"] >= 1 and s.stats()["backward_error"] <= 1e-10


def test_noalloc_reports_notconv_without_fallback(gpu):
    # no refinement step allowed: the regular solve falls back to FP64
    # factors, the no-allocation solve cannot (that allocates) and says so
    import torch
    rp, ci, v = generators.laplace2d_perturbed(48, 48, seed=24)
    n = len(rp) - 1
    s = snu.Solver(nleaves=4, precision=snu.FP32_IR,
                   ir_max_iter=0).construct(rp, ci, v).factorize()
    B = generators.rhs(n, 2, seed=71)
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    out = torch.empty_like(dB)
    st = _entry(s._lib)(s._h, dB.data_ptr(), out.data_ptr(), 2, n, None)
    assert st == 7, (st, _err(s))  # SNU_ENOTCONV
    torch.cuda.synchronize()
    st_ = s.stats()
    assert st_["fp64_fallback"] == 0 and st_["backward_error"] > 1e-10
    X = out.cpu().numpy().T  # the FP32 solution is still there
    assert max(rel_resid(rp, ci, v, X[:, c], B[:, c]) for c in range(2)) <= 1e-5


def test_noalloc_refuses_oversized_work(gpu):
    import torch
    rp, ci, v = generators.laplace2d_perturbed(96, 96, seed=21)
    n = len(rp) - 1
    s = snu.Solver(nleaves=8).construct(rp, ci, v).factorize()
    nrhs = 600  # the residual alone (8 n nrhs bytes) exceeds 32 MiB
    dB = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    dX = torch.zeros_like(dB)
    st = _entry(s._lib)(s._h, dB.data_ptr(), dX.data_ptr(), nrhs, n, None)
    assert st == 1  # SNU_EINVAL
    assert "bytes" in _err(s)
