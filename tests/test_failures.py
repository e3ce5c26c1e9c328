"""Failure detection: errors come back as status codes, never as a fault.

Host-made failures only (a singular matrix, a memory budget that is too
small, calls out of order) plus the library's own bounded-wait self-test,
which waits on a flag nothing sets and must report SNU_ETIMEOUT with the
device still usable afterwards.  Nothing here traps, faults or hangs a GPU.
"""
import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators


@pytest.mark.gpu
def test_bounded_wait_reports_timeout_and_device_stays_usable(gpu):
    lib = snu.load_library()
    lib.snu_selftest_wait_timeout.restype = int
    st = lib.snu_selftest_wait_timeout(0)
    assert st == 4, snu.STATUS.get(st)  # SNU_ETIMEOUT
    # the context is intact: a normal solve still works
    rp, ci, v = generators.laplace2d_perturbed(20, 20, seed=1)
    b = np.ones(400)
    x = snu.Solver(nleaves=4).construct(rp, ci, v).factorize().solve(b)
    assert np.isfinite(x).all()


@pytest.mark.gpu
def test_zero_separator_pivot_is_singular(gpu):
    # zero the row and column of one vertex of the top separator: its pivot
    # stays exactly zero (no update reaches it) and separator pivots are not
    # guarded -- like getrf without pivoting in the reference
    rp, ci, v = generators.laplace2d_perturbed(24, 24, seed=3)
    n = len(rp) - 1
    s0 = snu.Solver(nleaves=4).analyze(rp, ci)
    order, sizes = s0.ordering()
    start, size = s0.blocks()
    top = start[1]  # block 1: the top separator, in the new numbering
    assert size[1] > 0
    x = int(np.nonzero(order == top)[0][0])
    rows = np.repeat(np.arange(n), np.diff(rp))
    v = v.copy()
    v[(rows == x) | (ci == x)] = 0.0
    s = snu.Solver(nleaves=4).construct(rp, ci, v)
    with pytest.raises(snu.SnuError) as e:
        s.factorize()
    assert e.value.status == 3  # SNU_ESINGULAR
    with pytest.raises(snu.SnuError) as e2:
        s.solve(np.ones(n))
    assert e2.value.status == 6  # SNU_ESTATE: no factors to solve with


@pytest.mark.gpu
def test_memory_budget_refused_cleanly(gpu):
    rp, ci, v = generators.convdiff3d(16)
    s = snu.Solver(nleaves=8, mem_budget=1 << 20)  # 1 MiB: far too small
    with pytest.raises(snu.SnuError) as e:
        s.construct(rp, ci, v).factorize()
    assert e.value.status == 2  # SNU_ENOMEM
    # a fresh handle with room works
    s2 = snu.Solver(nleaves=8).construct(rp, ci, v).factorize()
    assert np.isfinite(s2.solve(np.ones(len(rp) - 1))).all()
