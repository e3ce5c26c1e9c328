"""Batched mode: many independent matrices as one merged level schedule.

Each matrix of a batch keeps its own ordering and front tree; the trees are
merged by level so one launch per kernel and level covers the batch.  The
batch's solutions must equal each matrix solved alone: FP64 within 1e-12
relative (same factors up to rounding order), FP32 + FP64 refinement with
per-matrix backward error <= 1e-10.
"""
import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import rel_resid


def _batch(seed, count):
    rng = np.random.default_rng(seed)
    mats = []
    for k in range(count):
        nx, ny = (int(x) for x in rng.integers(8, 48, size=2))
        mats.append(generators.laplace2d_lognormal(nx, ny, seed=seed * 100 + k))
    mats.append(generators.convdiff3d(10))
    return mats


def test_batch_host_plan_builds_without_gpu():
    # on a machine without a GPU the host half (per-matrix ordering, plans,
    # merge, validation) completes and the engine then reports SNU_ECUDA
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    s = snu.Solver(nleaves=4)
    with pytest.raises(snu.SnuError) as e:
        s.construct_batch(_batch(1, 6))
    assert e.value.status == 5


def test_batch_rejects_entries_outside_blocks():
    a = generators.laplace2d_perturbed(5, 5, seed=1)
    s = snu.Solver(nleaves=2)
    rp = np.concatenate([a[0], a[0][1:] + a[0][-1]]).astype(np.int32)
    ci = np.concatenate([a[1], a[1]]).astype(np.int32)  # 2nd block points into the 1st
    v = np.concatenate([a[2], a[2]])
    st = np.array([0, 25, 50], np.int32)
    import ctypes as C
    rc = s._lib.snu_construct_batch(s._h, 2, st.ctypes.data_as(C.POINTER(C.c_int)),
                                    50, len(ci), rp.ctypes.data_as(C.POINTER(C.c_int)),
                                    ci.ctypes.data_as(C.POINTER(C.c_int)),
                                    v.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [snu.FP64, snu.FP32_IR])
def test_batch_matches_single_solves(gpu, precision):
    mats = _batch(3, 12)
    s = snu.Solver(nleaves=4, precision=precision).construct_batch(mats)
    B = generators.rhs(s.n, 3, seed=5)
    X = s.factorize().solve(B)
    st = s.row_start
    for b, (rp, ci, v) in enumerate(mats):
        xb, bb = X[st[b]:st[b + 1]], B[st[b]:st[b + 1]]
        for r in range(3):
            assert rel_resid(rp, ci, v, xb[:, r], bb[:, r]) <= (
                1e-12 if precision == snu.FP64 else 1e-10)
        if precision == snu.FP64:
            ref = snu.Solver(nleaves=4).construct(rp, ci, v).factorize().solve(bb)
            d = np.abs(xb - ref).max() / np.abs(ref).max()
            assert d <= 1e-12, (b, d)


@pytest.mark.gpu
def test_batch_refactor(gpu):
    mats = _batch(4, 8)
    s = snu.Solver(nleaves=4, precision=snu.FP32_IR).construct_batch(mats)
    s.factorize()
    rng = np.random.default_rng(9)
    scaled = [(rp, ci, v * rng.uniform(0.5, 2.0, len(v))) for rp, ci, v in mats]
    s.refactor(np.concatenate([m[2] for m in scaled]))
    B = generators.rhs(s.n, 2, seed=6)
    X = s.solve(B)
    st = s.row_start
    for b, (rp, ci, v) in enumerate(scaled):
        for r in range(2):
            assert rel_resid(rp, ci, v, X[st[b]:st[b + 1], r],
                             B[st[b]:st[b + 1], r]) <= 1e-10


@pytest.mark.gpu
def test_c3_full_batch(gpu):
    # the full batched workload: 256 grids, sides 32..256, FP32 factors with
    # FP64 refinement; every matrix reaches backward error <= 1e-10
    mats = generators.batch_config("c3_batch256")
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct_batch(mats)
    b = generators.rhs(s.n, 1, seed=3)[:, 0]
    x = s.factorize().solve(b)
    st = s.row_start
    worst = 0.0
    for k, (rp, ci, v) in enumerate(mats):
        worst = max(worst, rel_resid(rp, ci, v, x[st[k]:st[k + 1]],
                                     b[st[k]:st[k + 1]]))
    stats = s.stats()
    print(f"c3: n={s.n} fronts={stats['nfronts']} levels={stats['nlevels']} "
          f"analyze {stats['analyze_s']:.2f}s factor {stats['factor_s']*1e3:.1f}ms "
          f"solve {stats['solve_s']*1e3:.1f}ms worst backward error {worst:.2e}")
    assert worst <= 1e-10
