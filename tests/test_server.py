"""Request server (snu_server_*): continuous batching on one GPU.

The serving contract: requests admitted while others run overlap on the
device, and every result is the same alone and in the mix within the stated
tolerance (FP32 factors + FP64 refinement: backward error <= 1e-10 and
solutions within 1e-7 relative (max norm) of the same request run alone;
the factors are bitwise the same, the solve's atomic accumulations may
round differently, and refinement bounds what is left by the condition
number times 1e-10).  Memory
admission, plan reuse and request ordering per matrix are checked too.
"""
import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from snusolver_b200.server import Server
from util import rel_resid

# Both runs of a request refine to backward error <= 1e-10 from factors
# that differ in rounding (sibling updates add with atomics in a different
# order), so their solutions agree to about cond(A) x 1e-10; these
# Laplacians have infinity-norm condition numbers of a few thousand.
MIX_TOL = 1e-6


def _mats():
    out = []
    for k, (nx, ny) in enumerate([(48, 40), (64, 64), (30, 90)]):
        out.append(generators.laplace2d_perturbed(nx, ny, seed=40 + k))
    out.append(generators.convdiff3d(14))
    out.append(generators.laplace2d_lognormal(50, 45, seed=7))
    return out


def test_server_needs_a_gpu_or_reports_it():
    # without a CUDA device creation fails with SNU_ECUDA, never silently
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(snu.SnuError) as e:
        Server(slots=2)
    assert e.value.status == 5


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(gpu):
    mats = _mats()
    rng = np.random.default_rng(50)
    work = []  # (matrix index, scale or None, nrhs)
    for i in range(len(mats)):
        work.append((i, None, int(rng.integers(1, 9))))
    for i in range(len(mats)):
        work.append((i, rng.uniform(0.5, 2.0, len(mats[i][1])), 0))
        work.append((i, None, int(rng.integers(1, 17))))
    Bs = {j: generators.rhs(len(mats[w[0]][0]) - 1, w[2], seed=60 + j)
          for j, w in enumerate(work) if w[2]}

    def run(slots, interleave):
        out = {}
        with Server(slots=slots) as s:
            ids = {}
            for i, (rp, ci, v) in enumerate(mats):
                ids[i], _ = s.factor(rp, ci, v)
                if not interleave:
                    s.drain()
            for j, (i, scale, nrhs) in enumerate(work):
                if scale is not None:
                    s.refactor(ids[i], mats[i][2] * scale)
                elif nrhs:
                    _, X = s.solve(ids[i], Bs[j])
                    out[j] = X
                if not interleave:
                    s.drain()
            comps = s.drain()
        assert all(c["status"] == 0 for c in comps), comps
        return out, comps

    alone, _ = run(1, False)
    mixed, comps = run(4, True)
    assert any(c["queue_s"] > 0 for c in comps)
    for j, X in alone.items():
        i, _, nrhs = work[j]
        rp, ci, v = mats[i]
        # values in force: the last refactor before request j
        for jj in range(j):
            if work[jj][0] == i and work[jj][1] is not None:
                v = mats[i][2] * work[jj][1]
        for r in range(nrhs):
            assert rel_resid(rp, ci, v, X[:, r], Bs[j][:, r]) <= 1e-10
        d = np.abs(mixed[j] - X).max() / np.abs(X).max()
        assert d <= MIX_TOL, f"request {j}: mix differs from alone by {d:.2e}"


@pytest.mark.gpu
def test_plan_reuse_and_order_per_matrix(gpu):
    rp, ci, v = generators.laplace2d_perturbed(56, 56, seed=3)
    n = len(rp) - 1
    b = generators.rhs(n, 2, seed=4)
    with Server(slots=3) as s:
        m1, r1 = s.factor(rp, ci, v)
        _, X1 = s.solve(m1, b)           # must wait for m1's factor
        m2, r2 = s.factor(rp, ci, 2 * v)  # same pattern: cached plan
        _, X2 = s.solve(m2, b)
        rel = s.release(m1)
        _, X3 = s.solve(m1, b)           # after the release: refused
        comps = {c["request"]: c for c in s.drain()}
        st = s.stats()
    assert comps[r1]["status"] == 0 and comps[r2]["status"] == 0
    assert comps[r2]["plan_reused"] or comps[r1]["plan_reused"]
    assert comps[rel]["status"] == 0
    bad = [c for c in comps.values() if c["type"] == "solve" and c["status"]]
    assert len(bad) == 1 and bad[0]["status"] == 6  # SNU_ESTATE
    for r in range(2):
        assert rel_resid(rp, ci, v, X1[:, r], b[:, r]) <= 1e-10
        d = np.abs(X2[:, r] - 0.5 * X1[:, r]).max() / np.abs(X1[:, r]).max()
        assert d <= 1e-7, d
    assert st["matrices"] == 1 and st["cached_plans"] >= 1


@pytest.mark.gpu
def test_memory_budget_admission(gpu):
    rp, ci, v = generators.convdiff3d(20)
    # one matrix alone: its resident bytes a, and the high-water mark e of
    # resident + admitted, which is at least the admission estimate (the
    # estimate is made on the high side, so e is the estimate)
    with Server(slots=1) as s:
        m, _ = s.factor(rp, ci, v)
        s.drain()
        st = s.stats()
        a, e = st["resident_bytes"], st["peak_bytes"]
    assert 0 < a <= e
    # room for one resident matrix and one estimate, less a byte: a second
    # matrix waits for the first one's release
    with Server(slots=2, mem_budget=a + e - 1) as s:
        ma, ra = s.factor(rp, ci, v)
        first = s.drain()
        mb, rb = s.factor(rp, ci, v)  # does not fit beside ma
        rr = s.release(ma)            # queued after it; frees the memory
        comps = {c["request"]: c for c in first + s.drain()}
        assert comps[ra]["status"] == 0 and comps[rr]["status"] == 0
        assert comps[rb]["status"] == 0
        st = s.stats()
        assert st["peak_bytes"] <= st["budget_bytes"]
        # nothing left to free: a third matrix is refused, not left waiting
        mc, rc = s.factor(rp, ci, v)
        comps = {x["request"]: x for x in s.drain()}
        assert comps[rc]["status"] == 2  # SNU_ENOMEM
