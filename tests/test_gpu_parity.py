"""GPU numeric path against the reference numerics.

FP64 path: factors within 1e-10 of the reference's (normwise per array:
max |F - F_ref| <= 1e-10 * max |F_ref|), solution within 1e-10 relative,
relative residual <= 1e-12.  FP32+IR path: relative residual <= 1e-10.
The references are the golden fixtures (made by oracle/_ref, the reference
built from its sources) and the C restatement oracle/snu_oracle.c run live.
"""
import ctypes as C

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import (dense_block_array, free_blocks, golden, oracle_solve,
                  rel_resid)

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-10
X_TOL = 1e-10


def _close(got, ref, tol, what):
    scale = max(np.abs(ref).max() if ref.size else 0.0, 1e-300)
    err = np.abs(got - ref).max() / scale if ref.size else 0.0
    assert err <= tol, f"{what}: relative error {err:.3e} > {tol}"


@pytest.mark.parametrize("np_", [4, 8])
def test_matrix20_factors_and_solution(gpu, np_):
    g = golden(f"matrix20_np{np_}.npz")
    s = snu.Solver(nleaves=np_).construct(g["rowptr"], g["colidx"], g["vals"])
    s.factorize()
    x = s.solve(g["b"])
    _close(x, g["x"], X_TOL, "x")
    for r in range(np_):
        _close(s.leaf_factor(r), g[f"r{r}_LU_data"], FACTOR_TOL, f"leaf {r}")
    bz = g["block_size"]
    for key in g:
        if key.startswith("dense_"):
            i, j = map(int, key.split("_")[1:3])
            if bz[i] * bz[j] == 0:
                continue
            ref = g[key].reshape((bz[i], bz[j]), order="F")
            _close(s.dense_block(i, j), ref, FACTOR_TOL, f"LU[{i},{j}]")


def test_c1_against_golden_and_oracle(gpu):
    g = golden("c1_2d128_np8.npz")
    rp, ci, v, B = generators.config("c1_2d128")
    s = snu.Solver(nleaves=8).construct(rp, ci, v)
    s.factorize()
    x = s.solve(B[:, 0])
    _close(x, g["x"], X_TOL, "x vs reference")
    assert rel_resid(rp, ci, v, x, B[:, 0]) <= 1e-12
    order, sizes = s.ordering()
    xo, lus, blocks, lib = oracle_solve(rp, ci, v, B[:, 0], 8, order, sizes)
    try:
        _close(x, xo, X_TOL, "x vs oracle")
        for r in range(8):
            lu = s.leaf_factor(r)
            _close(lu, lus[r], FACTOR_TOL, f"leaf {r}")
            idx = g[f"r{r}_LU_data_idx"]
            _close(lu[idx], g[f"r{r}_LU_data_val"], FACTOR_TOL, f"leaf {r} golden")
        _, bz = s.blocks()
        for (i, j), p in blocks.items():
            if bz[i] * bz[j] == 0:
                continue
            ref = dense_block_array(lib, p, bz[i], bz[j])
            _close(s.dense_block(i, j), ref, FACTOR_TOL, f"LU[{i},{j}]")
    finally:
        free_blocks(lib, blocks)


def _random_unsym(rng, nx, ny, extra):
    rp, ci, v = generators.laplace2d_perturbed(nx, ny, seed=int(rng.integers(1 << 30)))
    n = nx * ny
    rows = list(np.repeat(np.arange(n), np.diff(rp)))
    cols, vals = list(ci), list(v)
    seen = set(zip(rows, cols))
    for _ in range(extra):
        r = int(rng.integers(n))
        c = int(min(n - 1, r + int(rng.integers(2, 4))))
        if (r, c) not in seen:
            seen.add((r, c))
            rows.append(r), cols.append(c), vals.append(0.3 * float(rng.normal()))
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    o = np.lexsort((cols, rows))
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols[o].astype(np.int32), vals[o]


@pytest.mark.parametrize("np_,nx,ny,extra", [(2, 20, 17, 30), (4, 33, 30, 80),
                                             (16, 48, 41, 150), (32, 70, 64, 100)])
def test_random_unsymmetric_against_oracle(gpu, np_, nx, ny, extra):
    rng = np.random.default_rng(7 * np_ + nx)
    rp, ci, v = _random_unsym(rng, nx, ny, extra)
    b = rng.uniform(-1, 1, len(rp) - 1)
    s = snu.Solver(nleaves=np_).construct(rp, ci, v)
    s.factorize()
    x = s.solve(b)
    order, sizes = s.ordering()
    xo, lus, blocks, lib = oracle_solve(rp, ci, v, b, np_, order, sizes)
    try:
        _close(x, xo, X_TOL, "x")
        for r in range(np_):
            _close(s.leaf_factor(r), lus[r], FACTOR_TOL, f"leaf {r}")
    finally:
        free_blocks(lib, blocks)
    assert rel_resid(rp, ci, v, x, b) <= 1e-12


def test_static_pivot_matches_oracle(gpu):
    # a leaf pivot that is exactly zero gets +eps, as in kernel_sparse.cu:742-749
    rp, ci, v = generators.laplace2d_perturbed(12, 12, seed=5)
    n = 144
    rows = np.repeat(np.arange(n), np.diff(rp))
    v = v.copy()
    s0 = snu.Solver(nleaves=2).analyze(rp, ci)
    order, sizes = s0.ordering()
    first = int(np.argmin(order))  # original row eliminated first
    v[(rows == first) & (ci == first)] = 0.0
    b = np.ones(n)
    s = snu.Solver(nleaves=2).construct(rp, ci, v)
    s.factorize()
    assert s.stats()["tiny_pivots"] >= 1
    xo, lus, blocks, lib = oracle_solve(rp, ci, v, b, 2, order, sizes)
    try:
        for r in range(2):
            _close(s.leaf_factor(r), lus[r], FACTOR_TOL, f"leaf {r}")
    finally:
        free_blocks(lib, blocks)


def test_multiple_rhs_and_refactor(gpu):
    rp, ci, v = generators.laplace2d_perturbed(64, 64, seed=11)
    n = len(rp) - 1
    B = generators.rhs(n, 5, seed=12)
    s = snu.Solver(nleaves=8).construct(rp, ci, v)
    s.factorize()
    X = s.solve(B)
    for r in range(5):
        assert rel_resid(rp, ci, v, X[:, r], B[:, r]) <= 1e-12
        _close(X[:, r], s.solve(B[:, r]), 1e-13, "column solve")
    rng = np.random.default_rng(13)
    v2 = v * rng.uniform(0.5, 2.0, len(v))
    s.refactor(v2)
    X2 = s.solve(B)
    fresh = snu.Solver(nleaves=8).construct(rp, ci, v2).factorize()
    # sibling fronts add their updates into a parent with atomics, so two
    # factorizations of the same values agree to rounding, not bit for bit
    _close(X2, fresh.solve(B), 1e-11, "refactor vs fresh")
    for r in range(5):
        assert rel_resid(rp, ci, v2, X2[:, r], B[:, r]) <= 1e-12


def test_fp32_ir_reaches_tolerance(gpu):
    rp, ci, v, B = generators.config("c1_2d128")
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    s.factorize()
    x = s.solve(B[:, 0])
    st = s.stats()
    assert st["backward_error"] <= 1e-10
    # FP32 factors accurate to FP32 level: refinement converges in a few
    # steps and never needs the FP64 fallback
    assert st["fp64_fallback"] == 0 and st["ir_iters"] <= 3, st
    assert rel_resid(rp, ci, v, x, B[:, 0]) <= 1e-10
    ref = snu.Solver(nleaves=8).construct(rp, ci, v).factorize().solve(B[:, 0])
    fwd = np.abs(x - ref).max() / np.abs(ref).max()
    assert fwd <= 1e-8, fwd


def test_fp32_ir_3d(gpu):
    # 3D fronts are large enough for the tensor-core GEMM path
    rp, ci, v = generators.convdiff3d(24)
    n = len(rp) - 1
    B = generators.rhs(n, 2, seed=9)
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    X = s.factorize().solve(B)
    st = s.stats()
    assert st["fp64_fallback"] == 0 and st["ir_iters"] <= 3, st
    for r in range(2):
        assert rel_resid(rp, ci, v, X[:, r], B[:, r]) <= 1e-10


def test_solve_device_pointers(gpu):
    import torch
    rp, ci, v = generators.laplace2d_perturbed(40, 40, seed=2)
    n = len(rp) - 1
    B = generators.rhs(n, 3, seed=4)
    s = snu.Solver(nleaves=4).construct(rp, ci, v).factorize()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()  # column-major
    dX = torch.empty_like(dB)
    s.solve_device(dB.data_ptr(), dX.data_ptr(), 3, n)
    torch.cuda.synchronize()
    X = dX.cpu().numpy().T
    _close(X, s.solve(B), 1e-14, "device vs host solve")


def test_autotuned_factorization_matches(gpu, tmp_path):
    # the autotuner times the tensor-core GEMM variants per batch (one CTA
    # per tile or persistent, tile width 128 or 64), keeps the fastest and
    # records the choice; results stay those of the default
    rp, ci, v = generators.convdiff3d(20)
    n = len(rp) - 1
    B = generators.rhs(n, 2, seed=3)
    cache = tmp_path / "tune.txt"
    ref = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    Xr = ref.factorize().solve(B)
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    s.set_autotune(True, str(cache))
    X = s.factorize().solve(B)
    lines = cache.read_text().split()
    assert len(lines) == 2 and set(lines[1]) <= set("01234567")
    for r in range(2):
        assert rel_resid(rp, ci, v, X[:, r], B[:, r]) <= 1e-10
    assert np.abs(X - Xr).max() <= 1e-8 * np.abs(Xr).max()
    # a second handle on the same pattern reads the cache (no new line)
    s2 = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    s2.set_autotune(True, str(cache))
    s2.factorize()
    assert cache.read_text().split() == lines


@pytest.mark.parametrize("env", [("SNU_PANEL_BLOCK", "0"), ("SNU_TC_GEMM", "0"),
                                 ("SNU_TC_PERSIST", "1"), ("SNU_TC_PERSIST", "0"),
                                 ("SNU_GRAPHS", "0"), ("SNU_TC_PANEL", "0"),
                                 ("SNU_TC_PANEL", "1"), ("SNU_SOLVE_FUSED", "1"),
                                 ("SNU_SOLVE_FUSED", "0"),
                                 ("SNU_TC_WIDTH", "64"), ("SNU_DMMA", "0"),
                                 ("SNU_SPLIT", "tf32"), ("SNU_SPLIT", "bf16"),
                                 ("SNU_DETERMINISTIC", "1")])
def test_alternative_paths_match(gpu, monkeypatch, env):
    # the paths behind the engine switches (read when an engine is made):
    # per-step panels instead of the fused outer-block kernel, SIMT instead
    # of tensor-core FP32 GEMMs, the persistent GEMM forced on or off, no
    # CUDA graph, the FP32 panel products on the tensor cores for no level
    # or for every level, the whole-tree solve sweeps instead of the
    # level-by-level ones, 64-wide tensor-core tiles, SIMT FP64 GEMMs
    # instead of mma.sync f64, every batch TF32x3 or BF16x3, the
    # fixed-order (bit-reproducible) reductions -- each must reproduce the
    # oracle like the default
    monkeypatch.setenv(*env)
    rng = np.random.default_rng(41)
    rp, ci, v = _random_unsym(rng, 33, 30, 80)
    b = rng.uniform(-1, 1, len(rp) - 1)
    s = snu.Solver(nleaves=4).construct(rp, ci, v)
    x = s.factorize().solve(b)
    order, sizes = s.ordering()
    xo, lus, blocks, lib = oracle_solve(rp, ci, v, b, 4, order, sizes)
    try:
        _close(x, xo, X_TOL, "x")
        for r in range(4):
            _close(s.leaf_factor(r), lus[r], FACTOR_TOL, f"leaf {r}")
    finally:
        free_blocks(lib, blocks)
    # FP32 fronts large enough for the tensor-core GEMMs and several outer
    # blocks per separator front
    rp, ci, v = generators.convdiff3d(24)
    B = generators.rhs(len(rp) - 1, 2, seed=9)
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    X = s.factorize().solve(B)
    st = s.stats()
    assert st["fp64_fallback"] == 0 and st["ir_iters"] <= 3, st
    for r in range(2):
        assert rel_resid(rp, ci, v, X[:, r], B[:, r]) <= 1e-10


def test_construct_reuses_analysis_and_plan(gpu):
    # analyze + plan, then construct of the same pattern: the plan is kept
    # (same fronts) and the solve matches a fresh handle's
    rp, ci, v = generators.laplace2d_perturbed(48, 40, seed=3)
    b = generators.rhs(len(rp) - 1, 1, seed=4)[:, 0]
    s = snu.Solver(nleaves=4).analyze(rp, ci).plan()
    planned = s.stats()["nfronts"]
    x = s.construct(rp, ci, v).factorize().solve(b)
    assert s.stats()["nfronts"] == planned
    ref = snu.Solver(nleaves=4).construct(rp, ci, v).factorize().solve(b)
    _close(x, ref, 1e-11, "reused plan vs fresh")  # atomics: rounding order
    assert rel_resid(rp, ci, v, x, b) <= 1e-12


def _sampled(got, g, key, tol, what):
    """got (flat, the reference's layout) against a golden sample of the
    reference's array: max |got[k] - ref[k]| <= tol * max |ref|."""
    idx, val = g[key + "_idx"], g[key + "_val"]
    scale = max(float(g[key + "_absmax"][0]), 1e-300)
    err = np.abs(got[idx] - val).max() / scale if len(idx) else 0.0
    assert err <= tol, f"{what}: relative error {err:.3e} > {tol}"
    return err


def test_c2_against_reference(gpu):
    # the 64^3 convection-diffusion workload against the reference's own
    # FP64 run (built from its sources, 8 ranks, the first right-hand side):
    # sampled leaf and separator factors and the solution within 1e-10, and
    # the FP32+IR solution's forward error against that same reference x
    g = golden("c2_convdiff64_np8.npz")
    rp, ci, v, B = generators.config("c2_convdiff64")
    s = snu.Solver(nleaves=8).construct(rp, ci, v).factorize()
    x = s.solve(B[:, 0])
    _sampled(x, g, "x", X_TOL, "x vs reference")
    assert rel_resid(rp, ci, v, x, B[:, 0]) <= 1e-12
    for r in range(8):
        _sampled(s.leaf_factor(r), g, f"r{r}_LU_data", FACTOR_TOL, f"leaf {r}")
    for key in g:
        if key.startswith("dense_") and key.endswith("_idx"):
            i, j = map(int, key.split("_")[1:3])
            _sampled(s.dense_block(i, j).ravel(order="F"), g, f"dense_{i}_{j}",
                     FACTOR_TOL, f"LU[{i},{j}]")
    s.close()
    s32 = snu.Solver(nleaves=8, precision=snu.FP32_IR).construct(rp, ci, v)
    x32 = s32.factorize().solve(B[:, 0])
    st = s32.stats()
    assert st["backward_error"] <= 1e-10 and st["fp64_fallback"] == 0, st
    fwd = _sampled(x32, g, "x", 1e-8, "FP32+IR x vs reference")
    assert fwd <= 1e-8


def test_fp64_fallback_when_refinement_stops(gpu):
    # no refinement step allowed: the FP32+IR solve must factor in FP64 on
    # demand, solve the correction with it and reach FP64 accuracy
    g = golden("c1_2d128_np8.npz")
    rp, ci, v, B = generators.config("c1_2d128")
    s = snu.Solver(nleaves=8, precision=snu.FP32_IR,
                   ir_max_iter=0).construct(rp, ci, v)
    x = s.factorize().solve(B[:, 0])
    st = s.stats()
    # (no front of this Laplacian stands out: the whole matrix in FP64, one
    # FP64 correction step)
    assert st["fp64_fallback"] == 1 and st["ir_iters"] == 1, st
    assert st["fp64_fronts"] == st["nfronts"], st
    assert st["backward_error"] <= 1e-12, st
    _close(x, g["x"], X_TOL, "x vs reference")
    assert rel_resid(rp, ci, v, x, B[:, 0]) <= 1e-12
    # a second solve reuses the FP64 factors
    x2 = s.solve(B[:, 0])
    assert s.stats()["fp64_fallback"] == 1
    _close(x2, x, 1e-11, "second solve")


def _plant_tiny_pivot(nx, block, delta, nleaves=4):
    """A perturbed nx^2 Laplacian whose separator front of heap block
    `block` gets a first pivot of `delta` in exact elimination: the FP64
    pivot value (host restatement of the front numerics) is shifted away
    through the matching diagonal entry."""
    from host_engine import HostEngine
    rp, ci, v = generators.laplace2d_perturbed(nx, nx, seed=21)
    v = np.array(v, dtype=np.float64)
    he = HostEngine(None, 1, nleaves=nleaves)
    he.construct(rp, ci, v)
    he.factor_phase(0)
    fp = he.fp
    f = [k for k in range(len(fp["p"]))
         if fp["block"][k] == block and fp["p"][k] > 0][0]
    u0 = he._front(f)[0, 0]
    r = he._gidx(f)[0]
    k = [j for j in range(rp[r], rp[r + 1]) if ci[j] == r][0]
    v[k] += delta - u0
    return rp, ci, v


@pytest.mark.parametrize("block,expect", [(1, 1), (2, 2)])
def test_fp64_refactor_of_the_fronts_that_stall_refinement(gpu, block, expect):
    # a pivot of 1e-6 planted in one separator front: no-pivot elimination
    # lets multipliers of ~1e6 through there, FP32 refinement falls short
    # (one step allowed), and the solve refactors that front and its
    # ancestors in FP64 (`expect` fronts), keeps the FP32 factors of the
    # rest and refines with FP64 solves over the mixed factors
    rp, ci, v = _plant_tiny_pivot(48, block, 1e-6)
    n = len(rp) - 1
    b = generators.rhs(n, 1, seed=5)[:, 0]
    s = snu.Solver(nleaves=4, precision=snu.FP32_IR,
                   ir_max_iter=1).construct(rp, ci, v)
    x = s.factorize().solve(b)
    st = s.stats()
    assert st["fp64_fallback"] == 1 and st["fp64_fronts"] == expect, st
    assert st["backward_error"] <= 1e-10, st
    assert rel_resid(rp, ci, v, x, b) <= 1e-10
    x64 = snu.Solver(nleaves=4).construct(rp, ci, v).factorize().solve(b)
    assert np.abs(x - x64).max() <= 1e-6 * np.abs(x64).max()
    # a second solve reuses the mixed factors; a refactor drops them
    x2 = s.solve(b)
    assert s.stats()["fp64_fronts"] == expect
    assert np.abs(x2 - x).max() <= 1e-9 * np.abs(x).max()
    s.refactor(v)
    x3 = s.solve(b)
    assert s.stats()["fp64_fronts"] == expect
    assert rel_resid(rp, ci, v, x3, b) <= 1e-10
    # fp64_growth 0: the whole matrix in FP64
    s0 = snu.Solver(nleaves=4, precision=snu.FP32_IR, ir_max_iter=1,
                    fp64_growth=0).construct(rp, ci, v)
    s0.factorize().solve(b)
    st0 = s0.stats()
    assert st0["fp64_fronts"] == st0["nfronts"], st0
    assert st0["backward_error"] <= 1e-10, st0


@pytest.mark.parametrize("precision", [snu.FP64, snu.FP32_IR])
def test_deterministic_mode_is_bit_reproducible(gpu, monkeypatch, precision):
    # SNU_DETERMINISTIC=1: sibling updates enter their parent in a fixed
    # order and the solve's products have one writer per row, so two
    # handles (and two factorizations of one handle) give identical bits
    monkeypatch.setenv("SNU_DETERMINISTIC", "1")
    rng = np.random.default_rng(43)
    cases = [_random_unsym(rng, 40, 37, 90), generators.convdiff3d(20)]
    for rp, ci, v in cases:
        n = len(rp) - 1
        B = generators.rhs(n, 3, seed=12)
        runs = []
        for _ in range(2):
            s = snu.Solver(nleaves=8, precision=precision).construct(rp, ci, v)
            X1 = s.factorize().solve(B)
            X2 = s.factorize().solve(B)
            assert np.array_equal(X1, X2)
            runs.append(X1)
            for r in range(3):
                assert rel_resid(rp, ci, v, X1[:, r], B[:, r]) <= 1e-10
        assert np.array_equal(runs[0], runs[1])


@pytest.mark.parametrize("precision,tol,res", [(snu.FP64, 1e-12, 1e-12),
                                               (snu.FP32_IR, 1e-9, 1e-10)])
def test_wide_solve_passes_and_host_copies(gpu, precision, tol, res):
    # 70 columns through the host API: one pass of 64 columns (the sweeps
    # run four register groups per staged tile, W rows in global memory)
    # and one of 6, the columns crossing the pinned ring's 1 Mi-element
    # slots mid-column; every column equals its own single-column solve
    rp, ci, v = generators.laplace2d_perturbed(200, 200, seed=31)
    n = len(rp) - 1
    B = generators.rhs(n, 70, seed=32)
    s = snu.Solver(nleaves=8, precision=precision).construct(rp, ci, v)
    X = s.factorize().solve(B)
    assert s.stats()["backward_error"] <= res
    for c in (0, 15, 16, 40, 63, 64, 69):
        x1 = s.solve(B[:, c])
        err = np.abs(X[:, c] - x1).max() / np.abs(x1).max()
        assert err <= tol, (c, err)
        assert rel_resid(rp, ci, v, X[:, c], B[:, c]) <= res
    # the device API, 40 columns in one pass, equals the host API's result
    import torch
    dB = torch.from_numpy(np.ascontiguousarray(B[:, :40].T)).cuda()
    dX = torch.empty_like(dB)
    s.solve_device(dB.data_ptr(), dX.data_ptr(), 40, n)
    torch.cuda.synchronize()
    Xd = dX.cpu().numpy().T
    assert np.abs(Xd - X[:, :40]).max() <= tol * np.abs(X[:, :40]).max()


def test_pivot_reciprocal_against_correctly_rounded(gpu):
    # the FP32 tile factorization's pivot reciprocal (hardware approximation
    # + one Newton-Raphson step) against CUDA's correctly rounded reciprocal
    lib = C.CDLL(snu.library_path())
    f = lib.snu_selftest_pivot_reciprocal
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int64, C.c_uint64, C.POINTER(C.c_int),
                  C.POINTER(C.c_int64)]
    n = 1 << 24
    mx, nd = C.c_int(-1), C.c_int64(-1)
    assert f(0, n, 11, C.byref(mx), C.byref(nd)) == 0
    assert 0 <= mx.value <= 1, (mx.value, nd.value)  # within one ulp
    assert 0 <= nd.value <= n // 10000, nd.value    # nearly always equal
