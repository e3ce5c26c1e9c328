"""Bit-exact host structure against the reference (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref, and live runs of oracle/_ref
when it is present)."""
import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import REF_BIN, golden


def _structure(h, np_):
    order, sizes = h.ordering()
    bs, bz = h.blocks()
    pm, cr, cc = h.coo()
    out = dict(order=order, sizes=sizes, block_start=bs, block_size=bz,
               perm_map=pm, coo_r=cr, coo_c=cc)
    for r in range(np_):
        info = h.leaf_info(r)
        pat = h.leaf_pattern(r)
        out[f"r{r}_meta"] = np.array([info["leaf"], info["leaf_size"],
                                      info["dense_row"], info["core_n"],
                                      info["core_nnz"],
                                      h.leaf_info(r)["LU_nnz"]], np.int32)
        for k, v in pat.items():
            out[f"r{r}_{k}"] = v
    return out


def _digest(a):
    return np.frombuffer(bytes.fromhex(hashlib.sha256(
        np.ascontiguousarray(a).tobytes()).hexdigest()), np.uint8)


def _compare(g, mine, np_, hashed):
    for name in ("order", "sizes", "perm_map", "coo_r", "coo_c"):
        ref = g[name]
        got = _digest(mine[name]) if hashed else mine[name]
        np.testing.assert_array_equal(got, ref, err_msg=name)
    # block arrays: entry 0 is unused by the reference
    for name in ("block_start", "block_size"):
        ref = g[name]
        got = mine[name]
        if hashed:
            got = got.copy()
            got[0] = 0
            # the reference leaves entry 0 uninitialised; compare 1..
            continue
        np.testing.assert_array_equal(got[1:], ref[1:], err_msg=name)
    for r in range(np_):
        np.testing.assert_array_equal(mine[f"r{r}_meta"], g[f"r{r}_meta"][:6],
                                      err_msg=f"rank {r} meta")
        for name in ("LU_rowptr", "LU_colidx", "LU_diag", "LU_bias", "core_map"):
            got = mine[f"r{r}_{name}"]
            got = _digest(got) if hashed else got
            np.testing.assert_array_equal(got, g[f"r{r}_{name}"],
                                          err_msg=f"rank {r} {name}")


@pytest.mark.parametrize("np_", [4, 8])
def test_matrix20_structure_bitexact(np_):
    g = golden(f"matrix20_np{np_}.npz")
    h = snu.Solver(nleaves=np_).analyze(g["rowptr"], g["colidx"])
    _compare(g, _structure(h, np_), np_, hashed=False)


def test_c1_structure_bitexact():
    g = golden("c1_2d128_np8.npz")
    rp, ci, v, _ = generators.config("c1_2d128")
    h = snu.Solver(nleaves=8).analyze(rp, ci)
    _compare(g, _structure(h, 8), 8, hashed=True)


def test_c2_structure_bitexact():
    # the 64^3 convection-diffusion workload: ordering, block layout, COO
    # split and every leaf's LU pattern against the reference's own run
    g = golden("c2_convdiff64_np8.npz")
    rp, ci, v, _ = generators.config("c2_convdiff64")
    h = snu.Solver(nleaves=8).analyze(rp, ci)
    _compare(g, _structure(h, 8), 8, hashed=True)


def test_c4_ordering_bitexact():
    # the 96^3 27-point workload: the reference's ordering call (METIS
    # nested dissection through its ParMETIS driver) gives the same order and
    # separator sizes as this library's analysis
    g = golden("c4_27pt96_np8_order.npz")
    rp, ci, v, _ = generators.config("c4_27pt96")
    h = snu.Solver(nleaves=8).analyze(rp, ci)
    order, sizes = h.ordering()
    np.testing.assert_array_equal(sizes, g["sizes"])
    np.testing.assert_array_equal(_digest(order), g["order"])


def test_read_mtx_matches_reference_csr(tmp_path):
    g = golden("matrix20_np4.npz")
    p = tmp_path / "m.mtx"
    # write the fixture in column order (like data/matrix_20.mtx) and read back
    rows = np.repeat(np.arange(20), np.diff(g["rowptr"]))
    order = np.lexsort((rows, g["colidx"]))
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n20 20 65\n")
        for k in order:
            f.write(f"{rows[k] + 1} {g['colidx'][k] + 1} {float(g['vals'][k])!r}\n")
    A = snu.read_matrix(str(p))
    np.testing.assert_array_equal(A.rowptr, g["rowptr"])
    np.testing.assert_array_equal(A.colidx, g["colidx"])
    np.testing.assert_array_equal(A.data, g["vals"])


def _random_matrix(rng, nx, ny, extra, dup=0):
    rp, ci, v = generators.laplace2d_perturbed(nx, ny, seed=int(rng.integers(1 << 30)))
    n = nx * ny
    rows = list(np.repeat(np.arange(n), np.diff(rp)))
    cols = list(ci)
    vals = list(v)
    # structurally unsymmetric extras between grid neighbours at distance 2
    for _ in range(extra):
        r = int(rng.integers(n))
        c = min(n - 1, r + 2)
        if c != r:
            rows.append(r), cols.append(c), vals.append(float(rng.normal()))
    for _ in range(dup):
        k = int(rng.integers(len(rows)))
        rows.append(rows[k]), cols.append(cols[k]), vals.append(0.5)
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    o = np.argsort(rows, kind="stable")
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols[o].astype(np.int32), vals[o]


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="oracle/_ref not built")
@pytest.mark.parametrize("np_,nx,ny,extra,dup", [(2, 9, 7, 5, 0), (4, 12, 11, 20, 0),
                                                 (8, 16, 13, 30, 3), (16, 24, 20, 40, 0)])
def test_structure_live_against_reference(np_, nx, ny, extra, dup, tmp_path):
    rng = np.random.default_rng(np_ * 1000 + nx)
    rp, ci, v = _random_matrix(rng, nx, ny, extra, dup)
    mtx = tmp_path / "a.mtx"
    generators.write_mtx(str(mtx), rp, ci, v)
    d = tmp_path / "dump"
    d.mkdir()
    env = dict(os.environ, SNU_MPI_NP=str(np_), CUDA_VISIBLE_DEVICES="",
               OPENBLAS_NUM_THREADS="1")
    subprocess.run([REF_BIN, str(mtx), "--dump", str(d)], env=env, check=True,
                   capture_output=True, timeout=120)

    def ld(name, r=0):
        return np.fromfile(f"{d}/r{r}_{name}.i32.bin", np.int32)

    g = {k: ld(k) for k in ("order", "sizes", "block_start", "block_size",
                            "perm_map", "coo_r", "coo_c")}
    for r in range(np_):
        g[f"r{r}_meta"] = ld("meta", r)
        for k in ("LU_rowptr", "LU_colidx", "LU_diag", "LU_bias", "core_map"):
            g[f"r{r}_{k}"] = ld(k, r)
    h = snu.Solver(nleaves=np_).analyze(rp, ci)
    _compare(g, _structure(h, np_), np_, hashed=False)
