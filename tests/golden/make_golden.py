"""Generates the golden fixtures of tests/golden from the reference itself.

Runs oracle/_ref/snu_ref -- the reference SnuSolver built from its own
sources by oracle/Makefile -- on

* the reference's bundled 20x20 fixture (data/matrix_20.mtx) with 4 ranks
  (the reference's run.sh) and 8 ranks (several empty blocks), and
* the 128x128 perturbed 2D Laplacian (generators.config("c1_2d128")) with
  8 ranks and its seeded right-hand side,
* the 64^3 convection-diffusion matrix (generators.config("c2_convdiff64"))
  with 8 ranks and the first of its seeded right-hand sides, and
* the ordering alone (the reference's call_parmetis, through the harness's
  --order-only) of the 96^3 27-point matrix (generators.config(
  "c4_27pt96")) with 8 ranks,

and stores what the new implementation must reproduce: ordering, block
layout, COO split, every leaf's LU pattern / core_map / LU_bias (full arrays
for the small cases, SHA-256 digests for the 2D case), the solution x, and
the leaf and dense factor values (full for the small cases; for the 2D case a
deterministic sample plus per-array max-abs norms; for the 3D case x too is
a sample plus its max-abs norm, and for the 96^3 case only the ordering's
digest and the separator sizes are kept).

usage: python tests/golden/make_golden.py [REFERENCE_DIR]   (small cases)
       python tests/golden/make_golden.py --3d               (64^3, 96^3)
"""
import glob
import hashlib
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from snusolver_b200 import generators  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "snu_ref")


def run_ref(mtx, np_, rhs=None, extra=()):
    d = tempfile.mkdtemp(prefix="snu_golden_")
    cmd = [REF_BIN, mtx, "--dump", d] + list(extra)
    if rhs is not None:
        fn = os.path.join(d, "rhs.bin")
        np.asarray(rhs, np.float64).tofile(fn)
        cmd += ["--rhs", fn]
    env = dict(os.environ, SNU_MPI_NP=str(np_), CUDA_VISIBLE_DEVICES="",
               OPENBLAS_NUM_THREADS="1", SNU_MPI_TIMEOUT="3600")
    out = subprocess.run(cmd, env=env, check=True, capture_output=True,
                         text=True).stdout
    return d, out


def load(d, name, rank=0, dt="i32"):
    return np.fromfile(f"{d}/r{rank}_{name}.{dt}.bin",
                       np.int32 if dt == "i32" else np.float64)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def read_mtx(path):
    rows, cols, vals = [], [], []
    with open(path) as f:
        f.readline()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        n, m, nz = map(int, line.split())
        for _ in range(nz):
            r, c, v = f.readline().split()
            rows.append(int(r) - 1)
            cols.append(int(c) - 1)
            vals.append(float(v))
    # CSR in file order per row (read_matrix.cpp:6-42)
    rows = np.array(rows)
    order = np.argsort(rows, kind="stable")
    rowptr = np.zeros(n + 1, np.int32)
    np.add.at(rowptr, rows + 1, 1)
    return (np.cumsum(rowptr).astype(np.int32),
            np.array(cols, np.int32)[order], np.array(vals)[order])


def collect(d, np_, full):
    out = {}
    for name in ("order", "sizes", "block_start", "block_size", "perm_map",
                 "coo_r", "coo_c"):
        a = load(d, name)
        out[name] = a if full else np.frombuffer(bytes.fromhex(digest(a)), np.uint8)
    out["x"] = load(d, "x", dt="f64")
    out["b"] = load(d, "b", dt="f64")
    rng = np.random.default_rng(123)
    for r in range(np_):
        out[f"r{r}_meta"] = load(d, "meta", r)
        for name in ("LU_rowptr", "LU_colidx", "LU_diag", "LU_bias", "core_map"):
            a = load(d, name, r)
            out[f"r{r}_{name}"] = a if full else np.frombuffer(
                bytes.fromhex(digest(a)), np.uint8)
        lu = load(d, "LU_data", r, "f64")
        if full:
            out[f"r{r}_LU_data"] = lu
        else:
            k = np.unique(rng.integers(0, max(len(lu), 1), size=min(len(lu), 400)))
            out[f"r{r}_LU_data_idx"] = k.astype(np.int64)
            out[f"r{r}_LU_data_val"] = lu[k] if len(lu) else lu
            out[f"r{r}_LU_data_absmax"] = np.array([np.abs(lu).max() if len(lu) else 0.0])
    for f in glob.glob(f"{d}/r*_LU_*_*.f64.bin"):
        m = re.search(r"LU_(\d+)_(\d+)\.f64", f)
        i, j = int(m.group(1)), int(m.group(2))
        a = np.fromfile(f, np.float64)
        if full:
            out[f"dense_{i}_{j}"] = a
        else:
            k = np.unique(rng.integers(0, max(len(a), 1), size=min(len(a), 200)))
            out[f"dense_{i}_{j}_idx"] = k.astype(np.int64)
            out[f"dense_{i}_{j}_val"] = a[k] if len(a) else a
            out[f"dense_{i}_{j}_absmax"] = np.array([np.abs(a).max() if len(a) else 0.0])
    return out


def sample_x(res, rng, count=20000):
    """Replaces the full solution by a deterministic sample and its norm."""
    x = res.pop("x")
    res.pop("b")
    k = np.unique(rng.integers(0, len(x), size=count))
    res["x_idx"] = k.astype(np.int64)
    res["x_val"] = x[k]
    res["x_absmax"] = np.array([np.abs(x).max()])


def c2_and_c4():
    rp, ci, v, B = generators.config("c2_convdiff64")
    tmp = tempfile.mkdtemp(prefix="snu_c2_")
    mtx = os.path.join(tmp, "c2.mtx")
    generators.write_mtx(mtx, rp, ci, v)
    d, out = run_ref(mtx, 8, B[:, 0])
    res = collect(d, 8, full=False)
    sample_x(res, np.random.default_rng(456))
    res.update(np=np.array([8]),
               generator_version=np.array([generators.GENERATOR_VERSION]))
    np.savez_compressed(os.path.join(HERE, "c2_convdiff64_np8.npz"), **res)
    print("c2_convdiff64", out.strip().splitlines()[-1])
    rp, ci, v, _ = generators.config("c4_27pt96")
    tmp = tempfile.mkdtemp(prefix="snu_c4_")
    mtx = os.path.join(tmp, "c4.mtx")
    generators.write_mtx(mtx, rp, ci, v)
    d = tempfile.mkdtemp(prefix="snu_golden_")
    env = dict(os.environ, SNU_MPI_NP="8", CUDA_VISIBLE_DEVICES="",
               SNU_MPI_TIMEOUT="3600")
    out = subprocess.run([REF_BIN, mtx, "--order-only", "--summary", d],
                         env=env, check=True, capture_output=True,
                         text=True).stdout
    order = load(d, "order")
    res = {"order": np.frombuffer(bytes.fromhex(digest(order)), np.uint8),
           "sizes": load(d, "sizes"), "n": np.array([len(order)]),
           "np": np.array([8]),
           "generator_version": np.array([generators.GENERATOR_VERSION])}
    np.savez_compressed(os.path.join(HERE, "c4_27pt96_np8_order.npz"), **res)
    print("c4_27pt96", out.strip().splitlines()[-1])


def main():
    if "--3d" in sys.argv:  # the 64^3 and 96^3 fixtures only (minutes)
        c2_and_c4()
        return
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(
        os.path.dirname(ROOT), "reference")
    m20 = os.path.join(ref_dir, "data", "matrix_20.mtx")
    rp, ci, v = read_mtx(m20)
    for np_ in (4, 8):
        d, out = run_ref(m20, np_)
        res = collect(d, np_, full=True)
        res.update(rowptr=rp, colidx=ci, vals=v, np=np.array([np_]))
        np.savez_compressed(os.path.join(HERE, f"matrix20_np{np_}.npz"), **res)
        print("matrix_20", np_, out.strip().splitlines()[-1])
    rp, ci, v, B = generators.config("c1_2d128")
    tmp = tempfile.mkdtemp(prefix="snu_c1_")
    mtx = os.path.join(tmp, "c1.mtx")
    generators.write_mtx(mtx, rp, ci, v)
    d, out = run_ref(mtx, 8, B[:, 0])
    res = collect(d, 8, full=False)
    res.update(np=np.array([8]), generator_version=np.array([generators.GENERATOR_VERSION]))
    np.savez_compressed(os.path.join(HERE, "c1_2d128_np8.npz"), **res)
    print("c1_2d128", out.strip().splitlines()[-1])


if __name__ == "__main__":
    main()
