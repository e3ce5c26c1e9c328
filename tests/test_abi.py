"""C-ABI boundary: the library loads, exports every declared entry point,
and rejects bad input with the documented status codes (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import snusolver_b200 as snu
from util import ROOT, golden

HEADER = os.path.join(ROOT, "include", "snusolver_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"SNU_API\s+[\w\s\*]+?\b(snu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(snu.library_path())
    names = declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_bad_options_rejected():
    with pytest.raises(snu.SnuError) as e:
        snu.Solver(nleaves=6)
    assert e.value.status == 1
    with pytest.raises(snu.SnuError):
        snu.Solver(nleaves=1024)


def test_precision_option_defaults_and_checks():
    # snu_opts: fp64_growth 1e3 and the automatic GEMM split by default;
    # the server's handles default to TF32x3; out-of-range values refused
    from snusolver_b200.server import _ServerOpts
    lib = snu.load_library()
    o = snu._Opts()
    lib.snu_default_opts(C.byref(o))
    assert o.fp64_growth == 1e3 and o.gemm_split == snu.SPLIT_AUTO
    assert C.sizeof(snu._Opts) == 72 and C.sizeof(snu._Stats) == 120
    so = _ServerOpts()
    lib.snu_server_default_opts(C.byref(so))
    assert so.gemm_split == snu.SPLIT_TF32
    for kw in ({"gemm_split": 3}, {"gemm_split": -1}, {"fp64_growth": -1.0}):
        with pytest.raises(snu.SnuError) as e:
            snu.Solver(**kw)
        assert e.value.status == 1, kw
    snu.Solver(gemm_split=snu.SPLIT_TF32, fp64_growth=0.0).close()


def test_bad_csr_rejected():
    s = snu.Solver(nleaves=2)
    with pytest.raises(snu.SnuError) as e:
        s.analyze(np.array([0, 2, 1]), np.array([0, 1]))
    assert e.value.status == 1
    with pytest.raises(snu.SnuError):
        s.analyze(np.array([0, 1, 2]), np.array([0, 5]))


def test_order_of_calls_checked():
    s = snu.Solver(nleaves=2)
    with pytest.raises(snu.SnuError) as e:
        s.factorize()
    assert e.value.status == 6  # SNU_ESTATE


def test_read_mtx_rejects_complex_and_pattern(tmp_path):
    p = tmp_path / "c.mtx"
    p.write_text("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n")
    with pytest.raises(snu.SnuError):
        snu.read_matrix(str(p))
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n1 1 1\n1 1\n")
    with pytest.raises(snu.SnuError):
        snu.read_matrix(str(p))


def test_construct_needs_the_gpu_path():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present: covered by the gpu tests")
    except Exception:
        pass
    g = golden("matrix20_np4.npz")
    s = snu.Solver(nleaves=4)
    with pytest.raises(snu.SnuError) as e:
        s.construct(g["rowptr"], g["colidx"], g["vals"])
    assert e.value.status == 5  # SNU_ECUDA: no CPU fallback


def test_duplicates_analyzed_but_rejected_numerically():
    from snusolver_b200 import generators
    rp, ci, v = generators.laplace2d_perturbed(6, 6, seed=3)
    # duplicate entry (0, 1): the structure keeps it like the reference does,
    # the numeric path refuses it (SNU_EINVAL) instead of guessing a meaning
    rp2 = rp.copy()
    rp2[1:] += 1
    ci2 = np.insert(ci, 1, ci[1])
    v2 = np.insert(v, 1, 0.25)
    s = snu.Solver(nleaves=2).analyze(rp2, ci2)
    order, sizes = s.ordering()
    assert sorted(order) == list(range(36))
    with pytest.raises(snu.SnuError) as e:
        snu.Solver(nleaves=2).construct(rp2, ci2, v2)
    assert e.value.status == 1
    assert "duplicate" in str(e.value)


@pytest.mark.parametrize("body,why", [
    ("3 3 4\n1 1 2\n2 2 3\n", "truncated"),
    ("3 3 2\n1 1 2\n4 2 3\n", "out of range"),
    ("3 3 2\n1 1 abc\n2 2 3\n", "truncated"),
    ("3 2 2\n1 1 1\n2 2 3\n", "not square"),
    ("x y z\n", "size line"),
])
def test_read_mtx_rejects_corrupt_files(tmp_path, body, why):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n" + body)
    with pytest.raises(snu.SnuError) as e:
        snu.read_matrix(str(p))
    assert e.value.status == 1 and why in str(e.value)


def _big_mtx(path, n=200_000, per_row=5, seed=7, broken_every=0, tail="",
             extra_nz=0, bad_last=False):
    """A file above the reader's parallel-parse threshold (16 MB); returns the
    expected CSR (rows keep file order)."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), per_row)
    cols = rng.integers(0, n, size=rows.size)
    vals = rng.standard_normal(rows.size)
    order = rng.permutation(rows.size)  # entries in random file order
    rows, cols, vals = rows[order], cols[order], vals[order]
    lines = []
    for k, (r, c, v) in enumerate(zip(rows.tolist(), cols.tolist(), vals.tolist())):
        if bad_last and k == rows.size - 1:
            r = n  # 0-based n -> 1-based n + 1: out of range
        sep = "\n" if broken_every and k % broken_every == 0 else " "
        lines.append(f"{r + 1}{sep}{c + 1}{sep}{v!r}\n")
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n% generated\n")
        f.write(f"{n} {n} {rows.size + extra_nz}\n")
        f.write("".join(lines))
        f.write(tail)
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    idx = np.argsort(rows, kind="stable")
    return rp, cols[idx], vals[idx]


@pytest.mark.parametrize("broken_every,tail", [(0, ""), (997, ""),
                                               (0, "1 1 1.0\ngarbage\n")])
def test_read_mtx_large_files_match_file_order(tmp_path, broken_every, tail):
    # large files are parsed in line-aligned chunks on host threads; the CSR
    # must be the sequential parse's (file order kept, entries broken over
    # lines and text after the last declared entry handled the same way)
    p = str(tmp_path / "big.mtx")
    rp, ci, v = _big_mtx(p, broken_every=broken_every, tail=tail)
    assert os.path.getsize(p) > 16 << 20
    A = snu.read_matrix(p)
    assert np.array_equal(np.asarray(A.rowptr), rp)
    assert np.array_equal(np.asarray(A.colidx), ci)
    assert np.array_equal(np.asarray(A.data), v)


@pytest.mark.parametrize("kw,why", [({"bad_last": True}, "out of range"),
                                    ({"extra_nz": 3}, "truncated")])
def test_read_mtx_large_files_rejected(tmp_path, kw, why):
    p = str(tmp_path / "big_bad.mtx")
    _big_mtx(p, **kw)
    with pytest.raises(snu.SnuError) as e:
        snu.read_matrix(p)
    assert e.value.status == 1 and why in str(e.value)


def test_read_mtx_binary_cache(tmp_path):
    # an opt-in binary CSR copy: reused while newer than the .mtx file and
    # written with the same expand_symmetric, rebuilt otherwise
    mtx, cache = tmp_path / "a.mtx", str(tmp_path / "a.csr.npz")
    hdr = "%%MatrixMarket matrix coordinate real symmetric\n"
    mtx.write_text(hdr + "3 3 3\n1 1 2.0\n2 1 -1.0\n3 3 4.0\n")
    A = snu.read_matrix(str(mtx), expand_symmetric=True, cache=cache)
    assert os.path.exists(cache) and A.nnz == 4
    # same (older) file name, other contents: the copy is what is read
    mtx.write_text(hdr + "3 3 1\n1 1 9.0\n")
    t = os.path.getmtime(cache) - 10
    os.utime(mtx, (t, t))
    B = snu.read_matrix(str(mtx), expand_symmetric=True, cache=cache)
    assert B.nnz == 4 and np.array_equal(B.data, A.data)
    # another expand_symmetric, or a newer file: parsed again
    C1 = snu.read_matrix(str(mtx), expand_symmetric=False, cache=cache)
    assert C1.nnz == 1 and C1.data[0] == 9.0
    assert snu.read_matrix(str(mtx), cache=cache).nnz == 1


def test_plan_on_the_host():
    # the front plan needs no device: deterministic, and refused before
    # analyze
    from snusolver_b200 import generators
    rp, ci, _ = generators.convdiff3d(20)
    keys = ("nfronts", "nlevels", "factor_entries", "factor_flops")
    a = snu.Solver(nleaves=8).analyze(rp, ci).plan().stats()
    b = snu.Solver(nleaves=8).analyze(rp, ci).plan().plan().stats()
    assert all(a[k] == b[k] for k in keys) and a["nfronts"] > 8
    assert a["factor_entries"] > 0 and a["factor_flops"] > 0
    with pytest.raises(snu.SnuError) as e:
        snu.Solver().plan()
    assert e.value.status == 6  # SNU_ESTATE
