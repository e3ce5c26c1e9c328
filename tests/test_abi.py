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
