"""The seeded synthetic workloads have the shapes the configurations name:
C1 2D 128^2 5-point (n 16,384, nnz 81,408, 1 RHS), C2 64^3 7-point
convection-diffusion (n 262,144, nnz 1,810,432, 4 RHS, diagonally dominant),
C3 256 grids of sides 32..256 (5,204,090 rows), C4 96^3 27-point
(n 884,736, nnz 23,393,656, 16 RHS); the draws are reproducible."""
import numpy as np

from snusolver_b200 import generators as g


def _rows(rp):
    return np.repeat(np.arange(len(rp) - 1), np.diff(rp))


def test_c1_c2_shapes_and_dominance():
    rp, ci, v, B = g.config("c1_2d128")
    assert (len(rp) - 1, len(ci), B.shape) == (16384, 81408, (16384, 1))
    rp, ci, v, B = g.config("c2_convdiff64")
    assert (len(rp) - 1, len(ci), B.shape) == (262144, 1810432, (262144, 4))
    rows = _rows(rp)
    diag = np.zeros(len(rp) - 1)
    off = np.zeros(len(rp) - 1)
    np.add.at(diag, rows[rows == ci], v[rows == ci])
    np.add.at(off, rows[rows != ci], np.abs(v[rows != ci]))
    assert (diag - off).min() >= 0.0  # weakly diagonally dominant rows
    rp2, ci2, v2, B2 = g.config("c2_convdiff64")
    assert np.array_equal(v, v2) and np.array_equal(B, B2)  # seeded


def test_c3_batch_and_c4_shapes():
    mats = g.batch_config("c3_batch256")
    sides_ok = all(32 * 32 <= len(m[0]) - 1 <= 256 * 256 for m in mats)
    assert len(mats) == 256 and sides_ok
    assert sum(len(m[0]) - 1 for m in mats) == 5204090
    rp, ci, v, B = g.config("c4_27pt96")
    assert (len(rp) - 1, len(ci), B.shape) == (884736, 23393656, (884736, 16))
