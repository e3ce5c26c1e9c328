"""The C restatement (oracle/snu_oracle.c) against outputs of the reference
itself (tests/golden, made from oracle/_ref)."""
import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import dense_block_array, free_blocks, golden, oracle_solve


@pytest.mark.parametrize("np_", [4, 8])
def test_oracle_matrix20(np_):
    g = golden(f"matrix20_np{np_}.npz")
    x, lus, blocks, lib = oracle_solve(g["rowptr"], g["colidx"], g["vals"],
                                       g["b"], np_, g["order"], g["sizes"])
    try:
        np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-12 * np.abs(g["x"]).max())
        for r in range(np_):
            np.testing.assert_array_equal(lus[r], g[f"r{r}_LU_data"])
        bz = g["block_size"]
        for key in g:
            if not key.startswith("dense_"):
                continue
            i, j = map(int, key.split("_")[1:3])
            if bz[i] * bz[j] == 0:
                continue
            ref = g[key].reshape((bz[i], bz[j]), order="F")
            got = dense_block_array(lib, blocks[(i, j)], bz[i], bz[j])
            np.testing.assert_allclose(got, ref, rtol=0,
                                       atol=1e-13 * max(np.abs(ref).max(), 1e-300))
    finally:
        free_blocks(lib, blocks)


def test_oracle_c1():
    g = golden("c1_2d128_np8.npz")
    rp, ci, v, B = generators.config("c1_2d128")
    np.testing.assert_array_equal(B[:, 0], g["b"])
    h = snu.Solver(nleaves=8).analyze(rp, ci)
    order, sizes = h.ordering()
    x, lus, blocks, lib = oracle_solve(rp, ci, v, B[:, 0], 8, order, sizes)
    try:
        np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-12 * np.abs(g["x"]).max())
        for r in range(8):
            idx = g[f"r{r}_LU_data_idx"]
            np.testing.assert_array_equal(lus[r][idx], g[f"r{r}_LU_data_val"])
            assert np.abs(lus[r]).max() == g[f"r{r}_LU_data_absmax"][0]
    finally:
        free_blocks(lib, blocks)
