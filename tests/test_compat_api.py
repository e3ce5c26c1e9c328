"""The reference's own C++ interface (include/snusolver.h) and the driver.

A C++ program written against the reference's API (csr_matrix,
read_matrix, coo_to_csr, initialize, solve, SnuMat) compiles and links
against libsnusolver_b200.so unchanged.  On CPU the file-reading half runs;
on a GPU the solve calls run and are checked by their residual and against
the Python API.
"""
import os
import subprocess

import numpy as np
import pytest

import snusolver_b200 as snu
from snusolver_b200 import generators
from util import ROOT, rel_resid

PROGRAM = r'''
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "snusolver.h"

int main(int argc, char** argv) {
  csr_matrix A = read_matrix(argc, argv);
  if (!strcmp(argv[2], "read")) {
    // entries per row in file order
    printf("%d %d %d\n", A.n, A.m, A.nnz);
    for (int i = 0; i <= A.n; i++) printf("%d ", A.rowptr[i]);
    printf("\n");
    for (int k = 0; k < A.nnz; k++) printf("%d:%.17g ", A.colidx[k], A.data[k]);
    printf("\n");
    free_csr_matrix(&A);
    return 0;
  }
  initialize();
  double* b = (double*)malloc(sizeof(double) * A.n);
  double* x = (double*)malloc(sizeof(double) * A.n);
  double* x2 = (double*)malloc(sizeof(double) * A.n);
  for (int i = 0; i < A.n; i++) b[i] = 1.0 + (i % 7) * 0.125;
  solve(A, b, x);                 // the reference's one-call entry
  {
    SnuMat Ab(A, b, nullptr, nullptr);
    Ab.solve(x2);                 // construct, then factor + solve
  }
  FILE* f = fopen(argv[3], "wb");
  fwrite(x, sizeof(double), A.n, f);
  fwrite(x2, sizeof(double), A.n, f);
  fclose(f);
  free(b); free(x); free(x2);
  free_csr_matrix(&A);
  return 0;
}
'''


def _build_program(tmp_path):
    src = tmp_path / "prog.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    libdir = os.path.dirname(snu.library_path())
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT}/include", str(src),
                    "-o", str(exe), f"-L{libdir}", "-lsnusolver_b200",
                    f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def _mtx(tmp_path, rp, ci, v, name="a.mtx"):
    p = tmp_path / name
    generators.write_mtx(str(p), rp, ci, v)
    return p


def test_reference_api_reads_matrix(tmp_path):
    exe = _build_program(tmp_path)
    # rows out of order and an unsorted row: CSR keeps file order per row
    p = tmp_path / "m.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n"
                 "3 3 5\n3 1 -1\n1 1 4\n3 3 5\n1 3 0.5\n2 2 2\n")
    out = subprocess.run([str(exe), str(p), "read"], check=True,
                         capture_output=True, text=True).stdout.split("\n")
    assert out[0].split() == ["3", "3", "5"]
    assert [int(t) for t in out[1].split()] == [0, 2, 3, 5]
    ent = [(int(a), float(b)) for a, b in (t.split(":") for t in out[2].split())]
    assert ent == [(0, 4.0), (2, 0.5), (1, 2.0), (0, -1.0), (2, 5.0)]
    # the Python reader sees the same arrays
    A = snu.read_matrix(str(p))
    assert list(A.rowptr) == [0, 2, 3, 5] and list(A.colidx) == [0, 2, 1, 0, 2]


def test_driver_usage_without_matrix():
    drv = os.path.join(os.path.dirname(snu.library_path()), "driver")
    r = subprocess.run([drv], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


@pytest.mark.gpu
def test_reference_api_solves(gpu, tmp_path):
    exe = _build_program(tmp_path)
    rp, ci, v = generators.laplace2d_perturbed(40, 37, seed=3)
    p = _mtx(tmp_path, rp, ci, v)
    out = tmp_path / "x.bin"
    env = dict(os.environ, SNU_NLEAVES="4")
    subprocess.run([str(exe), str(p), "solve", str(out)], check=True, env=env)
    xs = np.fromfile(out, dtype=np.float64).reshape(2, -1)
    n = len(rp) - 1
    b = 1.0 + (np.arange(n) % 7) * 0.125
    for x in xs:
        assert rel_resid(rp, ci, v, x, b) <= 1e-12
    ref = snu.Solver(nleaves=4).construct(rp, ci, v).factorize().solve(b)
    assert np.abs(xs[0] - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(xs[1] - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32ir"])
def test_driver_solves_mtx(gpu, tmp_path, precision):
    rp, ci, v = generators.convdiff3d(16)
    p = _mtx(tmp_path, rp, ci, v)
    drv = os.path.join(os.path.dirname(snu.library_path()), "driver")
    r = subprocess.run([drv, "--nrhs", "3", "--precision", precision,
                        "--nleaves", "8", str(p)], capture_output=True,
                       text=True, check=True)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("max |Ax-b|")]
    assert line, r.stdout
    assert float(line[0].split("=")[1]) <= 1e-9
