"""Test helpers: golden fixtures and the C oracle (oracle/snu_oracle.c)."""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libsnu_oracle.so")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "snu_ref")

_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def load_oracle():
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restated"],
                       check=True, capture_output=True)
    lib = C.CDLL(ORACLE_SO)
    lib.snu_oracle_solve.restype = C.c_int
    lib.snu_oracle_solve.argtypes = [C.c_int, _I, _I, _D, _D, C.c_int, _I, _I,
                                     C.c_double, _D, C.POINTER(_D), _I,
                                     C.POINTER(_D)]
    lib.snu_oracle_free.argtypes = [C.c_void_p]
    return lib


def oracle_solve(rowptr, colidx, vals, b, np_, order, sizes, eps=1e-15):
    """Reference numerics restated in C: x, per-rank leaf LU_data, dense
    separator blocks {(i, j): column-major array}."""
    lib = load_oracle()
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    v = np.ascontiguousarray(vals, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    order = np.ascontiguousarray(order, np.int32)
    sizes = np.ascontiguousarray(sizes, np.int32)
    n = len(rp) - 1
    x = np.zeros(n)
    nb2 = 2 * np_
    leaf = (_D * np_)()
    leafn = (C.c_int * np_)()
    dense = (_D * (nb2 * nb2))()
    rc = lib.snu_oracle_solve(n, rp.ctypes.data_as(_I), ci.ctypes.data_as(_I),
                              v.ctypes.data_as(_D), b.ctypes.data_as(_D), np_,
                              order.ctypes.data_as(_I), sizes.ctypes.data_as(_I),
                              eps, x.ctypes.data_as(_D), leaf, leafn, dense)
    assert rc == 0, rc
    lus = []
    for r in range(np_):
        m = leafn[r]
        lus.append(np.ctypeslib.as_array(leaf[r], (m,)).copy() if m else np.zeros(0))
        lib.snu_oracle_free(C.cast(leaf[r], C.c_void_p))
    blocks = {}
    for i in range(1, np_):
        for j in range(1, np_):
            p = dense[i * nb2 + j]
            if p:
                blocks[(i, j)] = p
    return x, lus, blocks, lib


def dense_block_array(lib, ptr, m, n):
    if m * n == 0:
        return np.zeros((m, n))
    a = np.ctypeslib.as_array(ptr, (m * n,)).copy().reshape((m, n), order="F")
    return a


def free_blocks(lib, blocks):
    for p in blocks.values():
        lib.snu_oracle_free(C.cast(p, C.c_void_p))


def rel_resid(rowptr, colidx, vals, x, b):
    """||b - A x||inf / (||A||inf ||x||inf + ||b||inf)."""
    n = len(rowptr) - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    Ax = np.zeros(n)
    np.add.at(Ax, rows, vals * x[colidx])
    anorm = np.zeros(n)
    np.add.at(anorm, rows, np.abs(vals))
    return np.abs(b - Ax).max() / (anorm.max() * np.abs(x).max() + np.abs(b).max())


def csr_from_dense(M):
    rows, cols = np.nonzero(M)
    rowptr = np.zeros(M.shape[0] + 1, np.int32)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols.astype(np.int32), M[rows, cols]
