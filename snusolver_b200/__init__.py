"""snusolver_b200 -- B200 numeric factorize-and-solve path of SnuSolver.

Python host mirror of the reference interface over the C-ABI in
``include/snusolver_b200.h`` (``libsnusolver_b200.so``, built in-tree by
``snusolver_b200.build``).  The numeric work runs in CUDA kernels for
sm_100a; there is no CPU fallback: without the library or a GPU the calls
raise ``SnuError``.

Reference surface mirrored (rhrnald/snusolver):
  * ``initialize()`` / ``solve(A, b, x)``      -- src/snusolver.h:5-6, src/solver.cu:35-89
  * ``SnuMat(A, b)`` + ``SnuMat.solve(x)``      -- src/SnuMat.h:142-147
  * ``read_matrix(path)``                       -- src/read_matrix.cpp:50-107
plus ``Solver`` (one handle: analyze / construct / factorize / refactor /
solve, device-pointer solves, stats and parity read-back).
"""
from __future__ import annotations

import ctypes as C
import os
from collections import namedtuple

import numpy as np

__all__ = ["SnuError", "Solver", "CsrMatrix", "read_matrix", "initialize",
           "solve", "SnuMat", "library_path", "load_library", "FP64", "FP32_IR",
           "SPLIT_AUTO", "SPLIT_TF32", "SPLIT_BF16", "STATUS"]

FP64, FP32_IR = 0, 1
SPLIT_AUTO, SPLIT_TF32, SPLIT_BF16 = 0, 1, 2  # FP32 tensor-core GEMM split
STATUS = {0: "SNU_OK", 1: "SNU_EINVAL", 2: "SNU_ENOMEM", 3: "SNU_ESINGULAR",
          4: "SNU_ETIMEOUT", 5: "SNU_ECUDA", 6: "SNU_ESTATE", 7: "SNU_ENOTCONV"}

# csr_matrix of src/matrix.h:9-13 (n, m, nnz, rowptr, colidx, data)
CsrMatrix = namedtuple("CsrMatrix", "n m nnz rowptr colidx data")

_HERE = os.path.dirname(os.path.abspath(__file__))


def library_path() -> str:
    return os.path.join(_HERE, "libsnusolver_b200.so")


class SnuError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class _Opts(C.Structure):
    _fields_ = [("nleaves", C.c_int), ("precision", C.c_int),
                ("pivot_eps", C.c_double), ("ir_tol", C.c_double),
                ("ir_max_iter", C.c_int), ("device", C.c_int),
                ("mem_budget", C.c_int64), ("fp64_growth", C.c_double),
                ("gemm_split", C.c_int), ("reserved", C.c_int * 5)]


class _Stats(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("nleaves", C.c_int),
                ("nfronts", C.c_int), ("nlevels", C.c_int),
                ("factor_entries", C.c_int64), ("device_bytes", C.c_int64),
                ("analyze_s", C.c_double), ("factor_s", C.c_double),
                ("solve_s", C.c_double), ("factor_flops", C.c_double),
                ("ir_iters", C.c_int), ("fp64_fallback", C.c_int),
                ("backward_error", C.c_double), ("tiny_pivots", C.c_int),
                ("factor_launches", C.c_int), ("solve_launches", C.c_int),
                ("fp64_fronts", C.c_int), ("reserved", C.c_int * 4)]


class _KStat(C.Structure):
    _fields_ = [("name", C.c_char_p), ("launches", C.c_int64),
                ("seconds", C.c_double), ("flops", C.c_double),
                ("bytes", C.c_double)]


class _LaunchRec(C.Structure):
    _fields_ = [("family", C.c_int), ("level", C.c_int),
                ("seconds", C.c_double), ("flops", C.c_double),
                ("bytes", C.c_double)]


KERNEL_FAMILIES = ("assemble", "extend_add", "diag_lu", "panel_trsm",
                   "gemm_trail", "gemm_schur", "solve_diag", "solve_gemm",
                   "solve_misc", "residual", "panel_block", "block_inv",
                   "gemm_panel", "sweep")

_lib = None
_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)
_EXPORTS = {
    "snu_default_opts": (None, [C.POINTER(_Opts)]),
    "snu_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(_Opts)]),
    "snu_destroy": (C.c_int, [C.c_void_p]),
    "snu_last_error": (C.c_char_p, [C.c_void_p]),
    "snu_status_string": (C.c_char_p, [C.c_int]),
    "snu_analyze": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _I, _I]),
    "snu_plan": (C.c_int, [C.c_void_p]),
    "snu_construct": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _I, _I, _D]),
    "snu_construct_batch": (C.c_int, [C.c_void_p, C.c_int, _I, C.c_int,
                                      C.c_int, _I, _I, _D]),
    "snu_factorize": (C.c_int, [C.c_void_p]),
    "snu_refactor": (C.c_int, [C.c_void_p, _D]),
    "snu_solve": (C.c_int, [C.c_void_p, _D, _D, C.c_int, C.c_int]),
    "snu_solve_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_int, C.c_void_p]),
    "snu_get_stats": (C.c_int, [C.c_void_p, C.POINTER(_Stats)]),
    "snu_get_ordering": (C.c_int, [C.c_void_p, _I, _I]),
    "snu_get_blocks": (C.c_int, [C.c_void_p, _I, _I]),
    "snu_get_coo": (C.c_int, [C.c_void_p, _I, _I, _I]),
    "snu_get_leaf_info": (C.c_int, [C.c_void_p, C.c_int, _I]),
    "snu_get_leaf_pattern": (C.c_int, [C.c_void_p, C.c_int, _I, _I, _I, _I, _I]),
    "snu_get_leaf_factor": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "snu_get_dense_block": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D]),
    "snu_read_mtx": (C.c_int, [C.c_char_p, C.c_int, _I, _I, C.POINTER(_I),
                               C.POINTER(_I), C.POINTER(_D)]),
    "snu_free": (None, [C.c_void_p]),
    "snu_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "snu_set_profiling": (C.c_int, [C.c_void_p, C.c_uint]),
    "snu_set_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
    "snu_get_trace": (C.c_int, [C.c_void_p, C.POINTER(_LaunchRec), C.c_int,
                                C.POINTER(C.c_int)]),
    "snu_get_profile": (C.c_int, [C.c_void_p, C.POINTER(_KStat), C.c_int,
                                  C.POINTER(C.c_int)]),
    "snu_reset_profile": (C.c_int, [C.c_void_p]),
    "snu_front_plan_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "snu_get_front_plan": (C.c_int, [C.c_void_p, _I, C.POINTER(C.c_int64), _I,
                                     _I, C.POINTER(C.c_int64), _I]),
}


def load_library(path: str | None = None):
    """Loads the native library (raises SnuError if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or library_path()
    if not os.path.exists(p):
        raise SnuError(5, f"native library not built: {p} "
                          "(run python -m snusolver_b200.build)")
    lib = C.CDLL(p)
    for name, (res, args) in _EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _iptr(a):
    return a.ctypes.data_as(_I)


def _dptr(a):
    return a.ctypes.data_as(_D)


class Solver:
    """One handle of the C-ABI: plan (host) + factors (device)."""

    def __init__(self, nleaves=8, precision=FP64, pivot_eps=1e-15,
                 ir_tol=1e-10, ir_max_iter=10, device=0, mem_budget=0,
                 fp64_growth=1e3, gemm_split=0):
        self._lib = load_library()
        o = _Opts()
        self._lib.snu_default_opts(C.byref(o))
        o.nleaves, o.precision = nleaves, precision
        o.pivot_eps, o.ir_tol, o.ir_max_iter = pivot_eps, ir_tol, ir_max_iter
        o.device, o.mem_budget = device, mem_budget
        o.fp64_growth = fp64_growth
        o.gemm_split = gemm_split  # SPLIT_AUTO, SPLIT_TF32 or SPLIT_BF16
        h = C.c_void_p()
        st = self._lib.snu_create(C.byref(h), C.byref(o))
        if st:
            raise SnuError(st, self._lib.snu_last_error(None).decode())
        self._h = h
        self.n = 0
        self.nnz = 0
        self.nleaves = nleaves

    def close(self):
        if getattr(self, "_h", None):
            self._lib.snu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, allow=()):
        if st and st not in allow:
            raise SnuError(st, self._lib.snu_last_error(self._h).decode())
        return st

    # ---------------------------------------------------------------- phases
    def analyze(self, rowptr, colidx):
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(colidx, dtype=np.int32)
        self._check(self._lib.snu_analyze(self._h, len(rp) - 1, len(ci),
                                          _iptr(rp), _iptr(ci)))
        self.n, self.nnz = len(rp) - 1, len(ci)
        return self

    def plan(self):
        """Front plan of the analyzed pattern, on the host: stats() then
        holds nfronts, nlevels, factor_entries and factor_flops; a construct
        of the same pattern reuses the analysis and the plan."""
        self._check(self._lib.snu_plan(self._h))
        return self

    def construct(self, rowptr, colidx, vals):
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(colidx, dtype=np.int32)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        self._check(self._lib.snu_construct(self._h, len(rp) - 1, len(ci),
                                            _iptr(rp), _iptr(ci), _dptr(v)))
        self.n, self.nnz = len(rp) - 1, len(ci)
        return self

    def construct_batch(self, mats):
        """A batch of independent matrices [(rowptr, colidx, vals), ...] as
        one block-diagonal system (see ``snu_construct_batch``).  Solves take
        the right-hand sides of all matrices stacked in matrix order;
        ``self.row_start`` gives each matrix's rows."""
        rps, cis, vs, starts = [], [], [], [0]
        nz = 0
        for rp, ci, v in mats:
            rp = np.asarray(rp, dtype=np.int64)
            rps.append(rp[:-1] + nz)
            cis.append(np.asarray(ci, dtype=np.int64) + starts[-1])
            vs.append(np.asarray(v, dtype=np.float64))
            nz += int(rp[-1])
            starts.append(starts[-1] + len(rp) - 1)
        rp = np.ascontiguousarray(np.concatenate(rps + [np.array([nz])]),
                                  dtype=np.int32)
        ci = np.ascontiguousarray(np.concatenate(cis), dtype=np.int32)
        v = np.ascontiguousarray(np.concatenate(vs))
        st = np.ascontiguousarray(starts, dtype=np.int32)
        self._check(self._lib.snu_construct_batch(
            self._h, len(mats), _iptr(st), len(rp) - 1, len(ci), _iptr(rp),
            _iptr(ci), _dptr(v)))
        self.n, self.nnz = len(rp) - 1, len(ci)
        self.row_start = st
        return self

    def factorize(self):
        self._check(self._lib.snu_factorize(self._h))
        return self

    def refactor(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        if len(v) != self.nnz:
            raise SnuError(1, "values length differs from the pattern")
        self._check(self._lib.snu_refactor(self._h, _dptr(v)))
        return self

    def solve(self, B, allow_notconv=False, out=None):
        """X = A^-1 B for a vector or a column-major (n, nrhs) array;
        ``out`` (same shape, Fortran order, float64) receives X if given."""
        B = np.asarray(B, dtype=np.float64)
        vec = B.ndim == 1
        Bm = np.asfortranarray(B.reshape(self.n, -1))
        if out is not None:
            X = out.reshape(self.n, -1)
            if X.dtype != np.float64 or not X.flags.f_contiguous:
                raise SnuError(1, "out must be a Fortran-ordered float64 array")
        else:
            X = np.empty_like(Bm, order="F")
        self._check(self._lib.snu_solve(self._h, _dptr(Bm), _dptr(X),
                                        Bm.shape[1], self.n),
                    allow=(7,) if allow_notconv else ())
        return X[:, 0] if vec else X

    def solve_device(self, dB, dX, nrhs, ldb, stream=0, allow_notconv=False):
        """Device-pointer solve (integers: CUDA device addresses / stream)."""
        return self._check(self._lib.snu_solve_device(
            self._h, C.c_void_p(dB), C.c_void_p(dX), nrhs, ldb,
            C.c_void_p(stream or None)), allow=(7,) if allow_notconv else ())

    def set_stream(self, stream):
        """CUDA stream (integer handle, 0 = the handle's own) for all work."""
        self._check(self._lib.snu_set_stream(self._h, C.c_void_p(stream or None)))
        return self

    def set_autotune(self, enable=True, cache_path=None):
        """Tune the tensor-core GEMM variant per batch at the next FP32
        factorization (see ``snu_set_autotune``)."""
        self._check(self._lib.snu_set_autotune(
            self._h, int(enable), cache_path.encode() if cache_path else None))
        return self

    def set_profiling(self, families=(), trace=False):
        """Per-launch CUDA-event timing for the named kernel families;
        ``trace`` also keeps every launch's record (see :meth:`trace`)."""
        mask = 0x80000000 if trace else 0
        for f in families:
            mask |= 1 << KERNEL_FAMILIES.index(f)
        self._check(self._lib.snu_set_profiling(self._h, mask))
        return self

    def profile(self):
        arr = (_KStat * 16)()
        cnt = C.c_int()
        self._check(self._lib.snu_get_profile(self._h, arr, 16, C.byref(cnt)))
        return {arr[i].name.decode(): dict(launches=arr[i].launches,
                                           seconds=arr[i].seconds,
                                           flops=arr[i].flops,
                                           bytes=arr[i].bytes)
                for i in range(cnt.value)}

    def trace(self):
        """Per-launch records (family, level, seconds, flops, bytes), in
        launch order; recorded while profiling runs with ``trace=True``."""
        cnt = C.c_int()
        self._check(self._lib.snu_get_trace(self._h, None, 0, C.byref(cnt)))
        arr = (_LaunchRec * max(cnt.value, 1))()
        self._check(self._lib.snu_get_trace(self._h, arr, cnt.value,
                                            C.byref(cnt)))
        return [(KERNEL_FAMILIES[r.family], r.level, r.seconds, r.flops,
                 r.bytes) for r in arr[:cnt.value]]

    def reset_profile(self):
        self._check(self._lib.snu_reset_profile(self._h))
        return self

    def stats(self):
        s = _Stats()
        self._check(self._lib.snu_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _Stats._fields_ if k != "reserved"}

    # ------------------------------------------------------ parity read-back
    def ordering(self):
        order = np.empty(self.n, np.int32)
        sizes = np.empty(2 * self.nleaves - 1, np.int32)
        self._check(self._lib.snu_get_ordering(self._h, _iptr(order), _iptr(sizes)))
        return order, sizes

    def blocks(self):
        bs = np.empty(2 * self.nleaves, np.int32)
        bz = np.empty(2 * self.nleaves, np.int32)
        self._check(self._lib.snu_get_blocks(self._h, _iptr(bs), _iptr(bz)))
        return bs, bz

    def coo(self):
        pm, r, c = (np.empty(self.nnz, np.int32) for _ in range(3))
        self._check(self._lib.snu_get_coo(self._h, _iptr(pm), _iptr(r), _iptr(c)))
        return pm, r, c

    def front_plan(self):
        """The front plan (after :meth:`plan` or :meth:`construct`): dict of
        per-front arrays p, q, ld, parent, level, block, guard, leaf_rank,
        offset, idx_offset, rel_offset, plus gidx, rel, asm_pos, asm_val,
        arena and nlevels (see ``snu_get_front_plan``)."""
        sz = (C.c_int64 * 6)()
        self._check(self._lib.snu_front_plan_sizes(self._h, sz))
        nf, ng, nr, na, arena, nl = (int(x) for x in sz)
        fr = np.empty((max(nf, 1), 8), np.int32)
        off = np.empty((max(nf, 1), 3), np.int64)
        gidx = np.empty(max(ng, 1), np.int32)
        rel = np.empty(max(nr, 1), np.int32)
        apos = np.empty(max(na, 1), np.int64)
        aval = np.empty(max(na, 1), np.int32)
        i64 = C.POINTER(C.c_int64)
        self._check(self._lib.snu_get_front_plan(
            self._h, _iptr(fr), off.ctypes.data_as(i64), _iptr(gidx),
            _iptr(rel), apos.ctypes.data_as(i64), _iptr(aval)))
        keys = ("p", "q", "ld", "parent", "level", "block", "guard", "leaf_rank")
        out = {k: fr[:nf, i].copy() for i, k in enumerate(keys)}
        for i, k in enumerate(("offset", "idx_offset", "rel_offset")):
            out[k] = off[:nf, i].copy()
        out.update(gidx=gidx[:ng], rel=rel[:nr], asm_pos=apos[:na],
                   asm_val=aval[:na], arena=arena, nlevels=nl)
        return out

    def leaf_info(self, rank):
        info = np.empty(8, np.int32)
        self._check(self._lib.snu_get_leaf_info(self._h, rank, _iptr(info)))
        keys = ("leaf", "leaf_size", "dense_row", "core_n", "core_nnz", "LU_nnz")
        return dict(zip(keys, (int(x) for x in info[:6])))

    def leaf_pattern(self, rank):
        self._check(self._lib.snu_get_leaf_pattern(self._h, rank, None, None,
                                                   None, None, None))
        info = self.leaf_info(rank)
        cn, nz = info["core_n"], info["LU_nnz"]
        out = dict(LU_rowptr=np.empty(cn + 1, np.int32),
                   LU_colidx=np.empty(nz, np.int32),
                   LU_diag=np.empty(cn, np.int32),
                   LU_bias=np.empty(info["leaf_size"], np.int32),
                   core_map=np.empty(info["core_nnz"], np.int32))
        self._check(self._lib.snu_get_leaf_pattern(
            self._h, rank, _iptr(out["LU_rowptr"]), _iptr(out["LU_colidx"]),
            _iptr(out["LU_diag"]), _iptr(out["LU_bias"]), _iptr(out["core_map"])))
        return out

    def leaf_factor(self, rank):
        self.leaf_pattern(rank)
        nz = self.leaf_info(rank)["LU_nnz"]
        out = np.empty(nz, np.float64)
        self._check(self._lib.snu_get_leaf_factor(self._h, rank, _dptr(out)))
        return out

    def dense_block(self, i, j):
        _, bz = self.blocks()
        out = np.empty(int(bz[i]) * int(bz[j]), np.float64)
        self._check(self._lib.snu_get_dense_block(self._h, i, j, _dptr(out)))
        return out.reshape((int(bz[i]), int(bz[j])), order="F")


def read_matrix(path, expand_symmetric=False, cache=None) -> CsrMatrix:
    """MatrixMarket reader with read_matrix.cpp semantics.

    cache: optional path of a binary CSR copy (numpy .npz).  When it exists,
    is newer than the .mtx file and was written with the same
    expand_symmetric, it is loaded instead of parsing; otherwise the file is
    parsed and the copy (re)written.  Nothing is written without it."""
    if cache is not None:
        try:
            if os.path.getmtime(cache) >= os.path.getmtime(path):
                with np.load(cache) as z:
                    if bool(z["expand_symmetric"]) == bool(expand_symmetric):
                        n = int(z["n"])
                        return CsrMatrix(n, n, int(z["data"].size),
                                         z["rowptr"].copy(), z["colidx"].copy(),
                                         z["data"].copy())
        except (OSError, KeyError, ValueError):
            pass  # missing or unreadable copy: parse the file
        A = read_matrix(path, expand_symmetric)
        tmp = f"{cache}.tmp.{os.getpid()}.npz"
        np.savez(tmp, n=np.int64(A.n), rowptr=A.rowptr, colidx=A.colidx,
                 data=A.data, expand_symmetric=np.bool_(expand_symmetric))
        os.replace(tmp, cache)  # readers never see a partial copy
        return A
    lib = load_library()
    n, nnz = C.c_int(), C.c_int()
    rp, ci, v = _I(), _I(), _D()
    st = lib.snu_read_mtx(path.encode(), int(expand_symmetric), C.byref(n),
                          C.byref(nnz), C.byref(rp), C.byref(ci), C.byref(v))
    if st:
        raise SnuError(st, lib.snu_last_error(None).decode())
    try:
        rowptr = np.ctypeslib.as_array(rp, (n.value + 1,)).copy()
        colidx = np.ctypeslib.as_array(ci, (max(nnz.value, 1),))[:nnz.value].copy()
        data = np.ctypeslib.as_array(v, (max(nnz.value, 1),))[:nnz.value].copy()
    finally:
        lib.snu_free(C.cast(rp, C.c_void_p))
        lib.snu_free(C.cast(ci, C.c_void_p))
        lib.snu_free(C.cast(v, C.c_void_p))
    return CsrMatrix(n.value, n.value, nnz.value, rowptr, colidx, data)


# ------------------------------------------------ reference-shaped interface
_default = {"nleaves": 8}


def initialize(nleaves=8, device=0):
    """solver.cu:35-49: selects the device; here also the leaf count (the
    reference takes it from the MPI world size)."""
    load_library()
    _default["nleaves"] = nleaves
    _default["device"] = device


class SnuMat:
    """SnuMat.h:142-147: construct from (A, b), then solve(x) factors and
    solves in one call, writing x."""

    def __init__(self, A: CsrMatrix, b, precision=FP64):
        self._s = Solver(nleaves=_default.get("nleaves", 8), precision=precision,
                         device=_default.get("device", 0))
        self._s.construct(A.rowptr, A.colidx, A.data)
        self._b = np.array(b, dtype=np.float64)

    def solve(self, x):
        self._s.factorize()
        x[:] = self._s.solve(self._b)

    @property
    def solver(self):
        return self._s


def solve(A: CsrMatrix, b, x):
    """solver.cu:51-89: construct + factor + solve, x written in place."""
    SnuMat(A, b).solve(x)
