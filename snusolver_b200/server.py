"""Request server over the C-ABI ``snu_server_*`` calls.

Factor, refactor-same-pattern and solve requests run on one GPU as they
arrive: up to ``slots`` at once on separate CUDA streams, admitted by a
device-memory budget, with factors resident until released.  Submissions
return request ids; :meth:`Server.poll` returns completions with their
queueing, service and end-to-end latencies.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import SnuError, FP32_IR, load_library

__all__ = ["Server", "REQUEST_TYPES"]

REQUEST_TYPES = ("factor", "refactor", "solve", "release")

_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class _ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int),
                ("mem_budget", C.c_int64), ("nleaves", C.c_int),
                ("precision", C.c_int), ("ir_tol", C.c_double),
                ("ir_max_iter", C.c_int), ("plan_cache", C.c_int),
                ("reserved", C.c_int * 8)]


class _Completion(C.Structure):
    _fields_ = [("request", C.c_int64), ("matrix", C.c_int64),
                ("type", C.c_int), ("status", C.c_int),
                ("queue_s", C.c_double), ("service_s", C.c_double),
                ("latency_s", C.c_double), ("backward_error", C.c_double),
                ("ir_iters", C.c_int), ("plan_reused", C.c_int),
                ("reserved", C.c_int * 6)]


class _ServerStats(C.Structure):
    _fields_ = [("resident_bytes", C.c_int64), ("peak_bytes", C.c_int64),
                ("budget_bytes", C.c_int64), ("submitted", C.c_int64),
                ("completed", C.c_int64), ("failed", C.c_int64),
                ("queued", C.c_int), ("running", C.c_int),
                ("matrices", C.c_int), ("cached_plans", C.c_int),
                ("reserved", C.c_int * 8)]


_SIGS = {
    "snu_server_default_opts": (None, [C.POINTER(_ServerOpts)]),
    "snu_server_create": (C.c_int, [C.POINTER(C.c_void_p),
                                    C.POINTER(_ServerOpts)]),
    "snu_server_destroy": (C.c_int, [C.c_void_p]),
    "snu_server_last_error": (C.c_char_p, [C.c_void_p]),
    "snu_server_factor": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _I, _I, _D,
                                    _I64, _I64]),
    "snu_server_refactor": (C.c_int, [C.c_void_p, C.c_int64, _D, _I64]),
    "snu_server_solve": (C.c_int, [C.c_void_p, C.c_int64, _D, _D, C.c_int,
                                   C.c_int, _I64]),
    "snu_server_release": (C.c_int, [C.c_void_p, C.c_int64, _I64]),
    "snu_server_poll": (C.c_int, [C.c_void_p, C.POINTER(_Completion), C.c_int,
                                  _I, C.c_int]),
    "snu_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(_ServerStats)]),
}


def _bind(lib):
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class Server:
    """A request server on one GPU (see the module docstring)."""

    def __init__(self, device=0, slots=4, mem_budget=120 << 30, nleaves=8,
                 precision=FP32_IR, ir_tol=1e-10, ir_max_iter=10,
                 plan_cache=64):
        self._lib = _bind(load_library())
        o = _ServerOpts()
        self._lib.snu_server_default_opts(C.byref(o))
        o.device, o.slots, o.mem_budget = device, slots, mem_budget
        o.nleaves, o.precision = nleaves, precision
        o.ir_tol, o.ir_max_iter, o.plan_cache = ir_tol, ir_max_iter, plan_cache
        s = C.c_void_p()
        st = self._lib.snu_server_create(C.byref(s), C.byref(o))
        if st:
            raise SnuError(st, self._lib.snu_server_last_error(None).decode())
        self._s = s
        self._keep = {}   # request id -> arrays that must outlive the request
        self._n = {}      # matrix id -> (n, nnz)

    def _check(self, st):
        if st:
            raise SnuError(st, self._lib.snu_server_last_error(self._s).decode())

    def close(self):
        if getattr(self, "_s", None):
            self._lib.snu_server_destroy(self._s)
            self._s = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factor(self, rowptr, colidx, vals):
        """Construct + factorize a new matrix; returns (matrix id, request id)."""
        rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        ci = np.ascontiguousarray(colidx, dtype=np.int32)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        n, nnz = len(rp) - 1, len(ci)
        m, r = C.c_int64(), C.c_int64()
        self._check(self._lib.snu_server_factor(
            self._s, n, nnz, rp.ctypes.data_as(_I), ci.ctypes.data_as(_I),
            v.ctypes.data_as(_D), C.byref(m), C.byref(r)))
        self._n[m.value] = (n, nnz)
        return m.value, r.value

    def refactor(self, matrix, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        if len(v) != self._n[matrix][1]:
            raise SnuError(1, "values do not match the pattern's nnz")
        r = C.c_int64()
        self._check(self._lib.snu_server_refactor(
            self._s, matrix, v.ctypes.data_as(_D), C.byref(r)))
        return r.value

    def solve(self, matrix, B, out=None):
        """Submits X = A^-1 B; returns (request id, X).  X is filled when the
        request completes (see :meth:`poll`)."""
        n = self._n[matrix][0]
        B = np.asarray(B, dtype=np.float64)
        one = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(n, -1))
        nrhs = Bf.shape[1]
        X = out if out is not None else np.empty((n, nrhs), order="F")
        if X.shape != (n, nrhs) or not X.flags.f_contiguous:
            raise SnuError(1, "out must be a Fortran-ordered (n, nrhs) array")
        r = C.c_int64()
        self._check(self._lib.snu_server_solve(
            self._s, matrix, Bf.ctypes.data_as(_D), X.ctypes.data_as(_D),
            nrhs, n, C.byref(r)))
        self._keep[r.value] = X
        return r.value, (X[:, 0] if one else X)

    def release(self, matrix):
        r = C.c_int64()
        self._check(self._lib.snu_server_release(self._s, matrix, C.byref(r)))
        return r.value

    def poll(self, wait_ms=-1, max_items=256):
        """Completions as dicts (oldest first).  wait_ms=-1 waits for one
        completion or until nothing is outstanding; 0 does not wait."""
        arr = (_Completion * max_items)()
        cnt = C.c_int()
        self._check(self._lib.snu_server_poll(self._s, arr, max_items,
                                              C.byref(cnt), wait_ms))
        out = []
        for c in arr[:cnt.value]:
            self._keep.pop(c.request, None)
            out.append(dict(request=c.request, matrix=c.matrix,
                            type=REQUEST_TYPES[c.type], status=c.status,
                            queue_s=c.queue_s, service_s=c.service_s,
                            latency_s=c.latency_s,
                            backward_error=c.backward_error,
                            ir_iters=c.ir_iters,
                            plan_reused=bool(c.plan_reused)))
        return out

    def drain(self):
        """Waits for every outstanding request; returns their completions."""
        out = []
        while True:
            got = self.poll(wait_ms=-1)
            if not got:
                st = self.stats()
                if st["queued"] == 0 and st["running"] == 0:
                    return out + self.poll(wait_ms=0)
            out += got

    def stats(self):
        s = _ServerStats()
        self._check(self._lib.snu_server_get_stats(self._s, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _ServerStats._fields_
                if k != "reserved"}
