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
                ("gemm_split", C.c_int), ("reserved", C.c_int * 7)]


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

    def __init__(self, device=0, slots=8, mem_budget=120 << 30, nleaves=8,
                 precision=FP32_IR, ir_tol=1e-10, ir_max_iter=10,
                 plan_cache=64, gemm_split=None):
        self._lib = _bind(load_library())
        o = _ServerOpts()
        self._lib.snu_server_default_opts(C.byref(o))
        o.device, o.slots, o.mem_budget = device, slots, mem_budget
        o.nleaves, o.precision = nleaves, precision
        o.ir_tol, o.ir_max_iter, o.plan_cache = ir_tol, ir_max_iter, plan_cache
        if gemm_split is not None:  # (default: the library's, TF32x3)
            o.gemm_split = gemm_split
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
        self._keep[r.value] = (Bf, X)  # both live until completion
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


# ---------------------------------------------------------------- workload
SERVE_SHAPES = ((100, 100), (224, 224), (400, 400), (707, 707),
                (22, 22, 22), (37, 37, 37), (54, 54, 54), (79, 79, 79))


def _laplacian(shape, seed):
    from . import generators
    if len(shape) == 2:
        return generators.laplace2d_lognormal(shape[0], shape[1], seed=seed)
    return generators.laplace3d_lognormal(*shape, seed=seed)


def rescale_values(rowptr, colidx, vals, rng, lo=0.5, hi=2.0):
    """Refactor values: every off-diagonal entry times U[lo, hi]; each
    diagonal entry scaled with its row's off-diagonal sum, so the row keeps
    its diagonal dominance (a no-pivot LU of a Laplacian whose entries are
    all rescaled independently can break down, in the reference too)."""
    rowptr = np.asarray(rowptr)
    n = len(rowptr) - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    off = np.asarray(colidx) != rows
    v = np.array(vals, dtype=np.float64)
    old = np.zeros(n)
    np.add.at(old, rows[off], np.abs(v[off]))
    v[off] *= rng.uniform(lo, hi, int(off.sum()))
    new = np.zeros(n)
    np.add.at(new, rows[off], np.abs(v[off]))
    ratio = np.where(old > 0, new / np.where(old > 0, old, 1.0), 1.0)
    v[~off] *= ratio[rows[~off]]
    return v


def run_stream(rate=200.0, duration=5.0, seed=5, mix=(0.05, 0.10, 0.85),
               slots=8, mem_budget=120 << 30, max_resident=4, warm=True,
               shapes=SERVE_SHAPES, device=0):
    """The serving workload: Poisson arrivals (mean `rate` per second, seeded)
    for `duration` seconds, mixing new-factor requests on 2D / 3D lognormal
    Laplacians (n from 1e4 to 5e5, shapes from `shapes`), refactor requests
    (off-diagonal values times U[0.5, 2] per entry, see rescale_values)
    and solve requests (1-64 right-hand
    sides) against resident matrices, FP32 factors + FP64 refinement to
    1e-10.  At most `max_resident` matrices are kept; the oldest is released
    when a factor request would pass that.  With `warm`, one matrix of every
    shape is factored (and released) first, so host plans are cached.
    Returns per-type p50 / p99 latency, throughput and failure counts."""
    import time
    rng = np.random.default_rng(seed)
    # the request list, drawn up front
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        u = rng.uniform()
        kind = 0 if u < mix[0] else (1 if u < mix[0] + mix[1] else 2)
        reqs.append((t, kind, int(rng.integers(len(shapes))),
                     int(rng.integers(1, 65)), int(rng.integers(1 << 30))))
    mats_cache = {}

    def matrix(k):
        if k not in mats_cache:
            mats_cache[k] = _laplacian(shapes[k], seed=1000 + k)
        return mats_cache[k]

    for k in range(len(shapes)):
        matrix(k)
    # right-hand sides and refactor values drawn before the clock starts:
    # per shape a pool of 64 RHS columns and 4 rescaled value sets
    prng = np.random.default_rng(seed + 1)
    rhs_pool = {k: np.asfortranarray(prng.uniform(-1.0, 1.0, size=(
        len(mats_cache[k][0]) - 1, 64))) for k in range(len(shapes))}
    val_pool = {k: [rescale_values(*mats_cache[k], prng) for _ in range(4)]
                for k in range(len(shapes))}
    out = {"requests": len(reqs), "rate": rate, "duration_s": duration,
           "slots": slots, "mix": list(mix)}
    with Server(slots=slots, mem_budget=mem_budget, device=device) as s:
        if warm:
            t0 = time.perf_counter()
            ids = [s.factor(*matrix(k))[0] for k in range(len(shapes))]
            s.drain()
            for m in ids:
                s.release(m)
            s.drain()
            out["warm_s"] = time.perf_counter() - t0
        resident = []   # (matrix id, shape index, values)
        keep = []
        lag = []
        start = time.perf_counter()
        for (ta, kind, k, nrhs, rs) in reqs:
            now = time.perf_counter() - start
            if ta > now:
                time.sleep(ta - now)
            lag.append(time.perf_counter() - start - ta)
            r2 = np.random.default_rng(rs)
            if kind == 0 or not resident:
                rp, ci, v = matrix(k)
                v = v * r2.uniform(0.5, 2.0) if kind == 0 else v
                m, _ = s.factor(rp, ci, v)
                resident.append((m, k, v))
                if len(resident) > max_resident:
                    old = resident.pop(0)
                    s.release(old[0])
            elif kind == 1:
                j = int(r2.integers(len(resident)))
                m, k2, v = resident[j]
                v2 = val_pool[k2][int(r2.integers(4))]
                s.refactor(m, v2)
                resident[j] = (m, k2, v2)
            else:
                j = int(r2.integers(len(resident)))
                m, k2, _ = resident[j]
                c0 = int(r2.integers(0, 65 - nrhs))
                B = rhs_pool[k2][:, c0:c0 + nrhs]
                _, X = s.solve(m, B)
                keep.append(X)
        comps = s.drain()
        end = time.perf_counter()
        st = s.stats()
    done = comps
    out["completed"] = len(done)
    out["wall_s"] = end - start
    out["throughput_rps"] = len([c for c in done if c["type"] != "release"]) / (end - start)
    out["peak_device_gb"] = st["peak_bytes"] / 1e9
    out["submit_lag_p99_ms"] = float(np.percentile(lag, 99) * 1e3) if lag else 0.0
    for typ in ("factor", "refactor", "solve"):
        lat = np.array([c["latency_s"] for c in done if c["type"] == typ
                        and c["status"] == 0])
        svc = np.array([c["service_s"] for c in done if c["type"] == typ
                        and c["status"] == 0])
        bad = [c for c in done if c["type"] == typ and c["status"] != 0]
        if len(lat):
            out[typ] = {"n": int(len(lat)),
                        "p50_ms": float(np.percentile(lat, 50) * 1e3),
                        "p99_ms": float(np.percentile(lat, 99) * 1e3),
                        "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
                        "failed": len(bad)}
        else:
            out[typ] = {"n": 0, "failed": len(bad)}
    be = [c["backward_error"] for c in done if c["type"] == "solve"
          and c["status"] == 0]
    out["solve_worst_backward_error"] = float(max(be)) if be else None
    out["statuses"] = sorted({int(c["status"]) for c in done})
    return out


if __name__ == "__main__":
    # python -m snusolver_b200.server [--rate R] [--duration S] [--slots K]
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    a = ap.parse_args()
    print(json.dumps(run_stream(rate=a.rate, duration=a.duration, seed=a.seed,
                                slots=a.slots,
                                mem_budget=int(a.budget_gb * (1 << 30)))))
