"""Separator-tree distribution of the factorize-and-solve path over ranks.

The reference runs one MPI rank per leaf of the separator tree: each rank
factors its leaf, the ranks reduce their Schur complements pairwise up the
tree (core_reduction, kernel_sparse.cu:54-90; reduction / reduction_gpu,
SnuMat_factorize.cu:29-124) and the solve scatters and reduces the
right-hand side the same way (scatter_b, SnuMat_factorize.cu:126-187).

Here a world of W ranks (one GPU each, W a power of two <= nleaves) splits
the front tree the same way: rank d factors every front of the subtree of
heap node 2W - 1 - d (its leaves' supernodes and the separators below that
node; with W = nleaves exactly the leaf of the reference's rank d); the
separators above (heap nodes 1 .. W-1) are shared.

* factorize: phase 1 on every rank (its subtree; the updates its fronts
  send to the shared fronts accumulate in its copy of them, and rank 0 alone
  assembles the shared fronts' original values), one all-reduce (sum) of
  the shared fronts, phase 2 on every rank (the shared fronts, the same on
  all ranks).
* solve (columns in groups of up to 16): phase 1 (the subtree's forward
  sweep; rank 0 alone loads B into the shared fronts), one all-reduce of the
  shared fronts' work vectors, phase 2 (shared fronts forward and back, the
  subtree back; rows of X other ranks own zeroed), one all-reduce of X.
  FP32 factors are refined in FP64 against the original matrix
  (snu_residual_device) until the backward error reaches ir_tol.

The collectives are torch.distributed's (NCCL between GPUs; gloo, through
host copies, for CPU tests and for ranks sharing a GPU).  The device steps
between them are the C-ABI calls snu_dist_* of the engine; ``engine`` may
be any object with the same methods (the CPU tests pass a host restatement
of the front numerics).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import FP32_IR, FP64, SnuError, Solver

__all__ = ["DeviceEngine", "DistSolver", "subtree_owner"]


def subtree_owner(block, world):
    """Rank whose subtree holds heap block `block`, -1 for the shared top
    blocks (block < world).  Rank d owns the subtree of heap node
    2 world - 1 - d, so with one rank per leaf it owns the leaf of the
    reference's rank d (SnuMat.cu:24-30: leaf 2 np - 1 - rank)."""
    if block < world:
        return -1
    while block >= 2 * world:
        block //= 2
    return 2 * world - 1 - block


def _bind(lib):
    sig = {
        "snu_dist_init": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "snu_dist_factorize": (C.c_int, [C.c_void_p, C.c_int]),
        "snu_dist_buffer": (C.c_int, [C.c_void_p, C.c_int, C.c_int,
                                      C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int)]),
        "snu_dist_copy": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                    C.c_void_p]),
        "snu_dist_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_int, C.c_int]),
        "snu_residual_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_int,
                                          C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class DeviceEngine:
    """The CUDA engine of one rank through the C-ABI (the product path)."""

    def __init__(self, rank, world, nleaves=8, precision=FP64, device=0,
                 ir_tol=1e-10, ir_max_iter=10):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.s = Solver(nleaves=nleaves, precision=precision, device=device,
                        ir_tol=ir_tol, ir_max_iter=ir_max_iter)
        self.lib = _bind(self.s._lib)
        self.s._check(self.lib.snu_dist_init(self.s._h, rank, world))
        self.precision = precision
        self.n = 0

    def _check(self, st):
        return self.s._check(st)

    def construct(self, rowptr, colidx, vals):
        self.s.construct(rowptr, colidx, vals)
        self.n = self.s.n

    def factor_phase(self, phase):
        self._check(self.lib.snu_dist_factorize(self.s._h, phase))

    def buffer(self, kind, nrhs=0):
        elems, es = C.c_int64(), C.c_int()
        self._check(self.lib.snu_dist_buffer(self.s._h, kind, nrhs,
                                             C.byref(elems), C.byref(es)))
        dt = self.torch.float64 if es.value == 8 else self.torch.float32
        return self.torch.empty(max(elems.value, 1), dtype=dt,
                                device=self.device)

    def copy(self, kind, direction, nrhs, buf):
        self._check(self.lib.snu_dist_copy(self.s._h, kind, direction, nrhs,
                                           C.c_void_p(buf.data_ptr())))

    def columns(self, B):
        """Device copy of host columns (n x k, FP64), column-major."""
        return self.torch.from_numpy(
            np.ascontiguousarray(np.asarray(B, np.float64).T)).to(self.device)

    def zeros_like(self, dB):
        return self.torch.zeros_like(dB)

    def solve_phase(self, phase, dB, dX):
        k = dB.shape[0]
        self._check(self.lib.snu_dist_solve(self.s._h, phase,
                                            C.c_void_p(dB.data_ptr()),
                                            C.c_void_p(dX.data_ptr()), k,
                                            self.n))

    def residual(self, dB, dX, dR):
        be = C.c_double()
        self._check(self.lib.snu_residual_device(
            self.s._h, C.c_void_p(dB.data_ptr()), C.c_void_p(dX.data_ptr()),
            C.c_void_p(dR.data_ptr()), dB.shape[0], self.n, C.byref(be)))
        return be.value

    def to_host(self, dX):
        self.torch.cuda.synchronize(self.device)
        return dX.cpu().numpy().T.copy()

    def close(self):
        self.s.close()


class DistSolver:
    """One rank of a distributed factorize-and-solve (see the module text).

    group: the torch.distributed process group (None: the default group).
    engine: the device steps (default: this rank's CUDA engine)."""

    def __init__(self, rank, world, nleaves=8, precision=FP64, device=None,
                 ir_tol=1e-10, ir_max_iter=10, group=None, engine=None):
        if world & (world - 1) or not 2 <= world <= nleaves:
            raise SnuError(1, "world must be a power of two, 2..nleaves "
                              "(one rank: snusolver_b200.Solver)")
        self.rank, self.world = rank, world
        self.precision = precision
        self.ir_tol, self.ir_max_iter = ir_tol, ir_max_iter
        self.group = group
        self.eng = engine if engine is not None else DeviceEngine(
            rank, world, nleaves, precision, device if device is not None else 0,
            ir_tol, ir_max_iter)
        self.stats = {}

    # ------------------------------------------------------- collectives
    def _allreduce(self, t):
        """Sum over the ranks, in place (gloo on device tensors: through a
        host copy)."""
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return t
        if getattr(t, "is_cuda", False) and dist.get_backend(self.group) == "gloo":
            h = t.cpu()
            dist.all_reduce(h, group=self.group)
            t.copy_(h)
        elif isinstance(t, np.ndarray):
            h = torch.from_numpy(t)
            dist.all_reduce(h, group=self.group)
        else:
            dist.all_reduce(t, group=self.group)
        return t

    # ------------------------------------------------------------ phases
    def construct(self, rowptr, colidx, vals):
        self.eng.construct(rowptr, colidx, vals)
        self.n = len(rowptr) - 1
        return self

    def factorize(self):
        self.eng.factor_phase(1)
        buf = self.eng.buffer(0)
        self.eng.copy(0, 0, 0, buf)
        self._allreduce(buf)
        self.eng.copy(0, 1, 0, buf)
        self.eng.factor_phase(2)
        return self

    def _solve_group(self, dB):
        """One distributed solve of up to 16 device columns (no refinement)."""
        k = dB.shape[0]
        dX = self.eng.zeros_like(dB)
        self.eng.solve_phase(1, dB, dX)
        buf = self.eng.buffer(1, k)
        self.eng.copy(1, 0, k, buf)
        self._allreduce(buf)
        self.eng.copy(1, 1, k, buf)
        self.eng.solve_phase(2, dB, dX)
        self._allreduce(dX)
        return dX

    def solve(self, B):
        """X = A^-1 B (host array, n or n x k); every rank returns all of X."""
        B = np.asarray(B, np.float64)
        vec = B.ndim == 1
        Bm = B.reshape(self.n, -1)
        out = np.empty_like(Bm, order="F")
        worst, iters = 0.0, 0
        for c0 in range(0, Bm.shape[1], 16):
            dB = self.eng.columns(Bm[:, c0:c0 + 16])
            dX = self._solve_group(dB)
            dR = self.eng.zeros_like(dB)
            be = self.eng.residual(dB, dX, dR)
            it = 0
            if self.precision == FP32_IR:
                # FP64 refinement against the original matrix: every rank
                # holds the same X and R, so all take the same steps
                prev, stagnant = float("inf"), 0
                while be > self.ir_tol:
                    if it >= self.ir_max_iter or stagnant >= 2:
                        raise SnuError(7, f"refinement stopped at backward "
                                          f"error {be:.3e}")
                    stagnant = stagnant + 1 if be > 0.5 * prev else 0
                    prev = be
                    dD = self._solve_group(dR)
                    dX += dD
                    be = self.eng.residual(dB, dX, dR)
                    it += 1
            worst, iters = max(worst, be), max(iters, it)
            out[:, c0:c0 + 16] = self.eng.to_host(dX)
        self.stats = {"backward_error": worst, "ir_iters": iters}
        return out[:, 0] if vec else out

    def close(self):
        if hasattr(self.eng, "close"):
            self.eng.close()
