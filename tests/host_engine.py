"""Test infrastructure: a host (numpy) restatement of the multifrontal
numerics behind the distributed phases of snusolver_b200.dist.

It plays the CUDA engine's part for the CPU tests of the distributed driver:
the same front plan (read back from the library's host analysis), the same
subtree / shared split, the same exchange buffers (shared fronts in front
order, each ld x (p + q) column-major; their solve work vectors, each
(p + q) x nrhs) and the same phases.  Numerics per front: LU without
pivoting of the pivot block with the reference's static pivot on leaf
pivots (|p| < eps -> +-eps, kernel_sparse.cu:742-749), L21 / U12 and the
Schur update in one right-looking sweep, the update added into the parent
through the child's index map (the reference's core_GEMM + core_reduction,
kernel_sparse.cu:54-90, 953-994).
"""
import numpy as np

import snusolver_b200 as snu
from snusolver_b200.dist import subtree_owner


class HostEngine:
    def __init__(self, rank, world, nleaves=8, precision=snu.FP64,
                 pivot_eps=1e-15):
        self.rank, self.world = rank, world
        self.nleaves = nleaves
        self.precision = precision
        self.eps = pivot_eps

    # ----------------------------------------------------------- set-up
    def construct(self, rowptr, colidx, vals):
        s = snu.Solver(nleaves=self.nleaves).analyze(rowptr, colidx).plan()
        self.fp = fp = s.front_plan()
        s.close()
        self.rowptr = np.asarray(rowptr, np.int64)
        self.colidx = np.asarray(colidx, np.int64)
        self.vals = np.asarray(vals, np.float64)
        self.n = len(rowptr) - 1
        nf = len(fp["p"])
        owner = np.array([subtree_owner(int(b), self.world) for b in fp["block"]])
        self.shared = owner < 0
        self.own = (owner == self.rank) if self.rank is not None else ~self.shared
        self.order = sorted(range(nf), key=lambda f: (fp["level"][f], f))
        self.children = [[] for _ in range(nf)]
        for f in range(nf):
            if fp["parent"][f] >= 0:
                self.children[fp["parent"][f]].append(f)
        # front of every assembly entry (fronts are laid out by offset)
        offs = fp["offset"]
        srt = np.argsort(offs, kind="stable")
        idx = np.searchsorted(offs[srt], fp["asm_pos"], side="right") - 1
        self.asm_front = srt[idx]
        self.arena = np.zeros(fp["arena"])

    def _front(self, f):
        """Column-major view (dim x dim) of front f in the arena."""
        fp = self.fp
        p, q, ld, o = fp["p"][f], fp["q"][f], fp["ld"][f], fp["offset"][f]
        dim = p + q
        return self.arena[o:o + ld * dim].reshape(dim, ld).T[:dim, :]

    def _gidx(self, f):
        fp = self.fp
        o = fp["idx_offset"][f]
        return fp["gidx"][o:o + fp["p"][f] + fp["q"][f]]

    def _rel(self, f):
        fp = self.fp
        o = fp["rel_offset"][f]
        return fp["rel"][o:o + fp["q"][f]]

    # ---------------------------------------------------- factorization
    def _factor_front(self, f):
        fp = self.fp
        F = self._front(f)
        p, q = fp["p"][f], fp["q"][f]
        guard = fp["guard"][f] != 0
        for k in range(p):
            piv = F[k, k]
            if guard and abs(piv) < self.eps:
                piv = -self.eps if piv < 0 else self.eps
                F[k, k] = piv
            F[k + 1:, k] *= 1.0 / piv
            F[k + 1:, k + 1:] -= np.outer(F[k + 1:, k], F[k, k + 1:])
        if q and fp["parent"][f] >= 0:
            P = self._front(fp["parent"][f])
            r = self._rel(f)
            P[np.ix_(r, r)] += F[p:, p:]

    def factor_phase(self, phase):
        fp = self.fp
        if phase in (0, 1):
            self.arena[:] = 0
            keep = self.own | (self.shared & (self.rank in (0, None)))
            sel = keep[self.asm_front]
            self.arena[fp["asm_pos"][sel]] = self.vals[fp["asm_val"][sel]]
        work = self.own if phase == 1 else (self.shared if phase == 2 else
                                            np.ones_like(self.own))
        for f in self.order:
            if work[f]:
                self._factor_front(f)

    def buffer(self, kind, nrhs=0):
        fp = self.fp
        tot = 0
        for f in range(len(fp["p"])):
            if self.shared[f]:
                dim = fp["p"][f] + fp["q"][f]
                tot += fp["ld"][f] * dim if kind == 0 else dim * nrhs
        return np.zeros(max(tot, 1))

    def copy(self, kind, direction, nrhs, buf):
        fp = self.fp
        at = 0
        for f in range(len(fp["p"])):
            if not self.shared[f]:
                continue
            dim = fp["p"][f] + fp["q"][f]
            if kind == 0:
                o, ln = fp["offset"][f], fp["ld"][f] * dim
                if direction == 0:
                    buf[at:at + ln] = self.arena[o:o + ln]
                else:
                    self.arena[o:o + ln] = buf[at:at + ln]
            else:
                ln = dim * nrhs
                if direction == 0:
                    buf[at:at + ln] = self.W[f].reshape(-1, order="F")
                else:
                    self.W[f][:] = buf[at:at + ln].reshape(dim, nrhs, order="F")
            at += ln

    # ------------------------------------------------------------ solve
    def columns(self, B):
        return np.ascontiguousarray(np.asarray(B, np.float64).T)

    def zeros_like(self, dB):
        return np.zeros_like(dB)

    def _forward(self, work, init, b):
        fp = self.fp
        for f in self.order:
            p = fp["p"][f]
            if work[f] and init:
                self.W[f][:] = 0
                self.W[f][:p] = b[self._gidx(f)[:p]]
            for c in self.children[f]:
                if work[c] and fp["q"][c]:
                    self.W[f][self._rel(c)] += self.W[c][fp["p"][c]:]
            if not work[f]:
                continue
            F = self._front(f)
            L11 = np.tril(F[:p, :p], -1) + np.eye(p)
            y = np.linalg.solve(L11, self.W[f][:p]) if p else self.W[f][:0]
            self.Y[f] = y
            self.W[f][p:] -= F[p:, :p] @ y

    def _backward(self, work, X):
        fp = self.fp
        for f in reversed(self.order):
            if not work[f]:
                continue
            p = fp["p"][f]
            g = self._gidx(f)
            F = self._front(f)
            w = self.Y[f] - F[:p, p:] @ X[g[p:]]
            U11 = np.triu(F[:p, :p])
            X[g[:p]] = np.linalg.solve(U11, w) if p else w

    def solve_phase(self, phase, dB, dX):
        fp = self.fp
        b = dB.T  # n x k views
        X = dX.T
        k = b.shape[1]
        nf = len(fp["p"])
        if phase == 1:
            self.W = [np.zeros((fp["p"][f] + fp["q"][f], k)) for f in range(nf)]
            self.Y = [None] * nf
            if self.rank in (0, None):
                for f in range(nf):
                    if self.shared[f]:
                        p = fp["p"][f]
                        self.W[f][:p] = b[self._gidx(f)[:p]]
            self._forward(self.own, True, b)
        else:
            self._forward(self.shared, False, b)
            self._backward(self.shared, X)
            self._backward(self.own, X)
            keep = np.zeros(self.n, bool)
            for f in range(nf):
                if self.own[f] or (self.shared[f] and self.rank in (0, None)):
                    keep[self._gidx(f)[:fp["p"][f]]] = True
            X[~keep] = 0.0

    def residual(self, dB, dX, dR):
        n = self.n
        rows = np.repeat(np.arange(n), np.diff(self.rowptr))
        worst = 0.0
        anorm = np.zeros(n)
        np.add.at(anorm, rows, np.abs(self.vals))
        an = anorm.max()
        for c in range(dB.shape[0]):
            Ax = np.zeros(n)
            np.add.at(Ax, rows, self.vals * dX[c][self.colidx])
            dR[c] = dB[c] - Ax
            den = an * np.abs(dX[c]).max() + np.abs(dB[c]).max()
            worst = max(worst, np.abs(dR[c]).max() / den if den else 0.0)
        return worst

    def to_host(self, dX):
        return dX.T.copy()
