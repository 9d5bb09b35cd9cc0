"""ORACLE — test infrastructure only (never imported by the product path).

FP64 sparse direct solver standing in for `faer::sparse::sp_cholesky(Side::Lower)`
as called by FerriX's DirectSolver (src/solver/solvers/direct.rs:19-55).
faer 0.23.2 is a third-party crate that is not vendored with the reference;
this file restates the published multifrontal Cholesky algorithm
(Duff & Reid 1983; Liu 1992, "The multifrontal method for sparse matrix
solution: theory and practice") with a geometric nested-dissection ordering
(George 1973) built from element centroids:

  * ordering: recursive median bisection of the element set along its longest
    centroid extent; the separator is the set of nodes shared by both halves;
    leaves hold the remaining nodes of small element groups;
  * symbolic: the assembly tree is the dissection tree; the update structure of
    a tree node is (adjacency of its variables  U  children's structures)
    restricted to variables eliminated later;
  * numeric: per tree node a dense frontal matrix receives the original
    entries of its columns and the children's update matrices (extend-add),
    then LAPACK dpotrf / BLAS dtrsm / dsyrk perform the partial factorisation;
  * solve: forward substitution in postorder, backward in reverse order.

A direct solve is exact up to rounding, so it reproduces faer's solution to
~1e-13 relative on the penalised stiffness systems used here. A failed
factorisation raises FerrixError("NumericalError", ... rigid body modes ...),
like direct.rs:46-50.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.linalg import blas, lapack, solve_triangular

from .inp import FerrixError


def _elem_csr(conn_groups, n_nodes):
    ptr = [np.zeros(1, dtype=np.int64)]
    idx = []
    total = 0
    for conn in conn_groups:
        e, npe = conn.shape
        ptr.append(total + npe * np.arange(1, e + 1, dtype=np.int64))
        idx.append(conn.reshape(-1).astype(np.int64))
        total += e * npe
    eptr = np.concatenate(ptr)
    eidx = np.concatenate(idx) if idx else np.zeros(0, dtype=np.int64)
    return eptr, eidx


class MultifrontalCholesky:
    def __init__(self, xyz: np.ndarray, conn_groups, leaf_elems: int = 48):
        n = xyz.shape[0]
        self.n_nodes = n
        eptr, eidx = _elem_csr(conn_groups, n)
        ne = len(eptr) - 1
        counts = np.diff(eptr)
        eid_of = np.repeat(np.arange(ne), counts)
        cent = np.zeros((ne, 3))
        for d in range(3):
            cent[:, d] = np.bincount(eid_of, weights=xyz[eidx, d], minlength=ne) / np.maximum(counts, 1)
        E = sp.csr_matrix((np.ones(len(eidx)), eidx, eptr), shape=(ne, n))
        self._E = E
        A = (E.T @ E).tocsr()
        A.sort_indices()
        self.adj = A

        assigned = np.zeros(n, dtype=bool)
        self.vars = []       # list of node arrays (elimination order within node)
        self.children = []   # list of child index lists

        def nodes_of(elems):
            if len(elems) == 0:
                return np.zeros(0, dtype=np.int64)
            return np.unique(E[elems].indices)

        # iterative post-order dissection (explicit stack; depth is small but be safe)
        def dissect(elems):
            stack = [("enter", elems, None)]
            results = []
            while stack:
                op, el, extra = stack.pop()
                if op == "enter":
                    nodes = nodes_of(el)
                    nodes = nodes[~assigned[nodes]]
                    if len(el) <= leaf_elems or len(nodes) <= 3 * 20:
                        assigned[nodes] = True
                        self.vars.append(nodes)
                        self.children.append([])
                        results.append(len(self.vars) - 1)
                        continue
                    c = cent[el]
                    axis = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
                    order = np.argsort(c[:, axis], kind="stable")
                    half = len(el) // 2
                    L, R = el[order[:half]], el[order[half:]]
                    sep = np.intersect1d(nodes_of(L), nodes_of(R), assume_unique=True)
                    sep = sep[~assigned[sep]]
                    assigned[sep] = True
                    stack.append(("exit", None, sep))
                    stack.append(("enter", R, None))
                    stack.append(("enter", L, None))
                else:
                    right = results.pop()
                    left = results.pop()
                    self.vars.append(extra)
                    self.children.append([left, right])
                    results.append(len(self.vars) - 1)
            return results.pop()

        root = dissect(np.arange(ne))
        orphans = np.nonzero(~assigned)[0]
        if len(orphans):
            assigned[orphans] = True
            self.vars.append(orphans)
            self.children.append([root])
            root = len(self.vars) - 1
        self.root = root
        nt = len(self.vars)
        pos = np.empty(n, dtype=np.int64)
        start = np.zeros(nt + 1, dtype=np.int64)
        p = 0
        for t in range(nt):  # creation order is already a post-order
            v = self.vars[t]
            pos[v] = np.arange(p, p + len(v))
            p += len(v)
            start[t + 1] = p
        self.pos = pos
        self.start = start
        # symbolic: struct(t) sorted by position
        struct = []
        for t in range(nt):
            v = self.vars[t]
            end = start[t + 1]
            cand = [A[v].indices] + [struct[c] for c in self.children[t]]
            cand = np.unique(np.concatenate(cand)) if cand else np.zeros(0, dtype=np.int64)
            cand = cand[pos[cand] >= end]
            struct.append(cand[np.argsort(pos[cand], kind="stable")])
        self.struct = struct
        self.fronts = []
        dofs = lambda nodes: (3 * np.asarray(nodes, dtype=np.int64)[:, None] + np.arange(3)).reshape(-1)
        for t in range(nt):
            self.fronts.append((dofs(self.vars[t]), dofs(struct[t])))
        self.L = None

    def stats(self):
        f = [(len(a), len(b)) for a, b in self.fronts]
        nnzL = sum(n1 * (n1 + 1) // 2 + n1 * n2 for n1, n2 in f)
        flops = sum(n1 ** 3 / 3 + n1 ** 2 * n2 + n1 * n2 ** 2 for n1, n2 in f)
        return {"tree_nodes": len(f), "max_front": max(a + b for a, b in f), "nnz_L": nnzL, "flops": flops}

    def factor(self, K: sp.csr_matrix) -> None:
        K = K.tocsr()
        n = K.shape[0]
        loc = np.full(n, -1, dtype=np.int64)
        updates = {}
        self.L = [None] * len(self.fronts)
        for t, (vd, sd) in enumerate(self.fronts):
            n1, n2 = len(vd), len(sd)
            m = n1 + n2
            fd = np.concatenate([vd, sd])
            loc[fd] = np.arange(m)
            F = np.zeros((m, m), order="F")
            sub = K[vd].tocoo()
            lj = loc[sub.col]
            keep = lj >= sub.row  # lower triangle, skipping already-eliminated variables (loc < 0)
            F[lj[keep], sub.row[keep]] += sub.data[keep]
            for c in self.children[t]:
                if c not in updates:  # child with an empty update structure
                    continue
                U, csd = updates.pop(c)
                li = loc[csd]
                if len(li) and li[-1] - li[0] == len(li) - 1:
                    F[li[0]:li[-1] + 1, li[0]:li[-1] + 1] += U
                else:
                    F[np.ix_(li, li)] += U
                del U
            loc[fd] = -1
            F11 = np.asfortranarray(F[:n1, :n1])
            L11, info = lapack.dpotrf(F11, lower=1, clean=1, overwrite_a=1)
            if info != 0:
                raise FerrixError("NumericalError",
                                  f"Cholesky factorization failed: not positive definite (pivot {info}). "
                                  "Check for rigid body modes!")
            if n2:
                F21 = np.asfortranarray(F[n1:, :n1])
                L21 = blas.dtrsm(1.0, L11, F21, side=1, lower=1, trans_a=1, overwrite_b=1)
                F22 = np.asfortranarray(F[n1:, n1:])
                U = blas.dsyrk(-1.0, L21, beta=1.0, c=F22, lower=1, overwrite_c=1)
                U = np.tril(U)
                updates[t] = (U, sd)
            else:
                L21 = np.zeros((0, n1))
            self.L[t] = (L11, L21)
            del F

    def solve(self, b: np.ndarray) -> np.ndarray:
        y = np.array(b, dtype=np.float64, copy=True)
        for t, (vd, sd) in enumerate(self.fronts):
            L11, L21 = self.L[t]
            yv = solve_triangular(L11, y[vd], lower=True, check_finite=False)
            y[vd] = yv
            if len(sd):
                y[sd] -= L21 @ yv
        x = y
        for t in range(len(self.fronts) - 1, -1, -1):
            vd, sd = self.fronts[t]
            L11, L21 = self.L[t]
            rhs = x[vd]
            if len(sd):
                rhs = rhs - L21.T @ x[sd]
            x[vd] = solve_triangular(L11, rhs, lower=True, trans="T", check_finite=False)
        return x
