"""TDVP with a real prefactor on the CPU: the oracle for the device's ``dmrg_tdvp`` (test
infrastructure only).

Restates ``algs/time.jl:182-203`` (``krylovTimeEvol``), ``:205-209`` (``OC_update``, the zero-site
Heff), ``:211-286`` (``tdvp``) and ``:288-363`` (``tdvp_twosite``) with 0-based indices, on dense
tensors whose bond states carry integer charges (as ``oracle/dmrg3s.py``), so that the truncation
is grouped by charge exactly as the block-sparse device code groups it.

krylovTimeEvol: Lanczos from the normalised start with r vectors (full re-orthogonalisation,
breakdown below betatest), T the tridiagonal, the result sum_k (exp(tau T) e_1)_k V_k (the first
column of I + T when those coefficients sum to zero), and En = the lowest eigenvalue of T.
Truncation: svd with m, minm, cutoff and weights relative to the total (the default mag = 0).
One call = L-1 steps from the centre, turning at the edge. The single-site reference runs L steps
and reads past the chain's end on the last one; this restatement stops at the edge (documented in
the device header as well). Both forms evolve the bond and the site with the same tau.
"""
from __future__ import annotations

import numpy as np

from .dmrg import Lupdate, Rupdate
from .dmrg3s import _add, _groups, _trunc, heff1


def heff2(L, R, AA, W1, W2):
    """The two-site Heff on AA[a,s1,s2,d] (make2site / joinedtwosite_update)."""
    LA = np.tensordot(L, AA, axes=(2, 0))                     # [a, w, s1, s2, d]
    LAW = np.tensordot(LA, W1, axes=((1, 2), (0, 1)))         # [a, s2, d, t1, w']
    LAWW = np.tensordot(LAW, W2, axes=((4, 1), (0, 1)))       # [a, d, t1, t2, w'']
    out = np.tensordot(LAWW, R, axes=((1, 4), (0, 1)))        # [a, t1, t2, d']
    return out


def heff0(L, R, C):
    """``OC_update``: L[a,w,b] C[b,c] R[c,w,d] -> [a,d]."""
    LC = np.tensordot(L, C, axes=(2, 0))                      # [a, w, c]
    return np.tensordot(LC, R, axes=((1, 2), (1, 0)))         # [a, d]


def krylov_exp(apply, x, r, tau, betatest=1e-10):
    V = [x / np.linalg.norm(x)]
    alphas, betas = [], []
    for jj in range(max(2, r)):
        w = apply(V[jj])
        a = float(np.sum(V[jj] * w))
        alphas.append(a)
        if jj == max(2, r) - 1:
            break
        w = w - a * V[jj]
        if jj > 0:
            w = w - betas[jj - 1] * V[jj - 1]
        for _ in range(2):
            for u in V:
                w = w - float(np.sum(u * w)) * u
        b = float(np.linalg.norm(w))
        if b <= betatest:
            break
        betas.append(b)
        V.append(w / b)
    n = len(alphas)
    T = np.diag(alphas) + np.diag(betas[:n - 1], 1) + np.diag(betas[:n - 1], -1)
    lam, U = np.linalg.eigh(T)
    coef = U @ (np.exp(tau * lam) * U[0, :])
    if float(np.sum(coef)) == 0.0:
        coef = (np.eye(n) + T)[:, 0]
    out = coef[0] * V[0]
    for k in range(1, n):
        out = out + coef[k] * V[k]
    return out, float(lam[0])


class StateT:
    def __init__(self, psi, mpo, phys, bond_labels, oc=0):
        self.psi = [np.array(a, dtype=float) for a in psi]
        self.mpo = mpo
        self.phys = phys
        self.q = [list(map(tuple, b)) for b in bond_labels]
        self.oc = oc
        L = len(psi)
        self.Lenv = [None] * L
        self.Renv = [None] * L
        self.Lenv[0] = np.ones((1, 1, 1))
        self.Renv[L - 1] = np.ones((1, 1, 1))
        for i in range(oc):
            self.Lenv[i + 1] = Lupdate(self.Lenv[i], self.psi[i], self.psi[i], mpo[i])
        for i in range(L - 1, oc, -1):
            self.Renv[i - 1] = Rupdate(self.Renv[i], self.psi[i], self.psi[i], mpo[i])


def _split_rows(M, rlab, P):
    """Groups by row charge, rho = M M^T: (U [rows x k], new labels, truncerr, kept count)."""
    G = [(Q, rows, M[rows] @ M[rows].T) for Q, rows in _groups(rlab)]
    res, terr, D = _trunc(G, P["maxm"], P["minm"], P["cutoff"], P["degen_rtol"])
    k = sum(u.shape[1] for u, _ in res)
    U = np.zeros((M.shape[0], k))
    newq, o = [], 0
    for (Q, rows, _), (u, _) in zip(G, res):
        U[rows, o:o + u.shape[1]] = u
        newq += [Q] * u.shape[1]
        o += u.shape[1]
    return U, newq, terr, len(D)


def _split_cols(M, clab, P):
    """Groups by column charge, rho = M^T M: (V [cols x k], new labels, truncerr, kept count)."""
    G = [(Q, cols, M[:, cols].T @ M[:, cols]) for Q, cols in _groups(clab)]
    res, terr, D = _trunc(G, P["maxm"], P["minm"], P["cutoff"], P["degen_rtol"])
    k = sum(u.shape[1] for u, _ in res)
    V = np.zeros((M.shape[1], k))
    newq, o = [], 0
    for (Q, cols, _), (u, _) in zip(G, res):
        V[cols, o:o + u.shape[1]] = u
        newq += [Q] * u.shape[1]
        o += u.shape[1]
    return V, newq, terr, len(D)


def _norm(A):
    return A / np.linalg.norm(A)


def tdvp_call(S: StateT, P, twosite):
    """One call (L-1 steps). Returns (En, max truncerr, biggest m)."""
    L = len(S.psi)
    psi, mpo, phys = S.psi, S.mpo, S.phys
    tau = P["prefactor"] / (L - 1) / 2 if twosite else P["prefactor"] / L / 2
    j = -1 if S.oc == L - 1 else 1
    r = P["r"]
    En, mt, bm = 0.0, 0.0, 0
    for _ in range(L - 1):
        i = S.oc
        if twosite:
            iL, iR = (i, i + 1) if j > 0 else (i - 1, i)
            AA = np.tensordot(psi[iL], psi[iR], axes=(2, 0))
            a, d1, d2, dd = AA.shape
            new, En = krylov_exp(lambda x: heff2(S.Lenv[iL], S.Renv[iR], x, mpo[iL], mpo[iR]),
                                 AA, r, tau)
            M = _norm(new).reshape(a * d1, d2 * dd)
            if j > 0:
                rlab = [_add(S.q[iL][x], phys[iL][t]) for x in range(a) for t in range(d1)]
                U, newq, terr, k = _split_rows(M, rlab, P)
                psi[iL] = U.reshape(a, d1, -1)
                psi[iR] = _norm((U.T @ M).reshape(-1, d2, dd))
                S.q[iR] = newq
                S.Lenv[iR] = Lupdate(S.Lenv[iL], psi[iL], psi[iL], mpo[iL])
                psi[iR], En = krylov_exp(lambda x: heff1(S.Lenv[iR], S.Renv[iR], x, mpo[iR]),
                                         psi[iR], r, tau)
            else:
                clab = [_add(S.q[iR + 1][y], phys[iR][t], -1) for t in range(d2) for y in range(dd)]
                V, newq, terr, k = _split_cols(M, clab, P)
                psi[iR] = V.T.reshape(-1, d2, dd)
                psi[iL] = _norm((M @ V).reshape(a, d1, -1))
                S.q[iR] = newq
                S.Renv[iL] = Rupdate(S.Renv[iR], psi[iR], psi[iR], mpo[iR])
                psi[iL], En = krylov_exp(lambda x: heff1(S.Lenv[iL], S.Renv[iL], x, mpo[iL]),
                                         psi[iL], r, tau)
        else:
            A = psi[i]
            a, d, c = A.shape
            new, En = krylov_exp(lambda x: heff1(S.Lenv[i], S.Renv[i], x, mpo[i]), A, r, tau)
            new = _norm(new)
            if j > 0:
                M = new.reshape(a * d, c)
                rlab = [_add(S.q[i][x], phys[i][t]) for x in range(a) for t in range(d)]
                U, newq, terr, k = _split_rows(M, rlab, P)
                psi[i] = U.reshape(a, d, -1)
                DV = _norm(U.T @ M)
                S.q[i + 1] = newq
                S.Lenv[i + 1] = Lupdate(S.Lenv[i], psi[i], psi[i], mpo[i])
                DV, En = krylov_exp(lambda x: heff0(S.Lenv[i + 1], S.Renv[i], x), DV, r, tau)
                psi[i + 1] = np.tensordot(DV, psi[i + 1], axes=(1, 0))
            else:
                M = new.reshape(a, d * c)
                clab = [_add(S.q[i + 1][y], phys[i][t], -1) for t in range(d) for y in range(c)]
                V, newq, terr, k = _split_cols(M, clab, P)
                psi[i] = V.T.reshape(-1, d, c)
                UD = _norm(M @ V)
                S.q[i] = newq
                S.Renv[i - 1] = Rupdate(S.Renv[i], psi[i], psi[i], mpo[i])
                UD, En = krylov_exp(lambda x: heff0(S.Lenv[i], S.Renv[i - 1], x), UD, r, tau)
                psi[i - 1] = np.tensordot(psi[i - 1], UD, axes=(2, 0))
        mt = max(mt, terr)
        bm = max(bm, k)
        S.oc += j
        psi[S.oc] = _norm(psi[S.oc])
        if (S.oc == L - 1 and j > 0) or (S.oc == 0 and j < 0):
            j = -j
    return En, mt, bm


def tdvp(psi, mpo, phys, bond_labels, calls=1, prefactor=1.0, m=0, minm=2, cutoff=0.0, r=2,
         twosite=True, degen_rtol=0.0, oc=0):
    """``calls`` successive calls of tdvp_twosite (or tdvp) from a state with centre ``oc``.
    Returns (list of (En, maxtrunc, biggest m) per call, final state)."""
    S = StateT(psi, mpo, phys, bond_labels, oc=oc)
    P = dict(prefactor=prefactor, maxm=m, minm=minm, cutoff=cutoff, r=r, degen_rtol=degen_rtol)
    recs = [tdvp_call(S, P, twosite) for _ in range(calls)]
    return recs, S
