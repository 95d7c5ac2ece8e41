"""Single-site DMRG with subspace expansion ("3S") on the CPU: the oracle for the device's
``dmrg_sweep3s`` (test infrastructure only).

Restates ``algs/DMRG.jl:273-302`` (``Lexpand``, ``Rexpand``, ``alpha_update``), ``:324-360``
(``step3S``), ``:655-671`` (``dmrg3S``) and ``algs/optimizeMPS.jl:503-511`` (``singlesite_update``)
with 0-based indices, on dense tensors whose bond states carry integer charges (U(1)^n; the empty
tuple for a dense MPO). The charges group the truncation exactly as the block-sparse device code
does (one reduced density matrix per charge, global selection over the groups).

One bond step at site i, direction j (iL, iR = i, i+1 for j > 0, i-1, i for j < 0):
  * Lanczos (Krylov dimension ``krylov``, full re-orthogonalisation; 2 = the reference's default
    ``r``) on the single-site effective Hamiltonian L[i] W[i] R[i], from psi[i] normalised;
  * when alpha > noise_incr the tensor is enlarged by alpha times the partial Heff product:
    j > 0: P[a,t,(w',c)] = alpha sum L[a,w,b] A[b,s,c] W[w,s,t,w'] joined to A along its right
    index (new states (w',c) of charge q(c) - r(w')); j < 0: P[(a,w),t,d] = alpha sum
    A[a,s,c] W[w,s,t,w'] R[c,w',d] joined along its left index (charge q(a) - r(w));
  * truncated decomposition of the enlarged tensor through its reduced density matrix (moveR! /
    moveL! with ``condition``, ``lib/MPS/move.jl:124-199``; the truncation measures weights
    relative to the total, ``mag = 0``); the centre moves on: psi[iL] = U, psi[iR] = (U^T M)
    restricted to the original columns times psi[iR] (j > 0), mirrored for j < 0;
  * alpha <- alpha_update(alpha, truncerr, cutoff, E_last_sweep, E, noise_goal, noise_incr).
The truncation error reported is the discarded weight over the total weight.
"""
from __future__ import annotations

import math

import numpy as np

from .dmrg import Lupdate, Rupdate, entropy_of
from .qtensor import select_kept

ALPHA_MAX = 1.0


def heff1(L, R, A, W):
    """``singlesite_update`` (``algs/optimizeMPS.jl:503-511``): L[a,w,b] A[b,s,c] W[w,s,t,w']
    R[c,w',d] -> [a,t,d]."""
    LA = np.tensordot(L, A, axes=(2, 0))                      # [a, w, s, c]
    LAW = np.tensordot(LA, W, axes=((1, 2), (0, 1)))          # [a, c, t, w']
    return np.tensordot(LAW, R, axes=((1, 3), (0, 1)))       # [a, t, d]


def lexpand(L, A, W):
    """The expansion term of ``Lexpand`` without alpha: [a, t, w', c]."""
    LA = np.tensordot(L, A, axes=(2, 0))                      # [a, w, s, c]
    LAW = np.tensordot(LA, W, axes=((1, 2), (0, 1)))          # [a, c, t, w']
    return LAW.transpose(0, 2, 3, 1)


def rexpand(A, W, R):
    """The expansion term of ``Rexpand`` without alpha: [a, w, t, d]."""
    AR = np.tensordot(A, R, axes=(2, 0))                      # [a, s, w', d]
    WAR = np.tensordot(W, AR, axes=((1, 3), (1, 2)))          # [w, t, a, d]
    return WAR.transpose(2, 0, 1, 3)


def lanczos1(L, R, A, W, krylov, betatest=1e-10):
    """Lowest Ritz pair of the single-site Heff from A normalised (Krylov dim ``krylov``)."""
    V = [A / np.linalg.norm(A)]
    alphas, betas = [], []
    for jj in range(krylov):
        w = heff1(L, R, V[jj], W)
        a = float(np.sum(V[jj] * w))
        alphas.append(a)
        if jj == krylov - 1:
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
    ev, U = np.linalg.eigh(T)
    out = U[0, 0] * V[0]
    for k in range(1, n):
        out = out + U[k, 0] * V[k]
    return float(ev[0]), out


def alpha_update(alpha, truncerr, cutoff, last_energy, energy, noise_goal, dalpha):
    """``alpha_update`` (``algs/DMRG.jl:289-302``) in IEEE arithmetic, as the reference evaluates
    it (a zero energy ratio makes the site condition infinite, or NaN and so false)."""
    trunc_check = truncerr <= max(cutoff, 1e-12)
    err_est = abs(energy - last_energy) <= max(abs(energy * cutoff), 1e-12)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.float64(last_energy) / np.float64(energy) - 1.0
        sitecond = bool(abs(np.float64(truncerr * energy) / ratio) > noise_goal)
    if energy <= last_energy and (sitecond or err_est or trunc_check):
        alpha *= 1.0 - dalpha
    else:
        alpha *= 1.0 + dalpha
    return max(min(alpha, ALPHA_MAX), 1e-42)


def _add(a, b, sign=1):
    return tuple(x + sign * y for x, y in zip(a, b))


def _groups(labels):
    g = {}
    for n, q in enumerate(labels):
        g.setdefault(tuple(q), []).append(n)
    return [(q, g[q]) for q in sorted(g)]


def _trunc(G, maxm, minm, cutoff, degen_rtol):
    """G: list of (charge, index list, Gram matrix over those indices). Returns per group the
    kept eigenvectors (columns), the kept weights, the truncation error (relative) and D."""
    vals, vecs = [], []
    for _, _, gram in G:
        lam, U = np.linalg.eigh(gram)
        order = np.argsort(lam)[::-1]
        vals.append(lam[order])
        vecs.append(U[:, order])
    kept, terr = select_kept(vals, maxm, minm, cutoff, 0.0, degen_rtol)
    tot = float(sum(np.sum(v) for v in vals))
    D = np.sqrt(np.maximum(np.sort(np.concatenate([v[:k] for v, k in zip(vals, kept)]))[::-1],
                           0.0))
    return [(vecs[g][:, :kept[g]], vals[g][:kept[g]]) for g in range(len(G))], \
        (terr / tot if tot > 0 else 0.0), D


class State3S:
    """Dense MPS with charge labels per bond state, its MPO with labels, and the environments."""

    def __init__(self, psi, mpo, phys, bond_labels, oc=0):
        self.psi = [np.array(a, dtype=float) for a in psi]
        self.mpo = mpo
        self.phys = phys                     # phys[i][s]: charge tuple of state s of site i
        self.q = [list(map(tuple, b)) for b in bond_labels]   # q[b][state]
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


def step3s(S: State3S, i, j, P):
    psi, W = S.psi, S.mpo[i]
    E, A = lanczos1(S.Lenv[i], S.Renv[i], psi[i], W, P["krylov"])
    cond = P["noise"] > P["noise_incr"]
    a, d, c = A.shape
    if j > 0:
        rlab = [_add(S.q[i][x], S.phys[i][t]) for x in range(a) for t in range(d)]
        Mo = A.reshape(a * d, c)                          # rows (a, t), a-major
        M = Mo
        if cond:
            Pe = P["noise"] * lexpand(S.Lenv[i], A, W)
            M = np.hstack([Mo, Pe.reshape(a * d, -1)])
        G = []
        for Q, rows in _groups(rlab):
            G.append((Q, rows, M[rows] @ M[rows].T))
        res, terr, D = _trunc(G, P["maxm"], P["minm"], P["cutoff"], P["degen_rtol"])
        k = sum(u.shape[1] for u, _ in res)
        U = np.zeros((a * d, k))
        newq, o = [], 0
        for (Q, rows, _), (u, _) in zip(G, res):
            U[rows, o:o + u.shape[1]] = u
            newq += [Q] * u.shape[1]
            o += u.shape[1]
        psi[i] = U.reshape(a, d, k)
        DV = U.T @ Mo                                     # original columns only (condition)
        psi[i + 1] = np.tensordot(DV, psi[i + 1], axes=(1, 0))
        S.q[i + 1] = newq
    else:
        clab = [_add(S.q[i + 1][y], S.phys[i][t], -1) for t in range(d) for y in range(c)]
        Mo = A.reshape(a, d * c)                          # columns (t, d), t-major
        M = Mo
        if cond:
            Pe = P["noise"] * rexpand(A, W, S.Renv[i])
            M = np.vstack([Mo, Pe.reshape(-1, d * c)])
        G = []
        for Q, cols in _groups(clab):
            G.append((Q, cols, M[:, cols].T @ M[:, cols]))
        res, terr, D = _trunc(G, P["maxm"], P["minm"], P["cutoff"], P["degen_rtol"])
        k = sum(u.shape[1] for u, _ in res)
        V = np.zeros((d * c, k))
        newq, o = [], 0
        for (Q, cols, _), (u, _) in zip(G, res):
            V[cols, o:o + u.shape[1]] = u
            newq += [Q] * u.shape[1]
            o += u.shape[1]
        psi[i] = V.T.reshape(k, d, c)
        UD = Mo @ V                                       # original rows only (condition)
        psi[i - 1] = np.tensordot(psi[i - 1], UD, axes=(2, 0))
        S.q[i] = newq
    P["noise"] = alpha_update(P["noise"], terr, P["cutoff"], P["last_energy"], E,
                              P["noise_goal"], P["noise_incr"])
    return E, terr, D


def sweep3s(S: State3S, j, P, record):
    """One sweep (2(L-1) steps, ``optmps`` with ``step3S``): returns the new direction."""
    L = len(S.psi)
    record.update(maxtrunc=0.0, biggestm=0)
    for _ in range(2 * (L - 1)):
        i = S.oc
        E, terr, D = step3s(S, i, j, P)
        record["energy"] = E
        record["maxtrunc"] = max(record["maxtrunc"], terr)
        record["biggestm"] = max(record["biggestm"], len(D))
        if (i + 1) == min(max(2, P["svnbond"] + 1), L) and j < 0:
            record["entropy"] = entropy_of(D)
        if j > 0:
            S.Lenv[i + 1] = Lupdate(S.Lenv[i], S.psi[i], S.psi[i], S.mpo[i])
        else:
            S.Renv[i - 1] = Rupdate(S.Renv[i], S.psi[i], S.psi[i], S.mpo[i])
        S.oc += j
        if (S.oc == L - 1 and j > 0) or (S.oc == 0 and j < 0):
            j = -j
    return j


def dmrg3s(psi, mpo, phys, bond_labels, m=0, minm=2, sweeps=1, cutoff=0.0,
           krylov=2, noise=1.0, noise_goal=0.3, noise_incr=0.01, degen_rtol=0.0, svnbond=None, goal=0.0, cvgE=True):
    """``dmrg3S`` (``algs/DMRG.jl:655-671``) from a dense MPS with centre at site 0. Returns
    ``(energy, records, state)``; the starting energy (``startval``) opens the alpha bookkeeping
    and every sweep's last energy feeds the next sweep's ``alpha_update`` (``dmrgcvg``,
    ``algs/DMRG.jl:626-636``: the sweep ends the run when its energy moved by less than ``goal``,
    and only with ``cvgE`` does the last energy move on)."""
    L = len(psi)
    S = State3S(psi, mpo, phys, bond_labels, oc=0)
    e0 = float(np.sum(heff1(S.Lenv[0], S.Renv[0], S.psi[0], mpo[0]) * S.psi[0]))
    P = dict(maxm=m, minm=minm, cutoff=cutoff, krylov=krylov, noise=noise, noise_goal=noise_goal,
             noise_incr=noise_incr, degen_rtol=degen_rtol, last_energy=e0,
             svnbond=int(math.ceil(L / 2)) if svnbond is None else svnbond)
    recs = []
    j = 1
    for _ in range(sweeps):
        rec = {"entropy": 0.0}
        j = sweep3s(S, j, P, rec)
        rec["noise"] = P["noise"]
        recs.append(rec)
        if cvgE:
            if abs(rec["energy"] - P["last_energy"]) < goal:
                rec["converged"] = True
                break
            P["last_energy"] = rec["energy"]
    return recs[-1]["energy"], recs, S
