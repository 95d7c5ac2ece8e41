"""Measurements of an MPS on the CPU (test infrastructure): the oracle for the device measurements.

``expect_value`` restates ``lib/MPO_MPS/expect.jl:19-45``: the right environment is carried from
the last site to the first (``Renv = ccontract(dualpsi[i],3,Renv,..)``, the MPO, then ``psi[i]``),
then contracted with the left boundary. The value is not normalised.

``correlationmatrix`` restates ``lib/MPO_MPS/correlationmatrix.jl:21-56`` on dense tensors: the
orthogonality centre is moved to each site i with exact QR / LQ steps (``move!``,
``lib/MPS/move.jl:19-37,124-192``, the untruncated ``qr!`` / ``lq!`` branches), and the
element is contracted locally (the left part of the chain is the identity in that gauge).

``mps_vector`` and ``ed_correlation`` give the same quantities from the full state vector; they
pin the restatement on small chains.
"""
from __future__ import annotations

import numpy as np

from .dmrg import Rupdate, make_boundary


# ------------------------------------------------------------------ expect

def expect_value(psi, mpo):
    """``expect(psi, H)``: <psi|H|psi> (dense arrays or QTensors), not normalised."""
    Renv = make_boundary(psi, mpo, False)
    for i in range(len(psi) - 1, -1, -1):
        Renv = Rupdate(Renv, psi[i], psi[i], mpo[i])
    if isinstance(Renv, np.ndarray):
        return float(Renv.reshape(-1)[0])          # [1, 1, 1] against Lbound = ones(1, 1, 1)
    return float(sum(np.sum(v) for v in Renv.blocks.values()))


# ------------------------------------------------------------------ gauge moves

def move_right(psi, i):
    """``moveR!``: psi[i] = Q, psi[i+1] = R psi[i+1] (exact QR of psi[i] as [(a s), b])."""
    A = psi[i]
    a, d, b = A.shape
    Q, R = np.linalg.qr(A.reshape(a * d, b))
    psi[i] = Q.reshape(a, d, Q.shape[1])
    psi[i + 1] = np.tensordot(R, psi[i + 1], axes=(1, 0))


def move_left(psi, i):
    """``moveL!``: psi[i] = Q^T, psi[i-1] = psi[i-1] L (exact LQ of psi[i] as [a, (s b)])."""
    A = psi[i]
    a, d, b = A.shape
    Q, R = np.linalg.qr(A.reshape(a, d * b).T)
    psi[i] = Q.T.reshape(Q.shape[1], d, b)
    psi[i - 1] = np.tensordot(psi[i - 1], R.T, axes=(2, 0))


def move(psi, oc, target):
    """``move!(psi, target)`` from centre ``oc`` (0-based); returns the new centre."""
    while oc < target:
        move_right(psi, oc)
        oc += 1
    while oc > target:
        move_left(psi, oc)
        oc -= 1
    return oc


# ------------------------------------------------------------------ correlation matrix

def correlationmatrix(psi, oc, Cc, Ca, trail=None):
    """``correlationmatrix(psi, Cc, Ca; trail)`` for a normalised dense MPS with centre ``oc``.
    Operators are d x d arrays O[bra, ket] (``contract(O, 2, psi[i], 2)`` acts on the ket)."""
    psi = [np.array(A, dtype=float) for A in psi]
    L = len(psi)
    rho = np.zeros((L, L))
    FCc = Cc @ trail if trail is not None else Cc      # contract(Cc,2,trail,1)
    onsite = Cc @ Ca                                   # contract(Cc,2,Ca,1)
    for i in range(L):
        oc = move(psi, oc, i)
        top = np.einsum("ab,lbr->lar", onsite, psi[i])  # contract([2,1,3],onsite,2,psi[i],2)
        rho[i, i] = float(np.sum(top * psi[i]))         # contractc(TopTerm, dualpsi[i])
    for i in range(L - 1):
        oc = move(psi, oc, i)
        top = np.einsum("ab,lbr->alr", FCc, psi[i])     # contract(FCc,2,psi[i],2): [a,l,r]
        Lenv = np.einsum("alr,laq->rq", top, psi[i])    # contractc(top,(2,1),dual,(1,2)): [ket,bra]
        for j in range(i + 1, L):
            R = np.einsum("ab,lbr->alr", Ca, psi[j])    # contract(Ca,2,psi[j],2)
            R = np.einsum("alr,sar->ls", R, psi[j])     # contractc(R,(1,3),dual,(2,3)): [ket,bra]
            el = float(np.sum(Lenv * R))                # contract(Lenv, Renv)
            if j < L - 1:
                X = np.einsum("xy,xsr->ysr", Lenv, psi[j])           # contract(Lenv,1,psi[j],1)
                if trail is not None:
                    X = np.einsum("ysr,ts->yrt", X, trail)           # contract(Lenv,2,trail,2)
                    Lenv = np.einsum("yrt,ytq->rq", X, psi[j])       # contractc(..,(1,3),dual,(1,2))
                else:
                    Lenv = np.einsum("ysr,ysq->rq", X, psi[j])       # contractc(..,(1,2),dual,(1,2))
            rho[i, j] = el
            rho[j, i] = el
    return rho


# ------------------------------------------------------------------ exact references

def mps_vector(psi):
    """Full state vector psi[s_1, ..., s_L] (site 1 most significant), dense MPS."""
    v = np.asarray(psi[0])[0]                           # [s1, b]
    for A in psi[1:]:
        v = np.tensordot(v, A, axes=(v.ndim - 1, 0))
    return v.reshape(-1)


def _kron_all(ops):
    M = np.ones((1, 1))
    for O in ops:
        M = np.kron(M, O)
    return M


def ed_correlation(v, L, Cc, Ca, trail=None):
    """rho[i,j] = <v|(Cc F)_i F..F Ca_j|v> / <v|v> by full operator strings (small L only)."""
    d = Cc.shape[0]
    Id = np.eye(d)
    F = trail if trail is not None else Id
    nrm = float(v @ v)
    rho = np.zeros((L, L))
    for i in range(L):
        ops = [Id] * L
        ops[i] = Cc @ Ca
        rho[i, i] = float(v @ (_kron_all(ops) @ v)) / nrm
        for j in range(i + 1, L):
            ops = [Id] * L
            ops[i] = Cc @ F
            for k in range(i + 1, j):
                ops[k] = F
            ops[j] = Ca
            rho[i, j] = rho[j, i] = float(v @ (_kron_all(ops) @ v)) / nrm
    return rho


# ------------------------------------------------------------------ n-point correlation

def _apply(O, A):
    """``contract([2,1,3], O, 2, A, 2)``: the operator O[bra, ket] on the ket of a site tensor."""
    return np.einsum("ts,asb->atb", O, A)


def _lstep(Lm, A, B):
    """Left environment step <A|.|B> from bond b to b+1: Lm[a_bra, a_ket] -> [b_bra, b_ket]."""
    return np.einsum("xy,xsb,ysc->bc", Lm, A, B)


def _rstep(Rm, A, B):
    """Right environment step from bond b+1 to b: Rm[b_bra, b_ket] -> [a_bra, a_ket]."""
    return np.einsum("xy,asx,csy->ac", Rm, A, B)


def _oplists(ops):
    return [list(o) if isinstance(o, (list, tuple)) else [np.asarray(o)] for o in ops]


def _trails(trail, n, d):
    if trail is None or (isinstance(trail, (list, tuple)) and len(trail) == 0):
        return [None] * n
    if isinstance(trail, (list, tuple)):
        sub = [np.asarray(trail[w % len(trail)]) for w in range(n)]
    else:
        sub = [np.asarray(trail)] * n
    return [None if np.allclose(F, np.eye(d)) else F for F in sub]


def correlation(psi, ops, sites=None, trail=None):
    """Literal restatement of ``correlation(dualpsi = psi, psi, ops...; sites, trail)``
    (``lib/MPO_MPS/correlation.jl:98-237``) on a dense MPS: omega[p_1, ..., p_n] with operator k
    at ``sites[k][p_k]`` (0-based here; an operator given as a list acts on that many consecutive
    sites). For each combination of the positions of operators 2..n the ket copy gets operators
    n..2 (each after its trail on every site left of it, ``subtrail``), the right environments are
    rebuilt from the rightmost of them down (in place, ``Renv[a-1] = Rupdate(Renv[a], ...)``), and
    operator 1 runs over its positions with the left environment carried along, its trail left on
    each site it has passed. The multi-index of operators 2..n advances with its first index
    fastest (the increment of TensorPACK's ``position_incrementer!``, which is not vendored; its
    behaviour here is inferred from this call site). Not normalised. ``sites`` must be contiguous
    ranges starting at site 0 for the result to be indexed like the reference's (which stores at
    the site numbers themselves)."""
    L = len(psi)
    d = np.asarray(psi[0]).shape[1]
    O = _oplists(ops)
    n = len(O)
    lens = [len(o) for o in O]
    if sites is None:
        sites = [list(range(L)) for _ in range(n)]
    F = _trails(trail, n, d)
    base = [len(sites[k]) - (lens[k] - 1) for k in range(n)]
    # makeEnv(dualpsi, psi): Lenv[i] left of site i, Renv[i] right of site i
    Lenv = [None] * L
    Renv = [None] * L
    Lenv[0] = np.ones((1, 1))
    for i in range(L - 1):
        Lenv[i + 1] = _lstep(Lenv[i], psi[i], psi[i])
    Renv[L - 1] = np.ones((1, 1))
    for i in range(L - 1, 0, -1):
        Renv[i - 1] = _rstep(Renv[i], psi[i], psi[i])
    omega = np.zeros(base)
    bpos = [0] * n
    while all(bpos[w] < base[w] for w in range(n)):
        save = [np.asarray(A) for A in psi]
        pos = [sites[w][bpos[w]] for w in range(n)]
        maxops = 0
        for g in range(n - 1, 0, -1):
            maxops = max(pos[g] + lens[g] - 1, maxops)
            for p in range(lens[g]):
                save[pos[g] + p] = _apply(O[g][p], save[pos[g] + p])
            if F[g] is not None:
                for w in range(pos[g]):
                    save[w] = _apply(F[g], save[w])
        for a in range(maxops, 0, -1):
            Renv[a - 1] = _rstep(Renv[a], psi[a], save[a])
        for y in range(base[0]):
            w = sites[0][y]
            X = Lenv[w]
            for p in range(lens[0]):
                X = _lstep(X, psi[w + p], _apply(O[0][p], save[w + p]))
            res = float(np.sum(X * Renv[w + lens[0] - 1]))
            omega[(y,) + tuple(bpos[1:])] = res
            if F[0] is not None:
                save[w] = _apply(F[0], save[w])
            if y + 1 < len(sites[0]):
                for r in range(w, sites[0][y + 1] + 1):
                    if r < L - 1:
                        Lenv[r + 1] = _lstep(Lenv[r], psi[r], save[r])
        # position_incrementer!: the first index is exhausted, carry into the next ones
        bpos[0] = base[0]
        k = 0
        while k < n - 1 and bpos[k] >= base[k]:
            bpos[k] = 0
            bpos[k + 1] += 1
            k += 1
        if n == 1:
            break
    return omega


def ed_correlation_n(v, L, d, ops, sites=None, trail=None):
    """omega[p_1, ..., p_n] = <v| prod_s O(s) |v> from the full state vector (small L only), with
    O(s) = A_1(s) A_2(s) ... A_n(s), A_g(s) = trail_g if s lies left of operator g's first site,
    operator g's factor on its sites, the identity elsewhere (the order in which the reference
    applies them to the ket). Not normalised."""
    O = _oplists(ops)
    n = len(O)
    lens = [len(o) for o in O]
    if sites is None:
        sites = [list(range(L)) for _ in range(n)]
    F = _trails(trail, n, d)
    base = [len(sites[k]) - (lens[k] - 1) for k in range(n)]
    Id = np.eye(d)
    V = np.asarray(v, dtype=float).reshape((d,) * L)
    omega = np.zeros(base)
    for idx in np.ndindex(*base):
        pos = [sites[g][idx[g]] for g in range(n)]
        W = V
        for s in range(L):
            M = Id
            for g in range(n):
                if s < pos[g]:
                    A = F[g] if F[g] is not None else Id
                elif s < pos[g] + lens[g]:
                    A = O[g][s - pos[g]]
                else:
                    A = Id
                M = M @ A
            if not np.array_equal(M, Id):
                W = np.moveaxis(np.tensordot(M, W, axes=(1, s)), 0, s)
        omega[idx] = float(np.sum(V * W))
    return omega
