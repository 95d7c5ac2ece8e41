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
