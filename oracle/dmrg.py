"""Two-site DMRG on the CPU (test infrastructure): the oracle for the device engine.

Restates ``algs/DMRG.jl`` / ``algs/optimizeMPS.jl`` / ``lib/Env/makeEnv.jl`` /
``lib/MPO_MPS/{L,R}update.jl`` with 0-based indices (Julia index ``n`` becomes ``n-1``).
Works on dense ``numpy.ndarray`` tensors and on :class:`oracle.qtensor.QTensor` block-sparse ones.

Layouts (numpy order = the reference's Julia order):
  MPS site ``A[a, s, b]``; MPO ``W[w, s(ket), t(bra), w']``; left env ``L[a(bra), w, b(ket)]``;
  right env ``R[b(ket), w, a(bra)]`` (``lib/Env/makeEnv.jl:17-26``).
"""
from __future__ import annotations

import math
import time

import numpy as np

from .qtensor import (Index, QTensor, axpy, ccontract, contract, contractc, dmul, inner, norm,
                      rho_trunc, scale, svd_trunc)


# ------------------------------------------------------------------ environments

def make_boundary(psi, mpo, left=True):
    """``makeBoundary`` (``lib/Env/makeEnv.jl:49-93``): ones(1,1,1) dense or a 1x1x1 QTensor."""
    if isinstance(psi[0], np.ndarray):
        return np.ones((1, 1, 1))
    if left:
        ia = psi[0].indices[0]            # bond left of site 1 (arrow +1)
        iw = mpo[0].indices[0]            # MPO left edge (arrow +1)
        idx = [ia, iw.dual(), ia.dual()]
    else:
        ib = psi[-1].indices[2]           # bond right of site L (arrow -1)
        iw = mpo[-1].indices[3]           # MPO right edge (arrow -1)
        idx = [ib.dual(), iw.dual(), ib]
    if len(idx[0].dims) != 1 or len(idx[1].dims) != 1:
        raise ValueError("edge bonds must be one-dimensional")
    return QTensor(idx, {(0, 0, 0): np.ones((1, 1, 1))}, psi[0].flux)


def Lupdate(Lenv, dual, psi, W):
    """``lib/MPO_MPS/Lupdate.jl:17-26``: L'[a',w',b'] = conj(A[a,t,a']) L[a,w,b] W[w,s,t,w'] A[b,s,b']."""
    t = contractc(Lenv, 0, dual, 0)          # [w, b, t, a']
    t = contract(t, (0, 2), W, (0, 2))       # [b, a', s, w']
    return contract(t, (0, 2), psi, (0, 1))  # [a', w', b']


def Rupdate(Renv, dual, psi, W):
    """``lib/MPO_MPS/Rupdate.jl:17-26``: R[b,w,a] = A[b,s,b'] W[w,s,t,w'] conj(A[a,t,a']) R[b',w',a']."""
    t = ccontract(dual, 2, Renv, 2)          # [a, t, b', w']
    t = contract(W, (2, 3), t, (1, 3))       # [w, s, a, b']
    return contract(psi, (1, 2), t, (1, 3))  # [b, w, a]


def make_env(psi, mpo, oc):
    """``makeEnv`` (``lib/Env/makeEnv.jl:196-221``) with a 0-based centre ``oc``.
    Returns lists ``Lenv`` (valid for 0..oc) and ``Renv`` (valid for oc..L-1)."""
    L = len(psi)
    Lenv = [None] * L
    Renv = [None] * L
    Lenv[0] = make_boundary(psi, mpo, True)
    Renv[L - 1] = make_boundary(psi, mpo, False)
    for i in range(oc):
        Lenv[i + 1] = Lupdate(Lenv[i], psi[i], psi[i], mpo[i])
    for i in range(L - 1, oc, -1):
        Renv[i - 1] = Rupdate(Renv[i], psi[i], psi[i], mpo[i])
    return Lenv, Renv


# ------------------------------------------------------------------ effective Hamiltonian

def singlesite_update(Lenv, Renv, A, W):
    """``algs/optimizeMPS.jl:503-511``."""
    LA = contract(Lenv, 2, A, 0)             # [a, w, s, b]
    LWA = contract(LA, (1, 2), W, (0, 1))    # [a, b, t, w']
    return contract(LWA, (1, 3), Renv, (0, 1))  # [a, t, a']


def make2site(Lenv, Renv, psiL, psiR, WL, WR):
    """Heff #1, ``algs/DMRG.jl:48-54``."""
    Lpsi = contract(Lenv, 2, psiL, 0)             # [a, w, s1, c]
    LHpsi = contract(Lpsi, (1, 2), WL, (0, 1))    # [a, c, t1, w']
    LHpsipsi = contract(LHpsi, 1, psiR, 0)        # [a, t1, w', s2, d]
    LHH = contract(LHpsipsi, (2, 3), WR, (0, 1))  # [a, t1, d, t2, w'']
    return contract(LHH, (2, 4), Renv, (0, 1))    # [a, t1, t2, a']


def heff_twosite(Lenv, Renv, psi2, WL, WR):
    """Heff #2 on a 4-index vector, ``algs/DMRG.jl:69-73``."""
    H2 = contract(Lenv, 2, psi2, 0)               # [a, w, s1, s2, d]
    ops = contract(WL, 3, WR, 0)                  # [w, s1, t1, s2, t2, w'']
    H2 = contract(H2, (1, 2, 3), ops, (0, 1, 3))  # [a, d, t1, t2, w'']
    return contract(H2, (1, 4), Renv, (0, 1))     # [a, t1, t2, a']


def simplelanczos(Lenv, Renv, psiL, psiR, WL, WR, betatest=1e-10):
    """``algs/DMRG.jl:57-90``: one 2-vector Krylov step. Returns ``(energy, AA', nmatvec)``."""
    Hpsi = make2site(Lenv, Renv, psiL, psiR, WL, WR)
    AA = contract(psiL, 2, psiR, 0)
    AA = scale(AA, 1.0 / norm(AA))
    alpha1 = inner(AA, Hpsi)
    psi2 = axpy(1.0, Hpsi, -alpha1, AA)
    beta1 = norm(psi2)
    if beta1 > betatest:
        psi2 = scale(psi2, 1.0 / beta1)
        Hpsi2 = heff_twosite(Lenv, Renv, psi2, WL, WR)
        alpha2 = inner(psi2, Hpsi2)
        M = np.array([[alpha1, beta1], [beta1, alpha2]])
        D, U = np.linalg.eigh(M)
        return float(D[0]), axpy(U[0, 0], AA, U[1, 0], psi2), 2
    return float(alpha1), AA, 1


def lanczos_k(Lenv, Renv, psiL, psiR, WL, WR, krylov, betatest=1e-10):
    """Krylov-``krylov`` Lanczos with full (two-pass classical Gram-Schmidt) reorthogonalisation,
    the generalisation of :func:`simplelanczos` that the device engine runs for ``krylov > 2``.
    Vectors are Krylov basis vectors of the two-site state; ``krylov`` matvecs at most."""
    AA = contract(psiL, 2, psiR, 0)
    v = scale(AA, 1.0 / norm(AA))
    V = [v]
    alphas, betas = [], []
    nmv = 0
    for j in range(krylov):
        w = heff_twosite(Lenv, Renv, V[j], WL, WR)
        nmv += 1
        a = inner(V[j], w)
        alphas.append(a)
        if j == krylov - 1:
            break
        w = axpy(1.0, w, -a, V[j])
        if j > 0:
            w = axpy(1.0, w, -betas[j - 1], V[j - 1])
        for _ in range(2):
            for u in V:
                w = axpy(1.0, w, -inner(u, w), u)
        b = norm(w)
        if b <= betatest:
            break
        betas.append(b)
        V.append(scale(w, 1.0 / b))
    n = len(alphas)
    T = np.diag(alphas) + np.diag(betas[:n - 1], 1) + np.diag(betas[:n - 1], -1)
    ev, U = np.linalg.eigh(T)
    out = scale(V[0], U[0, 0])
    for i in range(1, n):
        out = axpy(1.0, out, U[i, 0], V[i])
    return float(ev[0]), out, nmv


# ------------------------------------------------------------------ one bond and the sweep

class Params:
    """The subset of ``algvars`` (``algs/optimizeMPS.jl:514-577``) the two-site path reads."""

    def __init__(self, L, maxm=0, minm=2, cutoff=0.0, krylov=2, trunc="svd", svnbond=None,
                 degen_rtol=0.0, betatest=1e-10):
        self.maxm, self.minm, self.cutoff = int(maxm), int(minm), float(cutoff)
        self.krylov, self.trunc = int(krylov), trunc
        self.svnbond = int(math.ceil(L / 2)) if svnbond is None else int(svnbond)
        self.degen_rtol, self.betatest = float(degen_rtol), float(betatest)
        self.energy = 0.0
        self.truncerr = 0.0
        self.maxtrunc = 0.0
        self.biggestm = 0
        self.entropy = 0.0
        self.storeD = []
        self.nmatvec = 0


def entropy_of(D):
    """``-sum D^2 log D^2`` (``algs/DMRG.jl:172-210``), with 0 log 0 taken as 0."""
    s = 0.0
    for x in D:
        p = float(x) ** 2
        if p > 0:
            s -= p * math.log(p)
    return s


def _flatD(D):
    if isinstance(D, list):
        return np.sort(np.concatenate([np.asarray(d) for d in D]) if D else np.zeros(0))[::-1]
    return np.asarray(D)


def twostep(j, i, iL, iR, psi, mpo, Lenv, Renv, P: Params):
    """``twostep`` (``algs/DMRG.jl:362-405``) without the unused third Heff (``:374``)."""
    L = len(psi)
    if j > 0:
        psi[iL] = scale(psi[iL], 1.0 / norm(psi[iL]))
    else:
        psi[iR] = scale(psi[iR], 1.0 / norm(psi[iR]))
    if P.krylov <= 2:
        energy, AA, nmv = simplelanczos(Lenv[iL], Renv[iR], psi[iL], psi[iR], mpo[iL], mpo[iR],
                                        P.betatest)
    else:
        energy, AA, nmv = lanczos_k(Lenv[iL], Renv[iR], psi[iL], psi[iR], mpo[iL], mpo[iR],
                                    P.krylov, P.betatest)
    P.nmatvec += nmv
    P.energy = energy
    if P.trunc == "svd":
        U, D, V, terr = svd_trunc(AA, [0, 1], [2, 3], P.maxm, P.minm, P.cutoff, 1.0, P.degen_rtol)
    else:
        U, D, V, terr = rho_trunc(AA, [0, 1], [2, 3], j, P.maxm, P.minm, P.cutoff, 1.0,
                                  P.degen_rtol)
    if P.trunc == "svd":
        if j < 0:
            psi[iL], psi[iR] = dmul(U, D, 2), V
        else:
            psi[iL], psi[iR] = U, dmul(V, D, 0)
    else:
        # the rho form already returns U.D (j<0) or D.V (j>0) on the non-isometric side
        psi[iL], psi[iR] = U, V
    P.truncerr = terr
    Dflat = _flatD(D)
    P.maxtrunc = max(P.maxtrunc, terr)
    P.biggestm = max(P.biggestm, len(Dflat))
    # SvNcheck!: 1-based i == min(max(2, SvNbond+1), L) and j < 0
    if (i + 1) == min(max(2, P.svnbond + 1), L) and j < 0:
        P.entropy = entropy_of(Dflat)
        P.storeD = list(Dflat[:8])


def sweep(psi, mpo, Lenv, Renv, oc, j, P: Params):
    """One ``optmps`` sweep (``algs/optimizeMPS.jl:790-835``): 2(L-1) bond steps, an environment
    update after each, reversal at the edges. Returns the new ``(oc, j)``."""
    L = len(psi)
    P.maxtrunc, P.biggestm = 0.0, 0
    for _ in range(2 * (L - 1)):
        i = oc
        iL, iR = (i, i + 1) if j > 0 else (i - 1, i)
        twostep(j, i, iL, iR, psi, mpo, Lenv, Renv, P)
        if j > 0:
            Lenv[i + 1] = Lupdate(Lenv[i], psi[i], psi[i], mpo[i])
        else:
            Renv[i - 1] = Rupdate(Renv[i], psi[i], psi[i], mpo[i])
        oc += j
        if (oc == L - 1 and j > 0) or (oc == 0 and j < 0):
            j = -j
    return oc, j


def startval(Lenv, Renv, A, W):
    """``algs/optimizeMPS.jl:255-258``: single-site <psi|H|psi> at the centre."""
    return inner(A, singlesite_update(Lenv, Renv, A, W))


def dmrg(psi, mpo, m=0, minm=2, sweeps=1, cutoff=0.0, oc=0, krylov=2, trunc="svd",
         svnbond=None, degen_rtol=0.0, maxm_schedule=None, record=None, goal=0.0, cvgE=True):
    """``dmrg(psi, mpo; m, minm, sweeps, cutoff)`` with ``method="twosite"`` (``algs/DMRG.jl:549-588``
    -> ``dmrg_twosite`` ``:675-691`` -> ``optmps``). ``psi`` (list of tensors) is modified in place.

    Returns ``(energy, info)``; ``energy`` is the energy of the last bond step
    (``algs/optimizeMPS.jl:848``). ``info`` holds per-sweep records (energy, maxtrunc, biggestm,
    entropy at bond ``svnbond``, seconds) and the final centre ``oc`` (0-based).
    ``maxm_schedule`` (optional list) overrides ``m`` per sweep.
    ``goal``/``cvgE``: the convergence test of ``dmrgcvg`` (``algs/DMRG.jl:610-652``): after each
    sweep, stop when |E - E_last| < goal (energy, ``cvgE``) or |S_last - S| < goal (entropy);
    E_last starts at ``startval`` (``algs/optimizeMPS.jl:365-371``), S_last at 0, and both are
    updated only when the test fails. ``goal = 0`` (the default, ``algs/optimizeMPS.jl:527``)
    never stops early.
    """
    L = len(psi)
    P = Params(L, m, minm, cutoff, krylov, trunc, svnbond, degen_rtol)
    Lenv, Renv = make_env(psi, mpo, oc)
    P.energy = startval(Lenv[oc], Renv[oc], psi[oc], mpo[oc])
    e0 = P.energy
    if oc == 0:
        j = 1
    elif oc == L - 1:
        j = -1
    else:
        j = 1
    recs = []
    last_e, last_s = e0, 0.0
    for n in range(sweeps):
        if maxm_schedule is not None:
            P.maxm = int(maxm_schedule[n])
        t0 = time.perf_counter()
        oc, j = sweep(psi, mpo, Lenv, Renv, oc, j, P)
        dt = time.perf_counter() - t0
        recs.append(dict(energy=P.energy, maxtrunc=P.maxtrunc, biggestm=P.biggestm,
                         entropy=P.entropy, seconds=dt, maxm=P.maxm))
        if record is not None:
            record(recs[-1])
        check = abs(P.energy - last_e) if cvgE else abs(last_s - P.entropy)
        if check < goal:
            break
        last_e, last_s = P.energy, P.entropy
    return P.energy, dict(sweeps=recs, oc=oc, e0=e0, nmatvec=P.nmatvec, storeD=P.storeD)


def expect(psi, mpo):
    """<psi|H|psi>/<psi|psi> by a full left-to-right contraction (``lib/MPO_MPS/expect.jl:19-56``)."""
    Lenv = make_boundary(psi, mpo, True)
    Nenv = None
    for i in range(len(psi)):
        Lenv = Lupdate(Lenv, psi[i], psi[i], mpo[i])
    R = make_boundary(psi, mpo, False)
    val = float(contract(Lenv, (0, 1, 2), R, (2, 1, 0))) if isinstance(Lenv, np.ndarray) else \
        sum(float(np.sum(Lenv.blocks[k] * np.transpose(R.blocks[(k[2], k[1], k[0])], (2, 1, 0))))
            for k in Lenv.blocks if (k[2], k[1], k[0]) in R.blocks)
    nrm = 1.0
    if Nenv is None:
        nrm = overlap(psi, psi)
    return val / nrm


def overlap(phi, psi):
    """<phi|psi> by transfer matrices."""
    if isinstance(psi[0], np.ndarray):
        E = np.ones((1, 1))
        for A, B in zip(phi, psi):
            E = np.einsum("ab,asc,bsd->cd", E, A, B)
        return float(E[0, 0])
    E = None
    from .qtensor import contract as c
    for A, B in zip(phi, psi):
        if E is None:
            E = ccontract(A, (0, 1), B, (0, 1))      # [a', b']
        else:
            E = c(ccontract(A, 0, E, 0), (0, 2), B, (1, 0))   # [s,a',b] x B[b,s,b']
    return float(sum(np.sum(v) for v in E.blocks.values()))
