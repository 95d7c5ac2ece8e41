"""Host-side model and MPO construction (the reference does this on the host too).

Mirrors ``lib/models.jl`` and ``lib/MPO/makeMPO.jl``:
  * ``spinOps`` (``lib/models.jl:30-55,95-105``), ``fermionOps`` (``lib/models.jl:142-164``)
  * ``heisenbergMPO`` (``lib/models.jl:237-244``), ``hubbardMPO`` (``lib/models.jl:264-273``)
  * ``makeMPO(H, physSize, Ns)`` (``lib/MPO/makeMPO.jl:59-92``): ``G[l,j,k,m] = H[j+(l-1)d, k+(m-1)d]``,
    site 1 keeps the last row and site Ns the first column of the lower-triangular bulk.
plus two builders the benchmark configurations need: the transverse-field Ising chain and the
Heisenberg model on a snake-ordered W x Lx cylinder (a finite-state-machine MPO).
Physical QN labels use the charge of each basis state (2Sz for spins, (N, 2Sz) for fermions).
"""
from __future__ import annotations

import numpy as np


def spinOps(s=0.5):
    """``Sp, Sm, Sz, Sy(None: real data only), Sx, O, Id`` with states ordered m = s, s-1, .., -s."""
    d = int(round(2 * s + 1))
    op = np.zeros((d, d))
    oz = np.zeros((d, d))
    for q in range(d):
        m = s - q
        oz[q, q] = 2 * m
        if m + 1 <= s:
            op[q - 1, q] = np.sqrt(s * (s + 1) - m * (m + 1))
    om = op.T.copy()
    return op, om, oz * s, None, (op + om) * s, np.zeros((d, d)), np.eye(d)


def fermionOps():
    """``Cup, Cdn, F, Nup, Ndn, Ndens, O, Id`` on the Fock basis [0, up, dn, updn]."""
    O = np.zeros((4, 4))
    Cup = O.copy(); Cup[0, 1] = 1.0; Cup[2, 3] = 1.0
    Cdn = O.copy(); Cdn[0, 2] = 1.0; Cdn[1, 3] = -1.0
    Nup = Cup.T @ Cup
    Ndn = Cdn.T @ Cdn
    F = np.diag([1.0, -1.0, -1.0, 1.0])
    return Cup, Cdn, F, Nup, Ndn, Nup + Ndn, O, np.eye(4)


def heisenbergMPO(i=None, spinmag=0.5, J=1.0):
    Sp, Sm, Sz, _, _, O, Id = spinOps(spinmag)
    return np.block([[Id, O, O, O, O],
                     [J * 0.5 * Sm, O, O, O, O],
                     [J * 0.5 * Sp, O, O, O, O],
                     [J * Sz, O, O, O, O],
                     [O, Sp, Sm, Sz, Id]])


XXZ = heisenbergMPO


def hubbardMPO(i=None, t=1.0, mu=-2.0, HubU=4.0):
    Cup, Cdn, F, Nup, Ndn, Ndens, O, Id = fermionOps()
    onsite = mu * Ndens + HubU * Nup @ Ndn
    return np.block([[Id, O, O, O, O, O],
                     [-t * Cup.T, O, O, O, O, O],
                     [t * Cup, O, O, O, O, O],
                     [-t * Cdn.T, O, O, O, O, O],
                     [t * Cdn, O, O, O, O, O],
                     [onsite, Cup @ F, Cup.T @ F, Cdn @ F, Cdn.T @ F, Id]])


def tfiMPO(i=None, h=1.0):
    """``H = -sum Z_i Z_{i+1} - h sum X_i`` (Pauli), bulk ``[Id 0 0; Z 0 0; -hX -Z Id]``."""
    Z = np.diag([1.0, -1.0])
    X = np.array([[0.0, 1.0], [1.0, 0.0]])
    O, Id = np.zeros((2, 2)), np.eye(2)
    return np.block([[Id, O, O], [Z, O, O], [-h * X, -Z, Id]])


def makeMPO(H, physSize, Ns=None, lower=True):
    """``makeMPO`` (``lib/MPO/makeMPO.jl:59-92``).

    ``H`` is a bulk matrix, a function ``H(i)`` of the 1-based site, or a list of bulk matrices.
    Returns a :class:`dmrjtensor_b200.MPO` of W[w,s,t,w'] arrays."""
    from .state import MPO
    if callable(H):
        bulks = [np.asarray(H(i + 1), dtype=float) for i in range(Ns)]
    elif isinstance(H, np.ndarray):
        bulks = [H] * Ns
    else:
        bulks = [np.asarray(h, dtype=float) for h in H]
    sizes = list(physSize) if np.ndim(physSize) else [int(physSize)]
    out = []
    for i, Hb in enumerate(bulks):
        Hb = Hb if lower else Hb.T
        d = sizes[i % len(sizes)]
        a1, a2 = Hb.shape[0] // d, Hb.shape[1] // d
        out.append(Hb.reshape(a1, d, a2, d).transpose(0, 1, 3, 2).copy())
    if lower:
        out[0] = out[0][-1:].copy()
        out[-1] = out[-1][..., :1].copy()
    else:
        out[0] = out[0][:1].copy()
        out[-1] = out[-1][..., -1:].copy()
    return MPO(out)


def cylinder_bonds(W, Lx):
    """Nearest-neighbour bonds (i < j, 0-based snake order) of a W x Lx cylinder, periodic in W."""
    def site(x, y):
        return x * W + (y if x % 2 == 0 else W - 1 - y)
    bonds = set()
    for x in range(Lx):
        for y in range(W):
            i = site(x, y)
            if W > 2 or y + 1 < W:
                j = site(x, (y + 1) % W)
                bonds.add((min(i, j), max(i, j)))
            if x + 1 < Lx:
                j = site(x + 1, y)
                bonds.add((min(i, j), max(i, j)))
    return sorted(bonds)


def heisenbergCylinderMPO(W, Lx, J=1.0):
    """Snake-ordered Heisenberg MPO on a W x Lx cylinder.

    Each bond (i, j) is a string S_i^a ... S_j^b; a string started at site i travels through one
    channel per (operator a, distance) while some bond from i still lies ahead, so the bond
    dimension is 2 + 3 x (number of strings crossing a cut): 14 for W = 4.
    """
    bonds = cylinder_bonds(W, Lx)
    N = W * Lx
    ahead = {i: [j for (a, j) in bonds if a == i] for i in range(N)}
    Sp, Sm, Sz, _, _, O, Id = spinOps(0.5)
    first = [Sp, Sm, Sz]
    second = [0.5 * J * Sm, 0.5 * J * Sp, J * Sz]
    # open channels on the bond right of site s: strings started at i <= s with a bond (i, j > s)
    chans = []
    for s in range(N + 1):
        chans.append([(i, a) for i in range(min(s, N)) for a in range(3)
                      if any(j >= s for j in ahead[i])])
    tensors = []
    for s in range(N):
        left = ["done"] + chans[s] + ["start"]
        right = ["done"] + chans[s + 1] + ["start"]
        li = {c: n for n, c in enumerate(left)}
        ri = {c: n for n, c in enumerate(right)}
        Wt = np.zeros((len(left), 2, 2, len(right)))

        def put(lc, rc, op):
            Wt[li[lc], :, :, ri[rc]] += op
        put("done", "done", Id)
        put("start", "start", Id)
        for a in range(3):
            if ahead[s] and (s, a) in ri:
                put("start", (s, a), first[a])
            for (i, aa) in chans[s]:
                if aa != a:
                    continue
                if s in ahead[i]:
                    put((i, a), "done", second[a])
                if (i, a) in ri:
                    put((i, a), (i, a), Id)
        tensors.append(Wt)
    tensors[0] = tensors[0][-1:].copy()
    tensors[-1] = tensors[-1][..., :1].copy()
    from .state import MPO
    return MPO(tensors)


SPIN_QN = [(1,), (-1,)]                               # 2Sz of [up, down]
HUBBARD_QN = [(0, 0), (1, 1), (1, -1), (2, 0)]          # (N, 2Sz) of [0, up, dn, updn]
