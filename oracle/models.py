"""MPO / MPS construction for the CPU oracle (test infrastructure).

Restates, in numpy:
* ``spinOps`` (``lib/models.jl:30-55,95-105``) and ``fermionOps`` (``lib/models.jl:142-164``);
* ``heisenbergMPO`` (``lib/models.jl:237-244``) and ``hubbardMPO`` (``lib/models.jl:264-273``);
* ``makeMPO`` (``lib/MPO/makeMPO.jl:59-92``): ``G[l,j,k,m] = H[j+(l-1)d, k+(m-1)d]``, first site keeps
  the last row, last site the first column (lower-triangular bulk form);
* QN assignment of MPO bonds (``lib/MPO/makeqMPO.jl:23-84``: the outgoing label of a right bond
  state is the QN with the largest summed weight) and MPS bonds (``assignflux!``,
  ``lib/MPS/MPS.jl:206-219``: the label of the largest-magnitude element).

Sign convention used by this oracle (self-consistent; TensorPACK folds arrows into labels
instead): with ``p(s)`` the physical QN and ``r`` the MPO bond label,
``r(w') = r(w) - p(ket) + p(bra)`` where ket is MPO index 2 and bra is index 3 (the reference
contracts the ket with index 2, ``lib/MPO_MPS/Lupdate.jl:20-25``).
"""
from __future__ import annotations

import numpy as np

from .qtensor import Index, QTensor, from_dense


# ------------------------------------------------------------------ operators

def spin_ops(s=0.5):
    """``Sp, Sm, Sz, Sy(None), Sx, O, Id`` for spin ``s`` (states ordered m = s .. -s)."""
    d = int(round(2 * s + 1))
    O = np.zeros((d, d))
    Id = np.eye(d)
    oz = np.zeros((d, d))
    op = np.zeros((d, d))
    ms = [s - q for q in range(d)]
    for q, m in enumerate(ms):
        oz[q, q] = 2 * m
        if m + 1 <= s:
            op[q - 1, q] = np.sqrt(s * (s + 1) - m * (m + 1))
    om = op.T.copy()
    ox = op + om
    return op, om, oz * s, None, ox * s, O, Id


def fermion_ops():
    """``Cup, Cdn, F, Nup, Ndn, Ndens, O, Id``; states [empty, up, dn, updn]."""
    O = np.zeros((4, 4))
    Id = np.eye(4)
    Cup = O.copy()
    Cup[0, 1] = 1.0
    Cup[2, 3] = 1.0
    Cdn = O.copy()
    Cdn[0, 2] = 1.0
    Cdn[1, 3] = -1.0
    Nup = Cup.T @ Cup
    Ndn = Cdn.T @ Cdn
    Ndens = Nup + Ndn
    F = Id.copy()
    F[1, 1] = -1.0
    F[2, 2] = -1.0
    return Cup, Cdn, F, Nup, Ndn, Ndens, O, Id


def _block(rows):
    return np.block(rows)


def heisenberg_bulk(J=1.0, spinmag=0.5):
    Sp, Sm, Sz, _, _, O, Id = spin_ops(spinmag)
    return _block([[Id, O, O, O, O],
                   [J * 0.5 * Sm, O, O, O, O],
                   [J * 0.5 * Sp, O, O, O, O],
                   [J * Sz, O, O, O, O],
                   [O, Sp, Sm, Sz, Id]])


def hubbard_bulk(t=1.0, mu=-2.0, U=4.0):
    Cup, Cdn, F, Nup, Ndn, Ndens, O, Id = fermion_ops()
    onsite = mu * Ndens + U * Nup @ Ndn
    return _block([[Id, O, O, O, O, O],
                   [-t * Cup.T, O, O, O, O, O],
                   [t * Cup, O, O, O, O, O],
                   [-t * Cdn.T, O, O, O, O, O],
                   [t * Cdn, O, O, O, O, O],
                   [onsite, Cup @ F, Cup.T @ F, Cdn @ F, Cdn.T @ F, Id]])


def tfi_bulk(h=1.0):
    """``H = -sum Z_i Z_{i+1} - h sum X_i`` (Pauli matrices), bulk ``[Id 0 0; Z 0 0; -hX -Z Id]``."""
    Z = np.diag([1.0, -1.0])
    X = np.array([[0.0, 1.0], [1.0, 0.0]])
    O = np.zeros((2, 2))
    Id = np.eye(2)
    return _block([[Id, O, O], [Z, O, O], [-h * X, -Z, Id]])


def make_mpo(bulks, d):
    """``makeMPO`` (``lib/MPO/makeMPO.jl:59-92``): list of site bulk matrices -> list of W[w,s,t,w']."""
    L = len(bulks)
    out = []
    for i, H in enumerate(bulks):
        a1 = H.shape[0] // d
        a2 = H.shape[1] // d
        G = H.reshape(a1, d, a2, d).transpose(0, 1, 3, 2).copy()  # G[l,j,k,m] = H[l*d+j, m*d+k]
        out.append(G)
    out[0] = out[0][-1:, :, :, :].copy()
    out[-1] = out[-1][:, :, :, :1].copy()
    return out


def cylinder_heisenberg_bulks(W, Lx, J=1.0):
    """Site bulk matrices of the Heisenberg model on a W x Lx cylinder (periodic in W, open in x),
    snake-ordered, built as a finite-state machine: every bond (i<j) of the lattice in 1-D order
    becomes a string ``S_i^a ... S_j^b`` carried by channels of range ``j-i``.

    Channel layout of the bulk matrix (size 2 + 3*R, R = max range):
    0 = "done" (identity to the right), 1..3R = open strings (op a in {Sp,Sm,Sz}, distance
    travelled), last = "not started" (identity to the left). Returns one bulk per site.
    """
    N = W * Lx

    def site(x, y):  # snake order
        return x * W + (y if x % 2 == 0 else W - 1 - y)

    bonds = set()
    for x in range(Lx):
        for y in range(W):
            i = site(x, y)
            j = site(x, (y + 1) % W)
            if W > 2 or y + 1 < W:
                bonds.add((min(i, j), max(i, j)))
            if x + 1 < Lx:
                j = site(x + 1, y)
                bonds.add((min(i, j), max(i, j)))
    R = max(j - i for i, j in bonds)
    Sp, Sm, Sz, _, _, O, Id = spin_ops(0.5)
    first = [Sp, Sm, Sz]              # op placed at the left site i
    second = [0.5 * J * Sm, 0.5 * J * Sp, J * Sz]   # op placed at the right site j
    nch = 2 + 3 * R
    bulks = []
    for s in range(N):
        M = [[O for _ in range(nch)] for _ in range(nch)]
        M[0][0] = Id
        M[nch - 1][nch - 1] = Id

        def ch(a, dist):
            return 1 + a * R + (dist - 1)

        # lower-triangular: row = left channel (after the site), col = right channel? In the
        # makeMPO convention the product runs W1 W2 ... with site 1 keeping the last ROW, so the
        # string enters from the last row and exits to the first column.
        # rows = left bond state, cols = right bond state; a string enters from the last row
        # ("not started") and leaves through column 0 ("done"), as in the bulk Heisenberg form.
        starts_here = any(i == s for (i, j) in bonds)
        for a in range(3):
            if starts_here:
                M[nch - 1][ch(a, 1)] = first[a]
            for dist in range(1, R + 1):
                i0 = s - dist                       # site where this string started
                if i0 < 0:
                    continue
                if (i0, s) in bonds:                # close bond (i0, s)
                    M[ch(a, dist)][0] = M[ch(a, dist)][0] + second[a]
                if dist < R and any(i == i0 and j > s for (i, j) in bonds):
                    M[ch(a, dist)][ch(a, dist + 1)] = Id
        bulks.append(np.block(M))
    return bulks


def prune_mpo(mpo):
    """Remove MPO bond states that carry no weight from either side (pure bookkeeping; keeps H)."""
    mpo = [w.copy() for w in mpo]
    changed = True
    while changed:
        changed = False
        for i in range(len(mpo) - 1):
            A, B = mpo[i], mpo[i + 1]
            keep = [w for w in range(A.shape[3])
                    if np.any(A[:, :, :, w] != 0) and np.any(B[w] != 0)]
            if len(keep) < A.shape[3]:
                mpo[i] = A[:, :, :, keep]
                mpo[i + 1] = B[keep]
                changed = True
    return mpo


# ------------------------------------------------------------------ QN labels

def mpo_bond_labels(mpo, phys_qn):
    """Right-bond labels of every MPO tensor (``makeqMPO`` rule: the QN carrying the largest
    summed weight ``|W|^4``). ``phys_qn[i]``: list of QN tuples of site i's states.
    Returns ``r`` with ``r[i]`` the labels of the bond left of site i (``r[0] = [0]``)."""
    nsym = len(phys_qn[0][0])
    zero = tuple(0 for _ in range(nsym))
    r = [[zero] * mpo[0].shape[0]]
    for i, W in enumerate(mpo):
        p = phys_qn[i]
        right = []
        for w2 in range(W.shape[3]):
            tot = {}
            for w1 in range(W.shape[0]):
                for s in range(W.shape[1]):
                    for t in range(W.shape[2]):
                        q = tuple(a - b + c for a, b, c in zip(r[i][w1], p[s], p[t]))
                        tot[q] = tot.get(q, 0.0) + abs(W[w1, s, t, w2]) ** 4
            best = max(tot.items(), key=lambda kv: kv[1]) if tot else (zero, 0.0)
            right.append(best[0] if best[1] > 0 else zero)
        r.append(right)
    return r


def mps_bond_labels(mps, phys_qn):
    """Bond labels of a dense MPS (``assignflux!``: label of the largest |element|).
    ``q[i]`` = labels of the bond left of site i; ``q[0] = [0]``; ``q[L]`` = total."""
    nsym = len(phys_qn[0][0])
    zero = tuple(0 for _ in range(nsym))
    q = [[zero] * mps[0].shape[0]]
    for i, A in enumerate(mps):
        right = []
        for b in range(A.shape[2]):
            blk = np.abs(A[:, :, b])
            a, s = np.unravel_index(int(np.argmax(blk)), blk.shape)
            right.append(tuple(x + y for x, y in zip(q[i][a], phys_qn[i][s])))
        q.append(right)
    return q


def _group_bond(labels):
    """Sectors (sorted unique QNs) and the permutation of states that groups them."""
    qs = sorted(set(labels))
    perm = []
    dims = []
    for qv in qs:
        idx = [n for n, x in enumerate(labels) if x == qv]
        perm += idx
        dims.append(len(idx))
    return qs, dims, perm


def to_qmps(mps, phys_qn):
    """Dense MPS + physical labels -> list of QTensor A[a(+1), s(+1), b(-1)] (bond states grouped
    by QN, i.e. a permutation of each bond basis -- a gauge change)."""
    q = mps_bond_labels(mps, phys_qn)
    L = len(mps)
    bonds = []
    perms = []
    for i in range(L + 1):
        qs, dims, perm = _group_bond(q[i])
        bonds.append((qs, dims))
        perms.append(perm)
    out = []
    for i, A in enumerate(mps):
        Ap = A[perms[i]][:, :, perms[i + 1]]
        ia = Index(bonds[i][0], bonds[i][1], +1)
        isx = Index(phys_qn[i], [1] * len(phys_qn[i]), +1)
        ib = Index(bonds[i + 1][0], bonds[i + 1][1], -1)
        out.append(from_dense(Ap, [ia, isx, ib], tuple(0 for _ in phys_qn[i][0])))
    return out


def to_qmpo(mpo, phys_qn):
    """Dense MPO + physical labels -> list of QTensor W[w(+1), s(-1), t(+1), w'(-1)]."""
    r = mpo_bond_labels(mpo, phys_qn)
    out = []
    for i, W in enumerate(mpo):
        iw = Index(r[i], [1] * len(r[i]), +1)
        ip = Index(phys_qn[i], [1] * len(phys_qn[i]), +1)
        iw2 = Index(r[i + 1], [1] * len(r[i + 1]), -1)
        out.append(from_dense(W, [iw, ip.dual(), ip, iw2], tuple(0 for _ in phys_qn[i][0])))
    return out


# ------------------------------------------------------------------ initial states

def neel_mps(L, d=2):
    """Product state: site i (1-based) up if odd, down if even (``test/dmrg_test.jl:55-58``)."""
    out = []
    for i in range(L):
        A = np.zeros((1, d, 1))
        A[0, 0 if i % 2 == 0 else 1, 0] = 1.0
        out.append(A)
    return out


def product_mps(states, d):
    out = []
    for s in states:
        A = np.zeros((1, d, 1))
        A[0, s, 0] = 1.0
        out.append(A)
    return out


def apply_ops(mps, sites, op, trail=None):
    """``applyOps!`` (``lib/MPO_MPS/applyMPO.jl:21-34``): ``psi[p] = Op . psi[p]`` on the physical
    index for every p in ``sites``, and the trailing operator on all sites left of p."""
    mps = [A.copy() for A in mps]
    for p in sites:
        mps[p] = np.einsum("st,atb->asb", op, mps[p])
        if trail is not None:
            for j in range(p):
                mps[j] = np.einsum("st,atb->asb", trail, mps[j])
    return mps


def hubbard_half_filling_mps(L):
    """N=L, Sz=0 start of ``test/dmrg_test.jl:62-75`` / ``test/model_test.jl:324-336``: apply
    Cup^dagger then Cdn^dagger (with the JW string F on the left) to the vacuum on sites 1..L/2."""
    Cup, Cdn, F, *_ = fermion_ops()
    psi = product_mps([0] * L, 4)
    nup = L // 2                                     # Ne_up = ceil(div(Ne,2)), Ne = L
    psi = apply_ops(psi, list(range(nup)), Cup.T, trail=F)
    psi = apply_ops(psi, list(range(L - nup)), Cdn.T, trail=F)
    return psi


def random_mps(L, d, m, rng):
    """Random dense MPS with bond dimension ``min(d^k, d^(L-k), m)`` after site k and entries
    ``rng.standard_normal``, each tensor normalised (the seeded stand-in for ``randMPS``'s uniform
    ``rand`` at ``lib/MPS/randMPS.jl:27-56``)."""
    dims = [min(d ** k, d ** (L - k), m) for k in range(L + 1)]
    out = []
    for i in range(L):
        A = rng.standard_normal((dims[i], d, dims[i + 1]))
        out.append(A / np.linalg.norm(A))
    return out


def right_canonicalize(mps):
    """Move the orthogonality centre to site 1 by LQ sweeps from the right (``moveL!`` with the
    exact ``lq`` branch, ``lib/MPS/move.jl:124-139``) and normalise the centre tensor."""
    mps = [A.copy() for A in mps]
    for i in range(len(mps) - 1, 0, -1):
        A = mps[i]
        a, d, b = A.shape
        M = A.reshape(a, d * b)
        Q, R = np.linalg.qr(M.T)          # M = R^T Q^T  (LQ)
        k = Q.shape[1]
        mps[i] = Q.T.reshape(k, d, b)
        mps[i - 1] = np.tensordot(mps[i - 1], R.T, axes=(2, 0))
    mps[0] = mps[0] / np.linalg.norm(mps[0])
    return mps
