"""Dense and abelian (U(1)^nsym) block-sparse tensors for the CPU oracle (test infrastructure).

DMRJtensor.jl takes all of its tensor arithmetic from TensorPACK 0.14.1 (``lib/imports.jl:44-81``),
which is not vendored with the reference. This module restates the published semantics the
reference's hot path relies on:

* ``contract(A, iA, B, iB)``: sum over the listed index pairs; the result keeps A's free indices
  in order followed by B's free indices (``contract``/``ccontract``/``contractc`` call sites at
  ``algs/DMRG.jl:23-90`` and ``lib/MPO_MPS/Lupdate.jl:20-25``). ``ccontract`` conjugates the first
  operand, ``contractc`` the second. Data here is real FP64, so conjugation only flips arrows.
* ``svd``/``eigh`` of a tensor reshaped into a matrix ``[[left],[right]]`` with a truncation that
  is global over all QN blocks (``fsvd!`` at ``algs/DMRG.jl:387``, ``eigen`` at ``algs/DMRG.jl:467``).

Quantum numbers: every index is a list of sectors (QN tuple, dimension) and an arrow (+1 in,
-1 out). A block ``(k_1..k_n)`` is allowed iff ``sum_i arrow_i * qn(k_i) == flux``.
Dense tensors are plain ``numpy.ndarray`` (column-major reasoning only matters at the boundary;
numpy index order here equals the Julia index order).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "Index", "QTensor", "contract", "ccontract", "contractc", "norm", "inner", "scale", "axpy",
    "permute", "svd_trunc", "eigh_trunc", "select_kept", "to_dense", "from_dense",
]


class Index:
    """One tensor index: ordered sectors ``qns[k]`` (tuple of ints) with ``dims[k]`` states."""

    __slots__ = ("qns", "dims", "arrow")

    def __init__(self, qns, dims, arrow):
        self.qns = tuple(tuple(int(x) for x in q) for q in qns)
        self.dims = tuple(int(d) for d in dims)
        self.arrow = int(arrow)

    def dual(self) -> "Index":
        return Index(self.qns, self.dims, -self.arrow)

    @property
    def size(self) -> int:
        return int(sum(self.dims))

    def offsets(self):
        off, out = 0, []
        for d in self.dims:
            out.append(off)
            off += d
        return out

    def same_space(self, other: "Index") -> bool:
        return self.qns == other.qns and self.dims == other.dims

    def __repr__(self):
        return f"Index({list(zip(self.qns, self.dims))}, arrow={self.arrow})"


def _qadd(a, b, sign=1):
    return tuple(x + sign * y for x, y in zip(a, b))


class QTensor:
    """Block-sparse tensor: ``blocks[(k_1..k_n)] -> ndarray`` of shape ``(dims[k_1], .., dims[k_n])``."""

    __slots__ = ("indices", "blocks", "flux")

    def __init__(self, indices, blocks, flux):
        self.indices = list(indices)
        self.blocks = dict(blocks)
        self.flux = tuple(int(x) for x in flux)

    @property
    def ndim(self):
        return len(self.indices)

    @property
    def shape(self):
        return tuple(ix.size for ix in self.indices)

    def copy(self):
        return QTensor(self.indices, {k: v.copy() for k, v in self.blocks.items()}, self.flux)

    def nnz(self):
        return int(sum(v.size for v in self.blocks.values()))

    def allowed(self, key) -> bool:
        tot = tuple(0 for _ in self.flux)
        for ix, k in zip(self.indices, key):
            tot = _qadd(tot, ix.qns[k], ix.arrow)
        return tot == self.flux


def _conj_t(T):
    if isinstance(T, np.ndarray):
        return T  # real data
    return QTensor([ix.dual() for ix in T.indices], T.blocks, tuple(-x for x in T.flux))


def _as_tuple(ix):
    if isinstance(ix, (int, np.integer)):
        return (int(ix),)
    return tuple(int(i) for i in ix)


def _tensordot_q(A: QTensor, B: QTensor, axA, axB) -> QTensor:
    for i, j in zip(axA, axB):
        a, b = A.indices[i], B.indices[j]
        if not a.same_space(b):
            raise ValueError(f"contracted index spaces differ: {a} vs {b}")
        if a.arrow == b.arrow:
            raise ValueError("contracted indices must have opposite arrows")
    freeA = [i for i in range(A.ndim) if i not in axA]
    freeB = [j for j in range(B.ndim) if j not in axB]
    out_idx = [A.indices[i] for i in freeA] + [B.indices[j] for j in freeB]
    flux = _qadd(A.flux, B.flux)
    groupB = {}
    for kb, vb in B.blocks.items():
        groupB.setdefault(tuple(kb[j] for j in axB), []).append((kb, vb))
    out = {}
    for ka, va in A.blocks.items():
        ck = tuple(ka[i] for i in axA)
        for kb, vb in groupB.get(ck, ()):
            key = tuple(ka[i] for i in freeA) + tuple(kb[j] for j in freeB)
            r = np.tensordot(va, vb, axes=(list(axA), list(axB)))
            if key in out:
                out[key] += r
            else:
                out[key] = r
    return QTensor(out_idx, out, flux)


def contract(A, iA, B, iB):
    """``contract(A,iA,B,iB)``: 0-based axes; free A indices then free B indices."""
    iA, iB = _as_tuple(iA), _as_tuple(iB)
    if isinstance(A, np.ndarray):
        return np.tensordot(A, B, axes=(list(iA), list(iB)))
    return _tensordot_q(A, B, iA, iB)


def ccontract(A, iA, B, iB):
    """conj(A) contracted with B."""
    return contract(_conj_t(A), iA, B, iB)


def contractc(A, iA, B, iB):
    """A contracted with conj(B)."""
    return contract(A, iA, _conj_t(B), iB)


def inner(A, B) -> float:
    """Full contraction ``ccontract(A,B)`` (the scalar <A|B>)."""
    if isinstance(A, np.ndarray):
        return float(np.vdot(A, B))
    s = 0.0
    for k, v in A.blocks.items():
        w = B.blocks.get(k)
        if w is not None:
            s += float(np.vdot(v, w))
    return s


def norm(A) -> float:
    if isinstance(A, np.ndarray):
        return float(np.linalg.norm(A))
    return float(np.sqrt(sum(float(np.vdot(v, v)) for v in A.blocks.values())))


def scale(A, c):
    if isinstance(A, np.ndarray):
        return A * c
    return QTensor(A.indices, {k: v * c for k, v in A.blocks.items()}, A.flux)


def axpy(ca, A, cb, B):
    """``ca*A + cb*B`` (same index structure)."""
    if isinstance(A, np.ndarray):
        return ca * A + cb * B
    out = {k: ca * v for k, v in A.blocks.items()}
    for k, v in B.blocks.items():
        if k in out:
            out[k] = out[k] + cb * v
        else:
            out[k] = cb * v
    return QTensor(A.indices, out, A.flux)


def permute(A, perm):
    perm = list(perm)
    if isinstance(A, np.ndarray):
        return np.transpose(A, perm)
    return QTensor([A.indices[p] for p in perm],
                   {tuple(k[p] for p in perm): np.transpose(v, perm) for k, v in A.blocks.items()},
                   A.flux)


def to_dense(A) -> np.ndarray:
    if isinstance(A, np.ndarray):
        return A
    out = np.zeros(A.shape)
    offs = [ix.offsets() for ix in A.indices]
    for k, v in A.blocks.items():
        sl = tuple(slice(offs[n][kk], offs[n][kk] + v.shape[n]) for n, kk in enumerate(k))
        out[sl] = v
    return out


def from_dense(arr, indices, flux, check_tol=1e-12) -> QTensor:
    """Blocks of ``arr`` that the QN rule allows; raises if a forbidden block is non-zero."""
    import itertools
    T = QTensor(indices, {}, flux)
    offs = [ix.offsets() for ix in indices]
    for key in itertools.product(*[range(len(ix.dims)) for ix in indices]):
        sl = tuple(slice(offs[n][k], offs[n][k] + indices[n].dims[k]) for n, k in enumerate(key))
        blk = arr[sl]
        if T.allowed(key):
            T.blocks[key] = np.array(blk, dtype=float)
        elif blk.size and np.max(np.abs(blk)) > check_tol:
            raise ValueError(f"non-zero data in QN-forbidden block {key}")
    return T


# ----------------------------------------------------------------------------------------------
# truncation rule (TensorPACK's is not visible; this one is written down and shared by all paths)
# ----------------------------------------------------------------------------------------------

def select_kept(groups_vals, maxm=0, minm=0, cutoff=0.0, mag=1.0, degen_rtol=0.0):
    """Choose how many values to keep per group.

    ``groups_vals``: list of 1-D arrays of *weights* (squared singular values / eigenvalues of the
    reduced density matrix), each sorted descending. Rule (global over all groups):

    1. Order all weights descending; ties broken by (group order, position in group).
    2. ``k_c`` = smallest k >= 1 with sum_{i>k} w_i <= cutoff * mag (``mag=1`` as at
       ``algs/DMRG.jl:387``; ``mag=0`` means "use the total weight").
    3. ``k = min(maxm, max(minm, k_c), N)`` (``maxm <= 0`` means unlimited).
    4. If ``degen_rtol > 0`` and the cut at k splits a cluster of weights that are equal within
       ``degen_rtol * w_k``, the whole cluster is dropped (never below ``max(minm,1)``).
    Returns ``(kept_per_group, truncerr)`` with truncerr = sum of the discarded weights.
    """
    flat = []
    for g, vals in enumerate(groups_vals):
        for i, v in enumerate(vals):
            flat.append((-float(v), g, i))
    flat.sort()
    w = np.array([-x[0] for x in flat], dtype=float)
    N = len(w)
    if N == 0:
        return [0 for _ in groups_vals], 0.0
    tot = float(np.sum(w)) if mag == 0 else float(mag)
    # tail[k] = sum_{i>=k} w_i  (0-based), so discarding from position k on costs tail[k]
    tail = np.concatenate([np.cumsum(w[::-1])[::-1], [0.0]])
    kc = N
    for k in range(1, N + 1):
        if tail[k] <= cutoff * tot:
            kc = k
            break
    k = max(minm, kc)
    if maxm and maxm > 0:
        k = min(k, maxm)
    k = max(1, min(k, N))
    if degen_rtol > 0 and k < N:
        thr = degen_rtol * abs(w[k - 1])
        if w[k - 1] - w[k] <= thr:                   # the cut splits a cluster
            j = k - 1
            while j >= 1 and w[j - 1] - w[j] <= thr:
                j -= 1
            if j >= max(minm, 1):                    # drop the whole cluster
                k = j
    kept = [0 for _ in groups_vals]
    for n in range(k):
        kept[flat[n][1]] += 1
    return kept, float(tail[k])


# ----------------------------------------------------------------------------------------------
# matricisation helpers for the decompositions
# ----------------------------------------------------------------------------------------------

def _matricize(T: QTensor, left, right):
    """Group blocks by the combined left charge. Returns {QL: dict} with row/col layouts."""
    groups = {}
    nsym = len(T.flux)
    for key, blk in T.blocks.items():
        QL = tuple(0 for _ in range(nsym))
        for a in left:
            QL = _qadd(QL, T.indices[a].qns[key[a]], T.indices[a].arrow)
        g = groups.setdefault(QL, {"rows": {}, "cols": {}, "blocks": []})
        lk = tuple(key[a] for a in left)
        rk = tuple(key[a] for a in right)
        g["rows"].setdefault(lk, int(np.prod([T.indices[a].dims[key[a]] for a in left])))
        g["cols"].setdefault(rk, int(np.prod([T.indices[a].dims[key[a]] for a in right])))
        g["blocks"].append((lk, rk, blk))
    out = {}
    for QL in sorted(groups):
        g = groups[QL]
        rkeys = sorted(g["rows"])
        ckeys = sorted(g["cols"])
        roff, o = {}, 0
        for r in rkeys:
            roff[r] = o
            o += g["rows"][r]
        nr = o
        coff, o = {}, 0
        for c in ckeys:
            coff[c] = o
            o += g["cols"][c]
        nc = o
        M = np.zeros((nr, nc))
        for lk, rk, blk in g["blocks"]:
            nrb, ncb = g["rows"][lk], g["cols"][rk]
            M[roff[lk]:roff[lk] + nrb, coff[rk]:coff[rk] + ncb] = blk.reshape(nrb, ncb, order="C")
        out[QL] = dict(M=M, rkeys=rkeys, roff=roff, rdim=g["rows"], ckeys=ckeys, coff=coff,
                       cdim=g["cols"])
    return out


def _left_shape(T, left, lk):
    return tuple(T.indices[a].dims[k] for a, k in zip(left, lk))


def svd_trunc(T, left, right, maxm=0, minm=0, cutoff=0.0, mag=1.0, degen_rtol=0.0):
    """Truncated SVD ``T[[left],[right]] = U D V`` (``fsvd!`` semantics at ``algs/DMRG.jl:387``).

    Returns ``U, D, V, truncerr`` where ``D`` is the vector of kept singular values (descending,
    global order) for dense input, or a list of per-sector vectors for block-sparse input.
    U carries the left indices plus the new bond; V the new bond plus the right indices.
    """
    left, right = list(left), list(right)
    if isinstance(T, np.ndarray):
        sl = [T.shape[a] for a in left]
        sr = [T.shape[a] for a in right]
        M = np.transpose(T, left + right).reshape(int(np.prod(sl)), int(np.prod(sr)))
        U, s, Vt = np.linalg.svd(M, full_matrices=False)
        kept, terr = select_kept([s ** 2], maxm, minm, cutoff, mag, degen_rtol)
        k = kept[0]
        return (U[:, :k].reshape(sl + [k]), s[:k].copy(), Vt[:k, :].reshape([k] + sr), terr)
    mats = _matricize(T, left, right)
    QLs = list(mats)
    svds = []
    for QL in QLs:
        U, s, Vt = np.linalg.svd(mats[QL]["M"], full_matrices=False)
        svds.append((U, s, Vt))
    kept, terr = select_kept([s ** 2 for _, s, _ in svds], maxm, minm, cutoff, mag, degen_rtol)
    nsym = len(T.flux)
    new_qns, new_dims, Ublk, Vblk, Ds = [], [], {}, {}, []
    for QL, (U, s, Vt), k in zip(QLs, svds, kept):
        if k == 0:
            continue
        sec = len(new_qns)
        new_qns.append(QL)
        new_dims.append(k)
        Ds.append(s[:k].copy())
        m = mats[QL]
        for lk in m["rkeys"]:
            r0, nr = m["roff"][lk], m["rdim"][lk]
            Ublk[lk + (sec,)] = U[r0:r0 + nr, :k].reshape(_left_shape(T, left, lk) + (k,))
        for rk in m["ckeys"]:
            c0, nc = m["coff"][rk], m["cdim"][rk]
            Vblk[(sec,) + rk] = Vt[:k, c0:c0 + nc].reshape((k,) + _left_shape(T, right, rk))
    bond_out = Index(new_qns, new_dims, -1)
    Ut = QTensor([T.indices[a] for a in left] + [bond_out], Ublk, tuple(0 for _ in range(nsym)))
    Vt_ = QTensor([bond_out.dual()] + [T.indices[a] for a in right], Vblk, T.flux)
    return Ut, Ds, Vt_, terr


def eigh_trunc(rho, left, right, maxm=0, minm=0, cutoff=0.0, mag=1.0, degen_rtol=0.0):
    """Truncated eigendecomposition of a Hermitian ``rho[[left],[right]]`` (``eigen`` at
    ``algs/DMRG.jl:467``). Returns ``D`` (kept eigenvalues), ``U`` with the left indices plus the
    new bond (columns = eigenvectors) and the truncation error (sum of discarded eigenvalues)."""
    left, right = list(left), list(right)
    if isinstance(rho, np.ndarray):
        sl = [rho.shape[a] for a in left]
        M = np.transpose(rho, left + right).reshape(int(np.prod(sl)), -1)
        M = 0.5 * (M + M.T)
        lam, V = np.linalg.eigh(M)
        lam, V = lam[::-1], V[:, ::-1]
        kept, terr = select_kept([lam], maxm, minm, cutoff, mag, degen_rtol)
        k = kept[0]
        return lam[:k].copy(), V[:, :k].reshape(sl + [k]), terr
    mats = _matricize(rho, left, right)
    QLs = list(mats)
    eigs = []
    for QL in QLs:
        m = mats[QL]
        if m["rkeys"] != m["ckeys"]:
            raise ValueError("density matrix block is not square in its row/col layout")
        M = 0.5 * (m["M"] + m["M"].T)
        lam, V = np.linalg.eigh(M)
        eigs.append((lam[::-1], V[:, ::-1]))
    kept, terr = select_kept([lam for lam, _ in eigs], maxm, minm, cutoff, mag, degen_rtol)
    nsym = len(rho.flux)
    new_qns, new_dims, Ublk, Ds = [], [], {}, []
    for QL, (lam, V), k in zip(QLs, eigs, kept):
        if k == 0:
            continue
        sec = len(new_qns)
        new_qns.append(QL)
        new_dims.append(k)
        Ds.append(lam[:k].copy())
        m = mats[QL]
        for lk in m["rkeys"]:
            r0, nr = m["roff"][lk], m["rdim"][lk]
            Ublk[lk + (sec,)] = V[r0:r0 + nr, :k].reshape(_left_shape(rho, left, lk) + (k,))
    bond_out = Index(new_qns, new_dims, -1)
    Ut = QTensor([rho.indices[a] for a in left] + [bond_out], Ublk, tuple(0 for _ in range(nsym)))
    return Ds, Ut, terr


def rho_trunc(T, left, right, side, maxm=0, minm=0, cutoff=0.0, mag=1.0, degen_rtol=0.0):
    """Truncated decomposition through the reduced density matrix (``algs/DMRG.jl:425-429,
    467,483-490``), returned in the same form as :func:`svd_trunc`.

    ``side=+1`` (sweep to the right): ``rho = M M^T``; U = kept eigenvectors (an isometry),
    V = U^T M (= D V of the SVD). ``side=-1``: ``rho = M^T M``; V = kept eigenvectors^T,
    U = M V^T (= U D). ``D`` holds sqrt of the kept eigenvalues (negative rounding clipped to 0);
    the truncation error is the sum of the discarded eigenvalues.
    """
    left, right = list(left), list(right)

    def _decomp(M):
        G = M @ M.T if side > 0 else M.T @ M
        G = 0.5 * (G + G.T)
        lam, X = np.linalg.eigh(G)
        return lam[::-1], X[:, ::-1]

    if isinstance(T, np.ndarray):
        sl = [T.shape[a] for a in left]
        sr = [T.shape[a] for a in right]
        M = np.transpose(T, left + right).reshape(int(np.prod(sl)), int(np.prod(sr)))
        lam, X = _decomp(M)
        kept, terr = select_kept([lam], maxm, minm, cutoff, mag, degen_rtol)
        k = kept[0]
        D = np.sqrt(np.clip(lam[:k], 0.0, None))
        if side > 0:
            U = X[:, :k]
            V = U.T @ M
        else:
            V = X[:, :k].T
            U = M @ V.T
        return U.reshape(sl + [k]), D, V.reshape([k] + sr), terr
    mats = _matricize(T, left, right)
    QLs = list(mats)
    dec = [_decomp(mats[QL]["M"]) for QL in QLs]
    kept, terr = select_kept([lam for lam, _ in dec], maxm, minm, cutoff, mag, degen_rtol)
    nsym = len(T.flux)
    new_qns, new_dims, Ublk, Vblk, Ds = [], [], {}, {}, []
    for QL, (lam, X), k in zip(QLs, dec, kept):
        if k == 0:
            continue
        m = mats[QL]
        M = m["M"]
        if side > 0:
            Um = X[:, :k]
            Vm = Um.T @ M
        else:
            Vm = X[:, :k].T
            Um = M @ Vm.T
        sec = len(new_qns)
        new_qns.append(QL)
        new_dims.append(k)
        Ds.append(np.sqrt(np.clip(lam[:k], 0.0, None)))
        for lk in m["rkeys"]:
            r0, nr = m["roff"][lk], m["rdim"][lk]
            Ublk[lk + (sec,)] = Um[r0:r0 + nr, :].reshape(_left_shape(T, left, lk) + (k,))
        for rk in m["ckeys"]:
            c0, nc = m["coff"][rk], m["cdim"][rk]
            Vblk[(sec,) + rk] = Vm[:, c0:c0 + nc].reshape((k,) + _left_shape(T, right, rk))
    bond_out = Index(new_qns, new_dims, -1)
    Ut = QTensor([T.indices[a] for a in left] + [bond_out], Ublk, tuple(0 for _ in range(nsym)))
    Vt_ = QTensor([bond_out.dual()] + [T.indices[a] for a in right], Vblk, T.flux)
    return Ut, Ds, Vt_, terr


def dmul(U, D, axis):
    """Scale ``U`` along ``axis`` (the new bond) by ``D`` (``U*D`` / ``D*V`` at ``algs/DMRG.jl:389-395``)."""
    if isinstance(U, np.ndarray):
        shp = [1] * U.ndim
        shp[axis] = -1
        return U * np.asarray(D).reshape(shp)
    out = {}
    for key, blk in U.blocks.items():
        d = D[key[axis]]
        shp = [1] * blk.ndim
        shp[axis] = -1
        out[key] = blk * d.reshape(shp)
    return QTensor(U.indices, out, U.flux)
