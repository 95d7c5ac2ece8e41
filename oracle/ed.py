"""Exact diagonalisation of a dense MPO (test infrastructure).

``fullH`` (``lib/MPO/fullmpo.jl:17-38``) contracts the MPO into the full Hamiltonian; the
reference's known answer ``test/MPtask_test.jl:317-334`` is its lowest eigenvalue. For chains
too long for a dense matrix a sparse ``scipy.sparse.linalg.eigsh`` is used instead.
"""
from __future__ import annotations

import numpy as np


def full_h(mpo):
    """Full Hamiltonian ``H[(s_1..s_L), (t_1..t_L)]`` from W[w,s,t,w'] (ket s, bra t)."""
    T = mpo[0][0]                      # [s, t, w']  (left edge dim 1)
    dim = mpo[0].shape[1]
    T = T.reshape(dim, dim, -1)
    for W in mpo[1:]:
        d = W.shape[1]
        # T[S, T, w] W[w, s, t, w'] -> [S s, T t, w']
        T = np.einsum("abw,wstv->asbtv", T, W)
        n1, n2 = T.shape[0] * T.shape[1], T.shape[2] * T.shape[3]
        T = T.reshape(n1, n2, -1)
    return T[:, :, 0]


def ground_energy(mpo):
    H = full_h(mpo)
    H = 0.5 * (H + H.T)
    return float(np.linalg.eigvalsh(H)[0])


def sparse_ground_energy(mpo, k=1):
    """Lowest eigenvalue through a matrix-free MPO application (for up to ~20 sites of d=2)."""
    from scipy.sparse.linalg import LinearOperator, eigsh
    dims = [W.shape[1] for W in mpo]
    N = int(np.prod(dims))

    def mv(x):
        # contract the MPO string with x[s_1..s_L] one site at a time
        v = x.reshape([1] + dims)                 # [w, s_1..s_L]
        for n, W in enumerate(mpo):
            # v[w, t_1..t_{n}, s_{n+1}..] -> apply W on site n (ket s -> bra t)
            v = np.tensordot(v, W, axes=([0, n + 1], [0, 1]))   # [.., t, w']
            v = np.moveaxis(v, -1, 0)                            # w' first
            v = np.moveaxis(v, -1, n + 1)                        # t back in place
        return v.reshape(N)

    op = LinearOperator((N, N), matvec=mv, dtype=float)
    vals = eigsh(op, k=k, which="SA", tol=1e-12)[0]
    return float(np.min(vals))
