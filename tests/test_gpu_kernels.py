"""Single-kernel checks through the C ABI test hooks: the grouped FP64 GEMM (NN/NT/TN, ragged
sizes around the 64x64x16 tile) and the batched Jacobi eigensolver, against numpy FP64.

Tolerance: FP64 GEMM results within 1e-13 relative to sum_k |a_ik||b_kj|; eigenvalues within
1e-13 * ||A||, eigenvectors orthonormal to 1e-12 and A V = V diag(w) to 1e-12 * ||A||.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DP = C.POINTER(C.c_double)


def _gemm(dmrgb, ctx, tA, tB, M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((K, M) if tA else (M, K))
    B = rng.standard_normal((N, K) if tB else (K, N))
    Af, Bf = np.asfortranarray(A), np.asfortranarray(B)
    Cf = np.asfortranarray(np.full((M, N), np.nan))
    code = dmrgb.lib().dmrg_test_gemm(ctx.h, int(tA), int(tB), M, N, K, Af.ctypes.data_as(DP),
                                      Af.shape[0], Bf.ctypes.data_as(DP), Bf.shape[0],
                                      Cf.ctypes.data_as(DP), M)
    assert code == 0, dmrgb.lib().dmrg_last_error(ctx.h)
    opA = A.T if tA else A
    opB = B.T if tB else B
    ref = opA @ opB
    scale = np.abs(opA) @ np.abs(opB) + 1e-300
    return float(np.max(np.abs(Cf - ref) / scale))


@pytest.mark.parametrize("tA,tB", [(0, 0), (0, 1), (1, 0)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (64, 64, 16), (65, 63, 17), (130, 7, 300),
                                   (5, 200, 33), (257, 129, 64)])
def test_gemm_variants(dmrgb, ctx, tA, tB, M, N, K):
    assert _gemm(dmrgb, ctx, tA, tB, M, N, K, seed=M * 7 + N + K) < 1e-13


def test_gemm_zero_k_writes_zero(dmrgb, ctx):
    M, N = 9, 5
    A = np.zeros((M, 1), order="F")
    B = np.zeros((1, N), order="F")
    Cf = np.asfortranarray(np.full((M, N), 7.0))
    code = dmrgb.lib().dmrg_test_gemm(ctx.h, 0, 0, M, N, 0, A.ctypes.data_as(DP), M,
                                      B.ctypes.data_as(DP), 1, Cf.ctypes.data_as(DP), M)
    assert code == 0
    assert np.all(Cf == 0.0)


@pytest.mark.parametrize("sizes", [[1, 2, 3, 17, 64, 100], [101, 160], [37, 250]])
def test_jacobi_batched(dmrgb, ctx, sizes):
    rng = np.random.default_rng(sum(sizes))
    mats = []
    for n in sizes:
        X = rng.standard_normal((n, max(1, n // 2)))
        mats.append(X @ X.T / n)   # PSD with a null space, like a reduced density matrix
    packed = np.concatenate([np.asfortranarray(M).ravel(order="F") for M in mats])
    w = np.zeros(sum(sizes))
    n_arr = (C.c_int * len(sizes))(*sizes)
    code = dmrgb.lib().dmrg_test_eigh(ctx.h, len(sizes), n_arr, packed.ctypes.data_as(DP),
                                      w.ctypes.data_as(DP))
    assert code == 0, dmrgb.lib().dmrg_last_error(ctx.h)
    off = woff = 0
    for n, M in zip(sizes, mats):
        V = packed[off:off + n * n].reshape((n, n), order="F")
        lam = w[woff:woff + n]
        ref = np.sort(np.linalg.eigvalsh(M))[::-1]
        nrm = np.linalg.norm(M, 2)
        assert np.all(np.diff(lam) <= 0)
        assert np.max(np.abs(lam - ref)) < 1e-13 * max(nrm, 1)
        assert np.max(np.abs(V.T @ V - np.eye(n))) < 1e-12
        assert np.max(np.abs(M @ V - V * lam)) < 1e-12 * max(nrm, 1)
        off += n * n
        woff += n
