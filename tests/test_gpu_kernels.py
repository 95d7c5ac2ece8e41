"""Single-kernel checks through the C ABI test hooks: the grouped FP64 GEMM (NN/NT/TN, ragged
sizes around the 64x64x16 tile) and the batched Jacobi eigensolver, against numpy FP64.

Tolerance: FP64 GEMM results within 1e-13 relative to sum_k |a_ik||b_kj|; eigenvalues within
tol * ||A||, eigenvectors orthonormal to tol and A V = V diag(w) to tol * ||A||, with
tol = 2e-13 sqrt(n) (rounding of O(n) rotations per sweep).
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


@pytest.mark.parametrize("sizes", [[1, 2, 3, 17, 64, 100], [101, 160], [37, 250, 5], [480], [1000]])
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
        tol = 2e-13 * np.sqrt(n)
        assert np.max(np.abs(lam - ref)) < tol * max(nrm, 1)
        assert np.max(np.abs(V.T @ V - np.eye(n))) < tol
        assert np.max(np.abs(M @ V - V * lam)) < tol * max(nrm, 1)
        off += n * n
        woff += n


def _rho_like(rng, n, kind):
    if kind == "rank":
        X = rng.standard_normal((n, max(1, n // 2)))
        return X @ X.T / n
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if kind == "deg":        # exact pairs and quadruplets (multiplets) and a null space
        w = np.zeros(n)
        m = n // 3
        w[:2 * m:2] = np.exp(-np.arange(m))
        w[1:2 * m:2] = np.exp(-np.arange(m))
    else:                    # 16 decades of decay, like a converged Schmidt spectrum
        w = 10.0 ** (-np.arange(n) * 16.0 / n)
    A = (Q * w) @ Q.T
    return 0.5 * (A + A.T)


@pytest.mark.parametrize("case", [[(66, "rank", 40), (1, "rank", 1), (2, "rank", 2), (3, "rank", 1)],
                                  [(66, "deg", 50), (90, "deg", 60)],
                                  [(112, "decay", 100), (40, "decay", 40)],
                                  # mid-size blocks (global-memory Householder steps, then shared)
                                  [(113, "decay", 113), (66, "rank", 30), (240, "rank", 120)],
                                  [(233, "deg", 150), (160, "decay", 1)],
                                  [(512, "decay", 400), (300, "rank", 150), (129, "deg", 80)]])
def test_tridiagonal_eigensolver(dmrgb, ctx, case):
    """All eigenvalues within 2e-14 ||A||; the k kept eigenvectors orthonormal to 1e-13 and with
    residual ||A u - lambda u|| <= 1e-12 ||A|| (the truncation's tolerance needs)."""
    rng = np.random.default_rng(len(case))
    mats = [_rho_like(rng, n, kind) for n, kind, _ in case]
    ns = [n for n, _, _ in case]
    ks = [k for _, _, k in case]
    A = np.concatenate([np.asfortranarray(M).ravel(order="F") for M in mats])
    w = np.zeros(sum(ns))
    U = np.zeros(sum(n * k for n, k in zip(ns, ks)))
    code = dmrgb.lib().dmrg_test_syevt(ctx.h, len(ns), (C.c_int * len(ns))(*ns),
                                       (C.c_int * len(ks))(*ks), A.ctypes.data_as(DP),
                                       w.ctypes.data_as(DP), U.ctypes.data_as(DP))
    assert code == 0, dmrgb.lib().dmrg_last_error(ctx.h)
    ow = ou = 0
    for M, n, k in zip(mats, ns, ks):
        lam = w[ow:ow + n]
        ref = np.sort(np.linalg.eigvalsh(M))[::-1]
        nrm = max(np.linalg.norm(M, 2), 1e-300)
        assert np.max(np.abs(lam - ref)) < 2e-14 * nrm
        Uk = U[ou:ou + n * k].reshape((n, k), order="F")
        assert np.max(np.abs(Uk.T @ Uk - np.eye(k))) < 1e-13
        assert np.max(np.abs(M @ Uk - Uk * lam[:k])) < 1e-12 * nrm
        ow += n
        ou += n * k


def test_tile_autotuner_keeps_every_number(dmrgb, ctx):
    """The FP64 GEMM tile autotuner (64 x 64 or 32 x 32 tiles per block-size histogram) changes
    only the time: a U(1) run with it and one with fixed 64 x 64 tiles agree bit for bit, and the
    tuner has timed both shapes for the histograms it met."""
    L = 40
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    out = {}
    for tune in (False, True):
        dev = dmrgb.DeviceState(dmrgb.neelMPS(L), mpo.device(ctx))
        dev.env_build()
        st = [dev.sweep(dmrgb.make_params(maxm=m, cutoff=1e-12, tune=tune))
              for m in (16, 32, 64, 64, 64)]
        out[tune] = ([s["energy"] for s in st], [s["max_truncerr"] for s in st],
                     dev.site_blocks(L // 2))
    assert out[True][0] == out[False][0]
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][2], out[False][2])
    sig, decided, small = ctx.tuner()
    assert sig > 0 and decided > 0 and 0 <= small <= decided


@pytest.mark.parametrize("krylov,precision", [(2, "fp64"), (8, "fp64"), (2, "3xtf32")])
def test_graph_krylov_step_keeps_every_number(dmrgb, ctx, krylov, precision):
    """The Lanczos step as one CUDA graph per bond step (graph = 1) gives the same bits as plain
    launches, and every bond step of the sweep ran its graph."""
    L = 24
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    out = {}
    for graph in (False, True):
        dev = dmrgb.DeviceState(dmrgb.neelMPS(L), mpo.device(ctx))
        dev.env_build()
        st = [dev.sweep(dmrgb.make_params(maxm=m, cutoff=1e-12, krylov=krylov,
                                          precision=precision, graph=graph))
              for m in (16, 32, 48)]
        out[graph] = ([s["energy"] for s in st], dev.site_blocks(L // 2))
        if graph:
            assert all(s["graph_launches"] == 2 * (L - 1) for s in st)
    assert out[True][0] == out[False][0]
    assert np.array_equal(out[True][1], out[False][1])
