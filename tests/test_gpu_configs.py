"""The benchmark definition's small configurations on the device against the oracle.

C1: dense Heisenberg L=20 from a bond-10 random MPS, maxm 100, cutoff 1e-12, 10 sweeps, Lanczos
with 8 Krylov vectors and the reference's 2-vector step (both converged by the last sweep, where
the invariants are compared: unconverged trajectories amplify rounding differences). Hubbard
U(1)xU(1) (N, 2Sz) at half filling from the product start of ``test/dmrg_test.jl:62-75`` (L=8). Invariants compared: energy 1e-10 relative, largest truncation
error and centre-bond entropy of the last sweep 1e-8.
"""
import numpy as np
import pytest

from oracle import dmrg as od, models as om

pytestmark = pytest.mark.gpu


def _compare(psi_dev, E, E0, info):
    st = psi_dev.sweep_stats[-1]
    o = info["sweeps"][-1]
    assert abs(E - E0) <= 1e-10 * abs(E0)
    assert abs(st["max_truncerr"] - o["maxtrunc"]) <= 1e-8
    assert abs(st["entropy"] - o["entropy"]) <= 1e-8


@pytest.mark.parametrize("krylov", [8, 2])
def test_c1_dense_heisenberg_l20(dmrgb, ctx, krylov):
    L = 20
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    ompo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    psi = dmrgb.randMPS(2, L, 10, seed=20)
    ref = [a.copy() for a in psi.tensors]
    E = dmrgb.dmrg(psi, mpo, m=100, sweeps=10, cutoff=1e-12, krylov=krylov, ctx=ctx)
    E0, info = od.dmrg(ref, ompo, m=100, sweeps=10, cutoff=1e-12, krylov=krylov, trunc="rho")
    _compare(psi, E, E0, info)
    assert psi.oc == 0


def test_hubbard_u1xu1_half_filling(dmrgb, ctx):
    L = 8
    hq = [(0, 0), (1, 1), (1, -1), (2, 0)]
    start = om.hubbard_half_filling_mps(L)
    mpo = dmrgb.makeMPO(dmrgb.hubbardMPO, 4, L).with_qn(dmrgb.HUBBARD_QN)
    psi = dmrgb.MPS([np.array(a) for a in start], oc=0)
    E = dmrgb.dmrg(psi, mpo, m=64, sweeps=6, cutoff=1e-10, ctx=ctx)
    ompo = om.to_qmpo(om.make_mpo([om.hubbard_bulk()] * L, 4), [hq] * L)
    E0, info = od.dmrg(om.to_qmps(start, [hq] * L), ompo, m=64, sweeps=6, cutoff=1e-10,
                       trunc="rho")
    _compare(psi, E, E0, info)
