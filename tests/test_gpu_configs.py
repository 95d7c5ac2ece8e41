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


# ---------------------------------------------------------------- capped benchmark configurations
# The oracle's converged invariants (tests/golden/config_parity.json, written by
# tests/golden/make_config_fixtures.py) on the L=100 Heisenberg U(1) ramp capped at maxm 128, the
# L=32 Hubbard U(1)xU(1) chain at maxm 256 and the 4x16 cylinder at maxm 256. The device runs the
# same deterministic inputs with the same schedule, Krylov dimension and goal; both stop at
# convergence, where the energy agrees to 1e-10 relative and the last sweep's largest truncation
# error and centre entropy to 1e-8. (Intermediate energies of a still-moving trajectory are not
# compared: near-ties of density-matrix weights at the cut, resolved only to ~1e-15 absolute, let
# two correct runs keep different states there; they reach the same fixed point.)

import json
from pathlib import Path

FIXTURES = json.loads((Path(__file__).resolve().parent / "golden" / "config_parity.json").read_text())


def _config_inputs(dmrgb, case):
    L = case["L"]
    if case["model"] == "heisenberg":
        return dmrgb.neelMPS(L), dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    if case["model"] == "hubbard":
        mpo = dmrgb.makeMPO(lambda i: dmrgb.hubbardMPO(t=case["t"], mu=case["mu"], HubU=case["U"]),
                            4, L).with_qn(dmrgb.HUBBARD_QN)
        return dmrgb.MPS([np.array(a) for a in om.hubbard_half_filling_mps(L)], oc=0), mpo
    mpo = dmrgb.heisenbergCylinderMPO(case["W"], case["Lx"]).with_qn(dmrgb.SPIN_QN)
    return dmrgb.neelMPS(L), mpo


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_capped_config_matches_oracle(dmrgb, ctx, name):
    fx = FIXTURES[name]
    case = fx["case"]
    psi, mpo = _config_inputs(dmrgb, case)
    E = dmrgb.dmrg(psi, mpo, m=case["schedule"], cutoff=case["cutoff"], krylov=case["krylov"],
                   degen_rtol=case["degen_rtol"], goal=case["goal"], ctx=ctx)
    assert len(fx["sweeps"]) < len(case["schedule"])          # the oracle converged
    assert psi.sweep_stats[-1]["converged"] == 1              # and so did the device
    d, o = psi.sweep_stats[-1], fx["sweeps"][-1]
    assert abs(E - fx["energy"]) <= 1e-10 * abs(fx["energy"])
    assert abs(d["max_truncerr"] - o["maxtrunc"]) <= 1e-8
    assert abs(d["entropy"] - o["entropy"]) <= 1e-8


def test_density_matrix_blocks_above_the_tridiagonal_limit(dmrgb, ctx):
    """Dense chain whose centre density matrix (m=64, d=2: side 128) is larger than the small
    tridiagonal kernel's limit (112), so the mid-size kernels run inside the sweep. The cutoff
    (1e-10) keeps the cut away from eigenvalues at the rounding level (~1e-16): at such a cut a
    noise-level state may or may not be kept, and a kept one enlarges the variational space of
    the following steps."""
    L = 12
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, 64, seed=7)
    ref = [a.copy() for a in psi.tensors]
    E = dmrgb.dmrg(psi, mpo, m=100, sweeps=3, cutoff=1e-10, krylov=2, ctx=ctx)
    E0, info = od.dmrg(ref, om.make_mpo([om.heisenberg_bulk()] * L, 2), m=100, sweeps=3,
                       cutoff=1e-10, krylov=2, trunc="rho")
    assert max(s["eig_max_n"] for s in psi.sweep_stats) > 112
    _compare(psi, E, E0, info)
