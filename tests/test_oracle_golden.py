"""The CPU oracle against the reference's own known answers (tests/golden/reference_pins.json).

These pin the oracle before it is used as the checker of the device engine: ED of the MPO,
two-site DMRG energies (dense and U(1)), the Hubbard known answer, the environment identities of
test/MPmeas_test.jl:150-206, and the agreement of the SVD and density-matrix truncation forms.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import dmrg as od, ed, models as om, qtensor as oq

PINS = json.loads((Path(__file__).parent / "golden" / "reference_pins.json").read_text())
SPIN = [(1,), (-1,)]


def heis(L):
    return om.make_mpo([om.heisenberg_bulk()] * L, 2)


def test_ed_known_answer():
    p = PINS["heisenberg_L10_ed"]
    assert abs(ed.ground_energy(heis(10)) - p["value"]) < p["tol"]
    assert abs(ed.sparse_ground_energy(heis(10)) - p["value"]) < 1e-10


@pytest.mark.parametrize("L", [3, 5, 7, 8, 9, 10])
def test_docstring_energies(L):
    p = PINS["heisenberg_docstring_dmrg"]
    psi = om.right_canonicalize(om.random_mps(L, 2, 8, np.random.default_rng(L)))
    E, _ = od.dmrg(psi, heis(L), m=100, sweeps=6, cutoff=1e-9)
    assert abs(E - p["values"][str(L)]) < p["tol"] + 1e-8
    assert abs(E - ed.ground_energy(heis(L))) < 2e-8


def test_dense_and_qn_agree_and_reach_ed():
    L = 12
    mpo = heis(L)
    dense = om.right_canonicalize(om.random_mps(L, 2, 6, np.random.default_rng(0)))
    Ed, _ = od.dmrg(dense, mpo, m=45, sweeps=6, cutoff=1e-12)
    q = om.to_qmps(om.neel_mps(L), [SPIN] * L)
    Eq, info = od.dmrg(q, om.to_qmpo(mpo, [SPIN] * L), m=45, sweeps=8, cutoff=1e-12)
    assert abs(Ed - Eq) < PINS["dense_vs_qn_agreement"]["tol"]
    assert abs(Eq - ed.sparse_ground_energy(mpo)) < 1e-8
    assert info["oc"] == 0


def test_hubbard_known_answer():
    p = PINS["hubbard_L10_qn_dmrg"]
    L = 10
    hq = [[(0, 0), (1, 1), (1, -1), (2, 0)]] * L
    psi = om.to_qmps(om.hubbard_half_filling_mps(L), hq)
    mpo = om.to_qmpo(om.make_mpo([om.hubbard_bulk()] * L, 4), hq)
    E, _ = od.dmrg(psi, mpo, m=45, sweeps=20, cutoff=1e-9)
    assert abs(E - p["value"]) < p["tol"]


def test_environment_identities():
    """makeEnv + single-site Heff at oc equals <psi|H|psi>; Lupdate/Rupdate reproduce the next
    environments (test/MPmeas_test.jl:150-206)."""
    L, oc = 10, 6
    mpo = heis(L)
    rng = np.random.default_rng(3)
    psi = om.right_canonicalize(om.random_mps(L, 2, 8, rng))
    # move the centre to oc with exact QR steps
    for i in range(oc):
        a, d, b = psi[i].shape
        Q, R = np.linalg.qr(psi[i].reshape(a * d, b))
        psi[i] = Q.reshape(a, d, Q.shape[1])
        psi[i + 1] = np.tensordot(R, psi[i + 1], axes=(1, 0))
    Lenv, Renv = od.make_env(psi, mpo, oc)
    e1 = od.startval(Lenv[oc], Renv[oc], psi[oc], mpo[oc]) / od.overlap(psi, psi)
    assert abs(e1 - od.expect(psi, mpo)) < 1e-12
    L5 = od.Lupdate(Lenv[4], psi[4], psi[4], mpo[4])
    assert np.max(np.abs(L5 - Lenv[5])) < 1e-12
    R8 = od.Rupdate(Renv[9], psi[9], psi[9], mpo[9])
    assert np.max(np.abs(R8 - Renv[8])) < 1e-12


def test_svd_and_density_matrix_forms_agree():
    L = 12
    mpo = heis(L)
    base = om.right_canonicalize(om.random_mps(L, 2, 8, np.random.default_rng(1)))
    E1, i1 = od.dmrg([a.copy() for a in base], mpo, m=20, sweeps=3, cutoff=1e-10, trunc="svd")
    E2, i2 = od.dmrg([a.copy() for a in base], mpo, m=20, sweeps=3, cutoff=1e-10, trunc="rho")
    assert abs(E1 - E2) < 1e-10 * abs(E1)
    assert abs(i1["sweeps"][-1]["entropy"] - i2["sweeps"][-1]["entropy"]) < 1e-8
    assert abs(i1["sweeps"][-1]["maxtrunc"] - i2["sweeps"][-1]["maxtrunc"]) < 1e-8


def test_truncation_rule():
    w = [np.array([0.5, 0.2, 1e-11]), np.array([0.3 - 1e-11, 1e-13])]
    kept, terr = oq.select_kept(w, maxm=0, minm=2, cutoff=1e-10)
    assert kept == [2, 1] and abs(terr - 1.01e-11) < 1e-24
    kept, _ = oq.select_kept(w, maxm=2, minm=2, cutoff=0.0)
    assert kept == [1, 1]
    kept, _ = oq.select_kept([np.array([1.0, 0.0, 0.0])], maxm=0, minm=2, cutoff=1e-12)
    assert kept == [2]
    # a cut inside a degenerate pair drops the pair when degen_rtol > 0
    kept, _ = oq.select_kept([np.array([0.6, 0.2, 0.2])], maxm=2, minm=1, cutoff=0, degen_rtol=1e-6)
    assert kept == [1]


def test_oracle_goal_semantics():
    """goal = 0 runs every sweep; a large goal stops after the first; the energy test compares the
    first sweep with startval (algs/optimizeMPS.jl:365-371, algs/DMRG.jl:627-637)."""
    L = 6
    mpo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    rng = np.random.default_rng(2)
    start = om.right_canonicalize(om.random_mps(L, 2, 4, rng))
    _, info = od.dmrg([a.copy() for a in start], mpo, m=16, sweeps=4, trunc="rho")
    assert len(info["sweeps"]) == 4
    _, info = od.dmrg([a.copy() for a in start], mpo, m=16, sweeps=4, trunc="rho", goal=1e3)
    assert len(info["sweeps"]) == 1
    e0 = info["e0"]
    assert e0 == pytest.approx(od.expect([a.copy() for a in start], mpo), rel=1e-12)


# ------------------------------------------------------------------ the 3S method (dmrg3S)

def test_3s_oracle_reaches_ed_with_and_without_charges():
    """test/dmrg_test.jl:82-85 (method "3S"): the dense and the charge-labelled runs agree (the
    reference allows 1e-4); both reach ED here."""
    from oracle import dmrg3s as o3
    L = 10
    mpo = heis(L)
    start = om.neel_mps(L)
    q = om.mps_bond_labels(start, [SPIN] * L)
    E, recs, _ = o3.dmrg3s(start, mpo, [SPIN] * L, q, m=45, sweeps=40, cutoff=1e-12)
    zero = [[(0,)] * len(b) for b in q]
    Ed, _, _ = o3.dmrg3s(start, mpo, [[(0,), (0,)]] * L, zero, m=45, sweeps=40, cutoff=1e-12)
    e0 = ed.sparse_ground_energy(mpo)
    assert abs(E - e0) < 1e-9
    assert abs(Ed - e0) < 1e-9
    assert all(r["biggestm"] <= 45 for r in recs)
    assert recs[-1]["noise"] < recs[0]["noise"]      # alpha decays once the energy settles


def test_3s_oracle_hubbard_known_answer():
    from oracle import dmrg3s as o3
    p = PINS["hubbard_L10_qn_dmrg"]
    L = 10
    hq = [(0, 0), (1, 1), (1, -1), (2, 0)]
    start = om.hubbard_half_filling_mps(L)
    E, _, _ = o3.dmrg3s(start, om.make_mpo([om.hubbard_bulk()] * L, 4), [hq] * L,
                        om.mps_bond_labels(start, [hq] * L), m=45, sweeps=20, cutoff=1e-9)
    assert abs(E - p["value"]) < p["tol"]


def test_alpha_update_rules():
    """alpha_update (algs/DMRG.jl:289-302): shrink by (1 - dalpha) when the energy did not rise
    and one of the three conditions holds, else grow; clamped to [1e-42, 1]; IEEE division."""
    from oracle.dmrg3s import alpha_update
    # truncation below the cutoff: shrink
    assert alpha_update(0.5, 1e-14, 1e-12, -1.0, -1.1, 0.3, 0.01) == pytest.approx(0.495)
    # energy rose: grow, whatever the truncation
    assert alpha_update(0.5, 0.0, 1e-12, -1.1, -1.0, 0.3, 0.01) == pytest.approx(0.505)
    # large truncation, energy moving: site condition |trunc E / (E_last/E - 1)| vs noise_goal
    assert alpha_update(0.5, 1e-3, 1e-12, -1.0, -1.01, 0.3, 0.01) == pytest.approx(0.505)
    assert alpha_update(0.5, 1e-2, 1e-12, -1.0, -1.01, 0.3, 0.01) == pytest.approx(0.495)
    # clamps
    assert alpha_update(1.0, 1.0, 0.0, -1.1, -1.0, 0.3, 0.01) == 1.0
    assert alpha_update(1e-42, 0.0, 1e-12, -1.0, -1.0, 0.3, 0.5) == 1e-42
    # equal energies: the site condition is 0/0 (NaN, false) but err_est holds: shrink
    assert alpha_update(0.5, 0.0, 0.0, -2.0, -2.0, 0.3, 0.1) == pytest.approx(0.45)


# ------------------------------------------------------------------ TDVP (real prefactor)

def test_krylov_exp_matches_the_matrix_exponential():
    """krylovTimeEvol (algs/time.jl:182-203) with a full Krylov space is exp(tau H) x / |x|."""
    import scipy.linalg
    from oracle.tdvp import krylov_exp
    rng = np.random.default_rng(4)
    H = rng.standard_normal((6, 6))
    H = H + H.T
    x = rng.standard_normal(6)
    for tau in (-0.3, 0.0, 0.2):
        y, En = krylov_exp(lambda v: H @ v, x, 6, tau)
        ref = scipy.linalg.expm(tau * H) @ (x / np.linalg.norm(x))
        assert np.max(np.abs(y - ref)) < 1e-10
        assert abs(En - np.linalg.eigvalsh(H)[0]) < 1e-10


def test_tdvp_oracle_imaginary_time_reaches_ed():
    """tdvp_twosite with a negative real prefactor projects onto the ground state; the single-site
    form keeps the bond dimensions of its start."""
    from oracle import tdvp as ot
    L = 10
    mpo = heis(L)
    start = om.neel_mps(L)
    recs, S = ot.tdvp(start, mpo, [SPIN] * L, om.mps_bond_labels(start, [SPIN] * L), calls=30,
                      prefactor=-2.0, m=32, cutoff=1e-12, r=2, twosite=True)
    e0 = ed.sparse_ground_energy(mpo)
    assert abs(recs[-1][0] - e0) < 1e-9
    assert abs(od.expect(S.psi, mpo) - e0) < 1e-9
    psi0 = om.right_canonicalize(om.random_mps(L, 2, 8, np.random.default_rng(3)))
    labels = [[(0,)] * A.shape[0] for A in psi0] + [[(0,)]]
    recs1, S1 = ot.tdvp(psi0, mpo, [[(0,), (0,)]] * L, labels, calls=20, prefactor=-2.0, m=32,
                        cutoff=1e-12, twosite=False)
    assert all(r[2] <= 8 for r in recs1)
    assert e0 - 1e-12 < od.expect(S1.psi, mpo) < e0 + 1e-3
