"""The measurement oracle (``expect``, ``correlationmatrix``) pinned against full state vectors.

``expect_value`` must equal <v|H|v> from the full Hamiltonian of the MPO, and the Neel state's known
value -(L-1)/4 for the Heisenberg chain (J = 1) in block form. ``correlationmatrix`` (the
reference's centre-moving algorithm, ``lib/MPO_MPS/correlationmatrix.jl:21-56``) must equal the full
operator strings <v|(Cc F)_i F..F Ca_j|v> on random normalised states: spin operators on a d=2
chain and the fermion creation / annihilation pair with its Jordan-Wigner trail on a d=4 chain.
"""
import numpy as np

from oracle import ed, measure as om, models as mo


def _mps_from_vector(v, L, d):
    """Exact MPS of a state vector by left-to-right SVDs; centre on the last site."""
    out = []
    rest = v.reshape(1, -1)
    for _ in range(L - 1):
        a = rest.shape[0]
        M = rest.reshape(a * d, -1)
        U, S, Vt = np.linalg.svd(M, full_matrices=False)
        k = int(np.sum(S > 1e-14 * S[0]))
        out.append(U[:, :k].reshape(a, d, k))
        rest = S[:k, None] * Vt[:k]
    out.append(rest.reshape(rest.shape[0], d, 1))
    return out


def test_expect_value_matches_full_hamiltonian():
    L, d = 6, 2
    rng = np.random.default_rng(3)
    psi = mo.random_mps(L, d, 4, rng)
    mpo = mo.make_mpo([mo.heisenberg_bulk()] * L, d)
    v = om.mps_vector(psi)
    H = ed.full_h(mpo)
    assert abs(om.expect_value(psi, mpo) - v @ H @ v) <= 1e-12 * abs(v @ H @ v)


def test_expect_value_neel_known_answer_block_form():
    L = 10
    hq = [(1,), (-1,)]
    mpo = mo.to_qmpo(mo.make_mpo([mo.heisenberg_bulk()] * L, 2), [hq] * L)
    psi = mo.to_qmps(mo.neel_mps(L), [hq] * L)
    assert abs(om.expect_value(psi, mpo) + (L - 1) / 4) <= 1e-14


def test_correlationmatrix_spin_matches_full_vector():
    L, d = 7, 2
    rng = np.random.default_rng(11)
    v = rng.standard_normal(d ** L)
    v /= np.linalg.norm(v)
    psi = _mps_from_vector(v, L, d)
    Sp, Sm, Sz, _, Sx, _, _ = mo.spin_ops()
    for Cc, Ca in [(Sz, Sz), (Sp, Sm), (Sx, Sz)]:
        rho = om.correlationmatrix(psi, L - 1, Cc, Ca)
        ref = om.ed_correlation(v, L, Cc, Ca)
        assert np.max(np.abs(rho - ref)) <= 1e-12


def test_correlationmatrix_fermion_trail_matches_full_vector():
    L, d = 4, 4
    rng = np.random.default_rng(12)
    v = rng.standard_normal(d ** L)
    v /= np.linalg.norm(v)
    psi = _mps_from_vector(v, L, d)
    Cup, Cdn, F, Nup, _, _, _, _ = mo.fermion_ops()
    for Cc, Ca in [(Cup.T, Cup), (Cdn.T, Cdn)]:
        rho = om.correlationmatrix(psi, L - 1, Cc, Ca, trail=F)
        ref = om.ed_correlation(v, L, Cc, Ca, trail=F)
        assert np.max(np.abs(rho - ref)) <= 1e-12
    rho = om.correlationmatrix(psi, L - 1, Cup.T, Cup, trail=F)
    nup = om.ed_correlation(v, L, Nup, np.eye(d))
    assert np.max(np.abs(np.diag(rho) - np.diag(nup))) <= 1e-12


def _spin_cases():
    Sp, Sm, Sz, _, Sx, _, _ = mo.spin_ops()
    F = np.diag([1.0, -1.0])
    return Sp, Sm, Sz, Sx, F


def test_correlation_restatement_matches_definition_for_two_operators():
    """``correlation`` (the reference's loop, ``lib/MPO_MPS/correlation.jl:98-237``) equals the
    full-vector definition for one and two operators: single-site operators, a trail, and
    multi-site operators in either place (unnormalised random state)."""
    L, d = 6, 2
    rng = np.random.default_rng(3)
    psi = mo.random_mps(L, d, 4, rng)
    v = om.mps_vector(psi)
    Sp, Sm, Sz, Sx, F = _spin_cases()
    for ops, tr in [((Sz,), None), ((Sp, Sm), None), ((Sz, Sx), None), ((Sp, Sm), F),
                    (([Sp, Sz], Sm), None), ((Sz, [Sm, Sp]), F)]:
        lit = om.correlation(psi, ops, trail=tr)
        ref = om.ed_correlation_n(v, L, d, ops, trail=tr)
        assert lit.shape == ref.shape
        assert np.max(np.abs(lit - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_correlation_of_two_operators_is_the_correlation_matrix():
    """The reference's own check (``test/MPmeas_test.jl:335-341``): on a normalised state,
    correlation(psi, Sp, Sm) equals correlationmatrix(psi, Sp, Sm) entry by entry."""
    L, d = 7, 2
    rng = np.random.default_rng(11)
    v = rng.standard_normal(d ** L)
    v /= np.linalg.norm(v)
    psi = _mps_from_vector(v, L, d)
    Sp, Sm, _, _, _ = _spin_cases()
    M = om.correlation(psi, (Sp, Sm))
    assert np.max(np.abs(M - om.correlationmatrix(psi, L - 1, Sp, Sm))) <= 1e-12


def test_correlation_reference_loop_reuses_right_environments_for_three_operators():
    """With three operators the reference's loop rebuilds its right environments in place from
    the rightmost operator of each position combination; when operator 2's position resets, the
    environments right of that point still hold the previous combination's operators. Its values
    agree with the definition up to the first reset (operator 3 at its first position) and differ
    after it; the device computes the definition."""
    L, d = 6, 2
    rng = np.random.default_rng(5)
    psi = mo.random_mps(L, d, 4, rng)
    v = om.mps_vector(psi)
    Sp, Sm, Sz, _, _ = _spin_cases()
    lit = om.correlation(psi, (Sz, Sz, Sz))
    ref = om.ed_correlation_n(v, L, d, (Sz, Sz, Sz))
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(lit[:, :, 0] - ref[:, :, 0])) <= 1e-12 * scale
    assert np.max(np.abs(lit - ref)) > 1e-6 * scale
