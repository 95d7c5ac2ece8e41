"""Device measurements against the oracle: ``expect`` and ``correlationmatrix``.

``expect`` (``lib/MPO_MPS/expect.jl:19-56``): raw <psi|H|psi> on a dense random MPS, and on the
block-form (U(1)) state a DMRG run leaves, compared with the oracle on the same tensors (relative
1e-12); linearity in the MPO (H with J = 1/2 gives half). ``correlationmatrix``
(``lib/MPO_MPS/correlationmatrix.jl:21-56``) against the oracle's centre-moving restatement
(absolute 1e-12 on random states, 1e-10 after DMRG): dense spin operators, U(1) spin operators
with charge (S+ S-), the Hubbard U(1)xU(1) creation / annihilation pairs with the Jordan-Wigner
trail, an unnormalised non-canonical input (gauge and norm invariance), and the charge check.
Edge cases: a charge-violating pair (S+ S+ under U(1)) gives exact zeros, a two-site chain, and an
MPO with other physical charges is refused by ``expect``.
"""
import numpy as np
import pytest

from oracle import measure as om, models as mo

pytestmark = pytest.mark.gpu


def _dense(psi):
    return [np.array(psi[i]) for i in range(len(psi))]


def test_expect_dense_random(dmrgb, ctx):
    L = 12
    psi = dmrgb.randMPS(2, L, 8, seed=4, oc=3)
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    ref = om.expect_value(_dense(psi), mo.make_mpo([mo.heisenberg_bulk()] * L, 2))
    val = dmrgb.expect(psi, mpo, ctx=ctx)
    assert abs(val - ref) <= 1e-12 * abs(ref)


def test_expect_u1_after_dmrg_and_linearity(dmrgb, ctx):
    L = 16
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    E = dmrgb.dmrg(psi, mpo, m=64, sweeps=4, cutoff=1e-12, ctx=ctx)
    val = dmrgb.expect(psi, mpo, ctx=ctx)
    ref = om.expect_value(_dense(psi), mo.make_mpo([mo.heisenberg_bulk()] * L, 2))
    assert abs(val - ref) <= 1e-12 * abs(ref)
    assert abs(val - E) <= 1e-8 * abs(E)
    half = dmrgb.makeMPO(lambda i=None: dmrgb.heisenbergMPO(i, J=0.5), 2, L).with_qn(dmrgb.SPIN_QN)
    assert abs(dmrgb.expect(psi, half, ctx=ctx) - 0.5 * val) <= 1e-12 * abs(val)


@pytest.mark.parametrize("pair", ["zz", "pm", "xz"])
def test_correlation_dense_random(dmrgb, ctx, pair):
    L = 10
    psi = dmrgb.randMPS(2, L, 6, seed=7, oc=0)
    Sp, Sm, Sz, _, Sx, _, _ = mo.spin_ops()
    Cc, Ca = {"zz": (Sz, Sz), "pm": (Sp, Sm), "xz": (Sx, Sz)}[pair]
    rho = dmrgb.correlationmatrix(psi, Cc, Ca, ctx=ctx)
    ref = om.correlationmatrix(_dense(psi), psi.oc, Cc, Ca)
    assert np.max(np.abs(rho - ref)) <= 1e-12
    assert psi.oc == 0


def test_correlation_unnormalised_non_canonical(dmrgb, ctx):
    L = 9
    rng = np.random.default_rng(21)
    T = mo.random_mps(L, 2, 5, rng)
    T[4] = 3.0 * T[4]
    psi = dmrgb.MPS(T, oc=0)
    Sp, Sm, Sz, _, _, _, _ = mo.spin_ops()
    rho = dmrgb.correlationmatrix(psi, Sp, Sm, ctx=ctx)
    ref = om.correlationmatrix(mo.right_canonicalize(T), 0, Sp, Sm)
    assert np.max(np.abs(rho - ref)) <= 1e-12


def test_correlation_u1_after_dmrg(dmrgb, ctx):
    L = 16
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dmrgb.dmrg(psi, mpo, m=64, sweeps=4, cutoff=1e-12, ctx=ctx)
    Sp, Sm, Sz, _, _, _, _ = mo.spin_ops()
    dense = _dense(psi)
    for Cc, Ca in [(Sz, Sz), (Sp, Sm), (Sm, Sp)]:
        rho = dmrgb.correlationmatrix(psi, Cc, Ca, ctx=ctx)
        ref = om.correlationmatrix(dense, psi.oc, Cc, Ca)
        assert np.max(np.abs(rho - ref)) <= 1e-10
    # total Sz = 0: every row of <Sz_i Sz_j> sums to zero
    rho = dmrgb.correlationmatrix(psi, Sz, Sz, ctx=ctx)
    assert np.max(np.abs(rho.sum(axis=1))) <= 1e-9


def test_correlation_hubbard_trail(dmrgb, ctx):
    L = 8
    start = mo.hubbard_half_filling_mps(L)
    mpo = dmrgb.makeMPO(dmrgb.hubbardMPO, 4, L).with_qn(dmrgb.HUBBARD_QN)
    psi = dmrgb.MPS([np.array(a) for a in start], oc=0)
    dmrgb.dmrg(psi, mpo, m=64, sweeps=4, cutoff=1e-10, ctx=ctx)
    Cup, Cdn, F, Nup, _, _, _, _ = mo.fermion_ops()
    dense = _dense(psi)
    for Cc, Ca in [(Cup.T, Cup), (Cdn.T, Cdn)]:
        rho = dmrgb.correlationmatrix(psi, Cc, Ca, trail=F, ctx=ctx)
        ref = om.correlationmatrix(dense, psi.oc, Cc, Ca, trail=F)
        assert np.max(np.abs(rho - ref)) <= 1e-10
    rho = dmrgb.correlationmatrix(psi, Cup.T, Cup, trail=F, ctx=ctx)
    assert abs(np.trace(rho) - L / 2) <= 1e-9       # N_up = L/2 at half filling, Sz = 0


def test_correlation_rejects_operator_without_fixed_charge(dmrgb, ctx):
    L = 8
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dmrgb.dmrg(psi, mpo, m=16, sweeps=1, ctx=ctx)
    _, _, Sz, _, Sx, _, _ = mo.spin_ops()
    with pytest.raises(dmrgb.DmrgError):
        dmrgb.correlationmatrix(psi, Sx, Sz, ctx=ctx)


def test_correlation_charge_violating_pair_is_zero_and_two_site_chain(dmrgb, ctx):
    L = 10
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dmrgb.dmrg(psi, mpo, m=16, sweeps=2, cutoff=1e-12, ctx=ctx)
    Sp, Sm, Sz, _, _, _, _ = mo.spin_ops()
    assert np.array_equal(dmrgb.correlationmatrix(psi, Sp, Sp, ctx=ctx), np.zeros((L, L)))
    two = dmrgb.randMPS(2, 2, 2, seed=3, oc=0)
    rho = dmrgb.correlationmatrix(two, Sp, Sm, ctx=ctx)
    ref = om.correlationmatrix(_dense(two), two.oc, Sp, Sm)
    assert np.max(np.abs(rho - ref)) <= 1e-13


def test_expect_rejects_mpo_with_other_physical_charges(dmrgb, ctx):
    L = 8
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dmrgb.dmrg(psi, mpo, m=16, sweeps=1, ctx=ctx)
    flipped = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn([[(-1,), (1,)]] * L)
    with pytest.raises(dmrgb.DmrgError):
        dmrgb.expect(psi, flipped, ctx=ctx)


def test_expect_of_an_operator_product(dmrgb, ctx):
    """expect(psi, H, H) = <psi|H^2|psi> against the full state vector; after DMRG the energy
    variance <H^2> - <H>^2 is small and not negative."""
    from oracle import ed
    L = 8
    psi = dmrgb.randMPS(2, L, 8, seed=12, oc=0)
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    v = om.mps_vector([np.array(psi[i]) for i in range(L)])
    Hm = ed.full_h(mpo.W).T
    ref = float(v @ (Hm @ (Hm @ v)))
    assert abs(dmrgb.expect(psi, mpo, mpo, ctx=ctx) - ref) <= 1e-12 * abs(ref)
    qmpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 16).with_qn(dmrgb.SPIN_QN)
    gs = dmrgb.neelMPS(16)
    E = dmrgb.dmrg(gs, qmpo, m=64, sweeps=4, cutoff=1e-12, ctx=ctx)
    var = dmrgb.expect(gs, qmpo, qmpo, ctx=ctx) - dmrgb.expect(gs, qmpo, ctx=ctx) ** 2
    assert -1e-9 <= var <= 1e-6, (E, var)


# ------------------------------------------------------------------ correlation (n-point)

def _corr_cases():
    Sp, Sm, Sz, _, Sx, _, _ = mo.spin_ops()
    F = np.diag([1.0, -1.0])
    return [((Sz,), None), ((Sp, Sm), None), ((Sz, Sx), F), (([Sp, Sz], Sm), None),
            ((Sz, [Sm, Sp]), F), ((Sz, Sz, Sz), None), ((Sp, Sz, Sm), F)]


@pytest.mark.parametrize("case", range(7))
def test_correlation_n_dense_random(dmrgb, ctx, case):
    """``correlation`` (``lib/MPO_MPS/correlation.jl:73-237``) on a dense random unnormalised
    state against the full-vector definition: one, two and three operators, trails, multi-site
    operators in first and second place (relative 1e-12 of the largest entry)."""
    L, d = 8, 2
    psi = dmrgb.randMPS(2, L, 6, seed=12, oc=2)
    ops, tr = _corr_cases()[case]
    omega = dmrgb.correlation(psi, *ops, trail=() if tr is None else tr, ctx=ctx)
    ref = om.ed_correlation_n(om.mps_vector(_dense(psi)), L, d, ops, trail=tr)
    assert omega.shape == ref.shape
    assert np.max(np.abs(omega - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert psi.oc == 2


def test_correlation_n_u1_equals_reference_loop_and_correlation_matrix(dmrgb, ctx):
    """On the U(1) state a DMRG run leaves, two operators: the device equals the oracle's
    restatement of the reference's loop, and (normalised state) the correlation matrix, as the
    reference's own test checks (``test/MPmeas_test.jl:335-341``); S+ S+ changes the charge by 2
    and gives exact zeros."""
    L = 12
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dmrgb.dmrg(psi, mpo, m=48, sweeps=4, cutoff=1e-12, ctx=ctx)
    Sp, Sm, Sz, _, _, _, _ = mo.spin_ops()
    dense = _dense(psi)
    for ops in [(Sp, Sm), (Sz, Sz), (Sm, Sp)]:
        omega = dmrgb.correlation(psi, *ops, ctx=ctx)
        assert np.max(np.abs(omega - om.correlation(dense, ops))) <= 1e-10
    nrm = float(np.sum(om.mps_vector(dense) ** 2))
    M = dmrgb.correlation(psi, Sp, Sm, ctx=ctx) / nrm
    assert np.max(np.abs(M - dmrgb.correlationmatrix(psi, Sp, Sm, ctx=ctx))) <= 1e-10
    assert np.array_equal(dmrgb.correlation(psi, Sp, Sp, ctx=ctx), np.zeros((L, L)))


def test_correlation_n_hubbard_trail_and_site_lists(dmrgb, ctx):
    """Hubbard U(1)xU(1) after DMRG (d = 4): the fermion pair with its Jordan-Wigner trail
    against the full-vector definition, with the default sites and with explicit 1-based site
    lists (entries indexed by their place in each list)."""
    L, d = 6, 4
    start = mo.hubbard_half_filling_mps(L)
    mpo = dmrgb.makeMPO(dmrgb.hubbardMPO, d, L).with_qn(dmrgb.HUBBARD_QN)
    psi = dmrgb.MPS([np.array(a) for a in start], oc=0)
    dmrgb.dmrg(psi, mpo, m=64, sweeps=4, cutoff=1e-10, ctx=ctx)
    Cup, Cdn, F, Nup, _, _, _, _ = mo.fermion_ops()
    v = om.mps_vector(_dense(psi))
    ops = (Cup.T, Cup)
    omega = dmrgb.correlation(psi, *ops, trail=F, ctx=ctx)
    ref = om.ed_correlation_n(v, L, d, ops, trail=F)
    assert np.max(np.abs(omega - ref)) <= 1e-10
    sites = ([2, 4, 5], [1, 3, 6])
    omega = dmrgb.correlation(psi, Cdn.T, Cdn, Nup, sites=(sites[0], sites[1], [2, 6]),
                              trail=(F, F, np.eye(d)), ctx=ctx)
    ref = om.ed_correlation_n(v, L, d, (Cdn.T, Cdn, Nup),
                              sites=[[s - 1 for s in sites[0]], [s - 1 for s in sites[1]], [1, 5]],
                              trail=(F, F, np.eye(d)))
    assert omega.shape == (3, 3, 2)
    assert np.max(np.abs(omega - ref)) <= 1e-10
