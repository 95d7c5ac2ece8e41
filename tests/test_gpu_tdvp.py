"""Device TDVP (``dmrg_tdvp``: ``tdvp_twosite`` and ``tdvp`` with a real prefactor,
algs/time.jl:182-363) against the oracle's restatement (oracle/tdvp.py).

Both start from the same state; each call's En (the lowest eigenvalue of the last Krylov
tridiagonal), largest kept dimension and truncation error are compared, and the final states
through their energy <psi|H|psi>. FP64 throughout: energies to 1e-9 relative.
"""
import numpy as np
import pytest

from oracle import dmrg as od, ed, models as om, tdvp as ot

pytestmark = pytest.mark.gpu

SPIN = [(1,), (-1,)]
HQ = [(0, 0), (1, 1), (1, -1), (2, 0)]


def _run_device(dmrgb, ctx, psi, mpo, calls, twosite, **kw):
    fn = dmrgb.tdvp_twosite if twosite else dmrgb.tdvp
    out = []
    for _ in range(calls):
        En = fn(psi, mpo, ctx=ctx, **kw)
        st = psi.sweep_stats[-1]
        out.append((En, st["max_truncerr"], st["biggest_m"]))
    return out


def _compare(dev, ref, rtol=1e-9):
    assert len(dev) == len(ref)
    for (e, t, m), (e0, t0, m0) in zip(dev, ref):
        assert abs(e - e0) <= rtol * abs(e0)
        assert m == m0
        assert abs(t - t0) <= 1e-8


@pytest.mark.parametrize("qn", [True, False])
def test_tdvp_twosite_matches_oracle(dmrgb, ctx, qn):
    L = 10
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    if qn:
        mpo = mpo.with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    dev = _run_device(dmrgb, ctx, psi, mpo, 4, True, m=32, cutoff=1e-12, prefactor=-0.5)
    start = om.neel_mps(L)
    q = om.mps_bond_labels(start, [SPIN] * L)
    phys = [SPIN] * L
    if not qn:
        q = [[(0,)] * len(b) for b in q]
        phys = [[(0,), (0,)]] * L
    ompo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    recs, S = ot.tdvp(start, ompo, phys, q, calls=4, prefactor=-0.5, m=32, cutoff=1e-12,
                      twosite=True)
    _compare(dev, recs)
    e_ref = od.expect(S.psi, ompo)
    assert abs(dmrgb.expect(psi, mpo, ctx=ctx) - e_ref) <= 1e-9 * abs(e_ref)


def test_tdvp_twosite_hubbard_u1xu1_matches_oracle(dmrgb, ctx):
    L = 8
    mpo = dmrgb.makeMPO(dmrgb.hubbardMPO, 4, L).with_qn(dmrgb.HUBBARD_QN)
    start = om.hubbard_half_filling_mps(L)
    psi = dmrgb.MPS([np.array(a) for a in start], oc=0)
    dev = _run_device(dmrgb, ctx, psi, mpo, 3, True, m=24, cutoff=1e-10, prefactor=-0.4, r=4)
    ompo = om.make_mpo([om.hubbard_bulk()] * L, 4)
    recs, _ = ot.tdvp(start, ompo, [HQ] * L, om.mps_bond_labels(start, [HQ] * L), calls=3,
                      prefactor=-0.4, m=24, cutoff=1e-10, r=4, twosite=True)
    _compare(dev, recs, rtol=1e-8)


def test_tdvp_single_site_matches_oracle(dmrgb, ctx):
    """tdvp: the site, then the bond matrix through the zero-site Heff (OC_update)."""
    L = 10
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, 8, seed=3)
    start = [a.copy() for a in psi.tensors]
    dev = _run_device(dmrgb, ctx, psi, mpo, 4, False, m=32, cutoff=1e-12, prefactor=-1.0)
    ompo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    labels = [[(0,)] * A.shape[0] for A in start] + [[(0,)]]
    recs, S = ot.tdvp(start, ompo, [[(0,), (0,)]] * L, labels, calls=4, prefactor=-1.0, m=32,
                      cutoff=1e-12, twosite=False)
    _compare(dev, recs)
    e_ref = od.expect(S.psi, ompo)
    assert abs(dmrgb.expect(psi, mpo, ctx=ctx) - e_ref) <= 1e-9 * abs(e_ref)


def test_tdvp_imaginary_time_reaches_the_ground_state(dmrgb, ctx):
    L = 10
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    psi = dmrgb.neelMPS(L)
    for _ in range(30):
        En = dmrgb.tdvp_twosite(psi, mpo, m=32, cutoff=1e-12, prefactor=-2.0, ctx=ctx)
    e0 = ed.sparse_ground_energy(om.make_mpo([om.heisenberg_bulk()] * L, 2))
    assert abs(En - e0) < 1e-9
    assert abs(dmrgb.expect(psi, mpo, ctx=ctx) - e0) < 1e-9


def test_tdvp_rejects_a_complex_prefactor(dmrgb, ctx):
    L = 6
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    with pytest.raises(ValueError, match="complex"):
        dmrgb.tdvp_twosite(dmrgb.neelMPS(L), mpo, prefactor=-0.01j, ctx=ctx)
