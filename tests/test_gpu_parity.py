"""Device vs oracle parity for the hot-path contractions (through the C ABI).

Tolerances: the plain form is FP64 end to end, so single contractions must agree to 1e-12
relative (max-abs error / max-abs value); whole sweeps are compared on invariants (energy,
truncation error, centre-bond entropy), never on gauge-dependent tensors.
"""
import numpy as np
import pytest

from oracle import dmrg as od, models as om, qtensor as oq

pytestmark = pytest.mark.gpu

RTOL_CONTRACT = 1e-12


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _heis(pkg, L, qn):
    mpo = pkg.makeMPO(pkg.heisenbergMPO, 2, L)
    ompo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    if qn:
        mpo = mpo.with_qn(pkg.SPIN_QN)
    return mpo, ompo


def _qn_random_mps(L, m, seed):
    """A U(1) MPS (Sz=0 sector) with random blocks: built by DMRG-free QN-aware random filling."""
    rng = np.random.default_rng(seed)
    pq = [[(1,), (-1,)]] * L
    # bond charges: allowed partial magnetisations, m states spread over sectors
    bonds = [[(0,)]]
    for k in range(1, L + 1):
        lo, hi = max(-k, -(L - k)), min(k, L - k)
        qs = [(q,) for q in range(lo, hi + 1) if (q - lo) % 2 == 0]
        bonds.append(qs)
    dims = []
    for k, qs in enumerate(bonds):
        if k == 0 or k == L:
            dims.append([1] * len(qs))
        else:
            per = max(1, m // len(qs))
            dims.append([per] * len(qs))
    tens = []
    for i in range(L):
        ia = oq.Index(bonds[i], dims[i], +1)
        isx = oq.Index(pq[i], [1, 1], +1)
        ib = oq.Index(bonds[i + 1], dims[i + 1], -1)
        T = oq.QTensor([ia, isx, ib], {}, (0,))
        for ka in range(len(bonds[i])):
            for s in range(2):
                q = bonds[i][ka][0] + pq[i][s][0]
                if (q,) in bonds[i + 1]:
                    kb = bonds[i + 1].index((q,))
                    T.blocks[(ka, s, kb)] = rng.standard_normal((dims[i][ka], 1, dims[i + 1][kb]))
        tens.append(T)
    return tens, bonds, dims


def _labels_from(bonds, dims):
    return [[q for q, d in zip(qs, ds) for _ in range(d)] for qs, ds in zip(bonds, dims)]


@pytest.mark.parametrize("qn", [False, True])
def test_env_and_heff_match_oracle(dmrgb, ctx, qn):
    L, m = 8, 12
    mpo, ompo = _heis(dmrgb, L, qn)
    if qn:
        qt, bonds, dims = _qn_random_mps(L, m, seed=7)
        dense = [oq.to_dense(T) for T in qt]
        psi = dmrgb.MPS(dense, oc=3, bond_labels=_labels_from(bonds, dims))
        otens = qt
        ompo_t = om.to_qmpo(ompo, [[(1,), (-1,)]] * L)
    else:
        rng = np.random.default_rng(5)
        dimsb = [min(2 ** k, 2 ** (L - k), m) for k in range(L + 1)]
        dense = [rng.standard_normal((dimsb[i], 2, dimsb[i + 1])) for i in range(L)]
        psi = dmrgb.MPS(dense, oc=3)
        otens = dense
        ompo_t = ompo
    Lenv, Renv = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    OL, OR = od.make_env(otens, ompo_t, 3)
    for i in range(0, 4):
        assert _rel(Lenv[i], oq.to_dense(OL[i])) < RTOL_CONTRACT, f"Lenv[{i}]"
    for i in range(3, L):
        assert _rel(Renv[i], oq.to_dense(OR[i])) < RTOL_CONTRACT, f"Renv[{i}]"
    # Heff on a random two-site vector at (iL, iL+1) = (3, 4) needs Renv[4]: move the right env
    dev = Lenv.dev
    # two-site vector in the QN-allowed pattern of the oracle
    AA = od.contract(otens[3], 2, otens[4], 0)
    if qn:
        rng = np.random.default_rng(11)
        AA = oq.QTensor(AA.indices, {k: rng.standard_normal(v.shape) for k, v in AA.blocks.items()},
                        AA.flux)
    x = oq.to_dense(AA)
    # Renv[4] is valid (built for oc=3); Lenv[3] valid
    y = dev.heff(3, x)
    yo = oq.to_dense(od.heff_twosite(OL[3], OR[4], AA, ompo_t[3], ompo_t[4]))
    assert _rel(y, yo) < RTOL_CONTRACT
    # make2site order gives the same vector (reference's two Heff forms agree)
    y2 = oq.to_dense(od.make2site(OL[3], OR[4], otens[3], otens[4], ompo_t[3], ompo_t[4]))
    if not qn:
        assert _rel(dev.heff(3, oq.to_dense(od.contract(otens[3], 2, otens[4], 0))), y2) < RTOL_CONTRACT
    # Lupdate! / Rupdate! through the Env API agree with the oracle's next environments
    dmrgb.Lupdate(3, Lenv)
    assert _rel(Lenv[4], oq.to_dense(od.Lupdate(OL[3], otens[3], otens[3], ompo_t[3]))) < RTOL_CONTRACT
    dmrgb.Rupdate(3, Renv)
    assert _rel(Renv[2], oq.to_dense(od.Rupdate(OR[3], otens[3], otens[3], ompo_t[3]))) < RTOL_CONTRACT


@pytest.mark.parametrize("krylov", [2, 6])
def test_dense_dmrg_matches_oracle(dmrgb, ctx, krylov):
    L = 10
    mpo, ompo = _heis(dmrgb, L, False)
    psi = dmrgb.randMPS(2, L, 8, seed=1)
    ref = [a.copy() for a in psi.tensors]
    E = dmrgb.dmrg(psi, mpo, m=32, sweeps=4, cutoff=1e-12, krylov=krylov, ctx=ctx)
    E0, info = od.dmrg(ref, ompo, m=32, sweeps=4, cutoff=1e-12, krylov=krylov, trunc="rho")
    st = psi.sweep_stats[-1]
    o = info["sweeps"][-1]
    assert abs(E - E0) <= 1e-10 * abs(E0)
    assert abs(st["max_truncerr"] - o["maxtrunc"]) <= 1e-8
    assert abs(st["entropy"] - o["entropy"]) <= 1e-8
    assert abs(E - (-4.258035207282883)) < 1e-8
    assert psi.oc == 0


def test_qn_heisenberg_dmrg_matches_oracle_and_ed(dmrgb, ctx):
    L = 10
    mpo, ompo = _heis(dmrgb, L, True)
    psi = dmrgb.neelMPS(L)
    ref = om.to_qmps(om.neel_mps(L), [[(1,), (-1,)]] * L)
    E = dmrgb.dmrg(psi, mpo, m=45, sweeps=8, cutoff=1e-12, ctx=ctx)
    E0, info = od.dmrg(ref, om.to_qmpo(ompo, [[(1,), (-1,)]] * L), m=45, sweeps=8, cutoff=1e-12,
                       trunc="rho")
    assert abs(E - E0) <= 1e-10 * abs(E0)
    assert abs(psi.sweep_stats[-1]["entropy"] - info["sweeps"][-1]["entropy"]) <= 1e-8
    assert abs(E - (-4.258035207282883)) < 1e-8


@pytest.mark.parametrize("cvgE", [True, False])
def test_goal_stops_after_the_same_sweep_as_the_oracle(dmrgb, ctx, cvgE):
    """dmrgcvg's convergence test (algs/DMRG.jl:610-652): with goal > 0 the run stops after the
    first sweep whose energy (cvgE) or centre entropy moved by less than goal, the first sweep
    compared with the starting energy (startval) or entropy 0."""
    L = 10
    mpo, ompo = _heis(dmrgb, L, False)
    psi = dmrgb.randMPS(2, L, 8, seed=1)
    ref = [a.copy() for a in psi.tensors]
    E = dmrgb.dmrg(psi, mpo, m=32, sweeps=20, cutoff=1e-12, goal=1e-7, cvgE=cvgE, ctx=ctx)
    E0, info = od.dmrg(ref, ompo, m=32, sweeps=20, cutoff=1e-12, trunc="rho", goal=1e-7,
                       cvgE=cvgE)
    assert len(psi.sweep_stats) == len(info["sweeps"]) < 20
    assert psi.sweep_stats[-1]["converged"] == 1
    assert all(s["converged"] == 0 for s in psi.sweep_stats[:-1])
    assert abs(E - E0) <= 1e-10 * abs(E0)


def test_functional_env_updates_match_oracle(dmrgb, ctx):
    """Lupdate(Lenv, dualpsi, psi, mpo) / Rupdate(Renv, dualpsi, psi, mpo) on dense tensors
    (lib/MPO_MPS/Lupdate.jl:17-26, Rupdate.jl:17-26) with a dual tensor different from psi."""
    rng = np.random.default_rng(21)
    ml, d, mr, wl, wr = 7, 3, 5, 4, 6
    psi = rng.standard_normal((ml, d, mr))
    dual = rng.standard_normal((ml, d, mr))
    W = rng.standard_normal((wl, d, d, wr))
    W[np.abs(W) < 0.5] = 0.0                   # sparse like a real MPO
    L = rng.standard_normal((ml, wl, ml))
    R = rng.standard_normal((mr, wr, mr))
    Lo = od.Lupdate(L, dual, psi, W)
    Ro = od.Rupdate(R, dual, psi, W)
    assert _rel(dmrgb.Lupdate(L, dual, psi, W, ctx=ctx), Lo) < RTOL_CONTRACT
    assert _rel(dmrgb.Rupdate(R, dual, psi, W, ctx=ctx), Ro) < RTOL_CONTRACT
    # dual = psi (the form every sweep uses)
    assert _rel(dmrgb.Lupdate(L, psi, psi, W, ctx=ctx), od.Lupdate(L, psi, psi, W)) < RTOL_CONTRACT


def test_block_upload_round_trip_at_a_4096_bond(dmrgb, ctx):
    """The block-form upload (dmrg_mps_upload_blocks, what the Julia binding sends for a Qtens
    MPS) at a bond of dimension 4096 in three U(1) sectors, the size of the 4x16 cylinder's largest
    bond: the blocks come back bit for bit, through the per-site and the batched downloads, and
    the environments built from them agree with the dense-equivalent contraction of the same
    state."""
    rng = np.random.default_rng(4)
    sectors = [[((0,), 1)], [((-1,), 1), ((1,), 1)], [((-2,), 1000), ((0,), 2096), ((2,), 1000)],
               [((-1,), 1), ((1,), 1)], [((0,), 1)]]
    phys = [[(1,), (-1,)]] * 4
    blocks = []
    for i in range(4):
        n = 0
        rq = {q: dd for q, dd in sectors[i + 1]}
        for qa, da in sectors[i]:
            for ps in phys[i]:
                qb = (qa[0] + ps[0],)
                if qb in rq:
                    n += da * rq[qb]
        blocks.append(rng.standard_normal(n))
    psi = dmrgb.MPS(oc=1)
    psi.sectors, psi.blocks, psi.phys = sectors, blocks, phys
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 4).with_qn(dmrgb.SPIN_QN)
    dev = dmrgb.DeviceState(psi, mpo.device(ctx))
    assert dev.bond(2) == sectors[2]
    for i in range(4):
        assert np.array_equal(dev.site_blocks(i), blocks[i])
    # the batched downloads (every bond / every site in one call) give the same
    assert dev.bonds() == [dev.bond(b) for b in range(5)] == sectors
    for a, b in zip(dev.all_site_blocks(), blocks):
        assert np.array_equal(a, b)
    dev.env_build()
    dense = [dev.site_dense(i) for i in range(4)]
    W = [np.asarray(w) for w in mpo.W]
    L2 = od.Lupdate(od.Lupdate(np.ones((1, 1, 1)), dense[0], dense[0], W[0]), dense[1], dense[1], W[1])
    dev.lupdate(1)
    assert _rel(dev.env(2, True), L2) < RTOL_CONTRACT


def test_two_half_sweeps_are_one_sweep(dmrgb, ctx):
    """halfsweep (algs/DMRG.jl:253): a sweep of L-1 steps in the current direction; two of them
    run exactly the steps of one full sweep, so every number is the same."""
    L = 10
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    a, b = dmrgb.neelMPS(L), dmrgb.neelMPS(L)
    Ea = dmrgb.dmrg(a, mpo, m=45, sweeps=3, cutoff=1e-12, ctx=ctx)
    Eb = dmrgb.dmrg(b, mpo, m=45, sweeps=6, cutoff=1e-12, halfsweep=True, ctx=ctx)
    assert Ea == Eb
    assert a.oc == b.oc == 0
    c = dmrgb.neelMPS(L)
    dmrgb.dmrg(c, mpo, m=45, sweeps=1, cutoff=1e-12, halfsweep=True, ctx=ctx)
    assert c.oc == L - 1
