"""Serving loop (dmrg_server_* through the C ABI): a solve gives the same result alone and in a mix.

The same five requests (transverse-field Ising chains and one U(1) Heisenberg chain) run one at
a time on a one-slot server, all at once on a four-slot server whose solves share their Heff
launches (the batched launches must have carried more than one solve on average), all at once
on a four-slot server without shared launches, and through the plain ``dmrg`` call; energies,
truncation errors, entropies and final tensors must agree bit for bit (every block of a shared
launch is computed as in a launch of its own, and the kernels are deterministic). The same holds
for the split-precision (3xTF32) option. One result is also checked against exact
diagonalisation, and a request larger than the HBM budget is refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(dmrgb):
    reqs = []
    for L, h in [(12, 0.7), (16, 1.0), (20, 1.3), (10, 0.9)]:
        mpo = dmrgb.makeMPO(dmrgb.tfiMPO(h=h), 2, L)
        plus = np.full((1, 2, 1), 1 / np.sqrt(2))
        psi = dmrgb.MPS([plus.copy() for _ in range(L)], oc=0)
        reqs.append((psi, mpo, dict(m=32, sweeps=3, cutoff=1e-10)))
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 16).with_qn(dmrgb.SPIN_QN)
    reqs.append((dmrgb.neelMPS(16), mpo, dict(m=32, sweeps=3, cutoff=1e-10)))
    return reqs


def _run(server, reqs, together):
    out = []
    if together:
        tickets = [server.submit(p, m, **kw) for p, m, kw in reqs]
        for t in tickets:
            out.append(server.result(t))
    else:
        for p, m, kw in reqs:
            out.append(server.result(server.submit(p, m, **kw)))
    return out


def _same(a, b):
    sa, pa = a
    sb, pb = b
    for k in ("energy", "max_truncerr", "entropy", "biggest_m", "sweeps_done"):
        assert sa[k] == sb[k], (k, sa[k], sb[k])
    assert pa.oc == pb.oc
    for x, y in zip(pa.tensors, pb.tensors):
        assert x.shape == y.shape and np.array_equal(x, y)


def test_alone_equals_mixed_equals_direct(dmrgb):
    reqs = _requests(dmrgb)
    with dmrgb.Server(slots=1) as s1:
        alone = _run(s1, reqs, together=False)
    with dmrgb.Server(slots=4) as s4:
        mixed = _run(s4, reqs, together=True)
        batches, carried = s4.stats()
    assert batches > 0 and carried / batches > 1.0     # Heff launches were shared
    with dmrgb.Server(slots=4, batched=False) as s4u:
        own = _run(s4u, reqs, together=True)
        assert s4u.stats() == (0, 0)
    for a, b, c in zip(alone, mixed, own):
        assert a[0]["status"] == 2
        _same(a, b)
        _same(a, c)
    # the plain dmrg() call computes the same numbers
    for (psi, mpo, kw), (st, _) in zip(reqs, alone):
        p = dmrgb.MPS([t.copy() for t in psi.tensors], oc=psi.oc)
        e = dmrgb.dmrg(p, mpo, m=kw["m"], sweeps=kw["sweeps"], cutoff=kw["cutoff"])
        assert e == st["energy"]


def test_split_precision_alone_equals_mixed(dmrgb):
    reqs = _requests(dmrgb)
    for _, _, kw in reqs:
        kw["precision"] = "3xtf32"
    with dmrgb.Server(slots=1) as s1:
        alone = _run(s1, reqs, together=False)
    with dmrgb.Server(slots=4) as s4:
        mixed = _run(s4, reqs, together=True)
    for a, b in zip(alone, mixed):
        assert a[0]["status"] == 2
        _same(a, b)


def test_served_energy_matches_exact_diagonalisation(dmrgb):
    from oracle import ed, models as om
    L, h = 10, 0.9
    psi = dmrgb.MPS([np.full((1, 2, 1), 1 / np.sqrt(2)) for _ in range(L)], oc=0)
    mpo = dmrgb.makeMPO(dmrgb.tfiMPO(h=h), 2, L)
    with dmrgb.Server(slots=2) as s:
        st, _ = s.result(s.submit(psi, mpo, m=64, sweeps=8, cutoff=1e-12, krylov=6))
    e0 = ed.ground_energy(om.make_mpo([om.tfi_bulk(h)] * L, 2))
    assert abs(st["energy"] - e0) <= 1e-9 * abs(e0)


def test_request_beyond_budget_is_refused(dmrgb):
    L = 40
    psi = dmrgb.MPS([np.full((1, 2, 1), 1 / np.sqrt(2)) for _ in range(L)], oc=0)
    mpo = dmrgb.makeMPO(dmrgb.tfiMPO(h=1.0), 2, L)
    with dmrgb.Server(slots=1, hbm_budget=1 << 20) as s:
        with pytest.raises(dmrgb.ServerError) as e:
            s.submit(psi, mpo, m=512, sweeps=1)
        assert e.value.code == 5   # DMRG_ERR_BUDGET
