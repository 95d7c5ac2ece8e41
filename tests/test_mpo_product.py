"""Host-side MPO product used by ``expect(psi, H1, ..., Hn)`` (``lib/MPO_MPS/expect.jl:19-45``:
Hn is next to the ket). The product MPO's full matrix must equal the operator product H1 H2 of the
factors' full matrices, in that order, for two operators that do not commute."""
import numpy as np

from oracle import ed


def test_mpo_product_is_the_operator_product_in_order(dmrgb):
    L = 5
    H = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    T = dmrgb.makeMPO(dmrgb.tfiMPO(h=0.7), 2, L)
    P = dmrgb.mpo_product(H, T)
    # ed.full_h returns M[ket, bra]; the operator O[bra, ket] is its transpose
    Oh, Ot, Op = ed.full_h(H.W).T, ed.full_h(T.W).T, ed.full_h(P.W).T
    assert np.max(np.abs(Oh @ Ot - Ot @ Oh)) > 1.0
    assert np.max(np.abs(Op - Oh @ Ot)) <= 1e-12
    assert P.W[0].shape[0] == 1 and P.W[-1].shape[3] == 1
    # weightless product states are dropped, so the bonds are at most w1 w2
    assert all(w.shape[0] <= H.W[i].shape[0] * T.W[i].shape[0] for i, w in enumerate(P.W))


def test_mpo_product_keeps_charge_labels_consistent(dmrgb):
    """The product of two U(1) Heisenberg MPOs, after dropping weightless bond states, admits the
    makeqMPO labels: every non-zero element conserves charge under the labels the oracle's
    restatement of the rule derives (the condition the device upload checks)."""
    from oracle import models as om
    L = 6
    H = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    P = dmrgb.mpo_product(H, H)
    phys = [[(1,), (-1,)]] * L
    r = om.mpo_bond_labels(P.W, phys)
    for i, W in enumerate(P.W):
        for w1, s, t, w2 in zip(*np.nonzero(W)):
            q = tuple(a - b + c for a, b, c in zip(r[i][w1], phys[i][s], phys[i][t]))
            assert q == r[i + 1][w2]
    Oh, Op = ed.full_h(H.W).T, ed.full_h(P.W).T
    assert np.max(np.abs(Op - Oh @ Oh)) <= 1e-12
