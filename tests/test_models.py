"""Host-side model builders of the package against the oracle's independent restatement, and the
cylinder MPO against a brute-force Hamiltonian (no GPU needed)."""
import itertools

import numpy as np
import pytest

from oracle import ed, models as om


@pytest.mark.parametrize("which", ["heis", "hub", "tfi"])
def test_bulk_mpos_match_oracle(dmrgb, which):
    L = 6
    if which == "heis":
        a = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
        b = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    elif which == "hub":
        a = dmrgb.makeMPO(dmrgb.hubbardMPO, 4, L)
        b = om.make_mpo([om.hubbard_bulk()] * L, 4)
    else:
        a = dmrgb.makeMPO(lambda i: dmrgb.tfiMPO(h=0.7), 2, L)
        b = om.make_mpo([om.tfi_bulk(0.7)] * L, 2)
    for wa, wb in zip(a.W, b):
        assert wa.shape == wb.shape and np.array_equal(wa, wb)


def test_cylinder_mpo_is_the_lattice_hamiltonian(dmrgb):
    W, Lx = 4, 3
    mpo = dmrgb.heisenbergCylinderMPO(W, Lx)
    assert max(w.shape[3] for w in mpo.W[:-1]) == 14
    H = ed.full_h(mpo.W)
    N = W * Lx
    sz = np.diag([0.5, -0.5]); sp = np.array([[0, 1.0], [0, 0]]); sm = sp.T

    def op(o, i):
        mats = [np.eye(2)] * N
        mats[i] = o
        r = mats[0]
        for m_ in mats[1:]:
            r = np.kron(r, m_)
        return r
    Hb = sum(op(sz, i) @ op(sz, j) + 0.5 * (op(sp, i) @ op(sm, j) + op(sm, i) @ op(sp, j))
             for i, j in dmrgb.cylinder_bonds(W, Lx))
    assert abs(np.linalg.eigvalsh(0.5 * (H + H.T))[0] - np.linalg.eigvalsh(Hb)[0]) < 1e-10
    assert len(dmrgb.cylinder_bonds(4, 16)) == 4 * 16 + 4 * 15


def test_hubbard_initial_state_matches_reference_construction(dmrgb):
    L = 6
    Cup, Cdn, F, *_ = dmrgb.fermionOps()
    psi = dmrgb.product_MPS([0] * L, 4)
    dmrgb.applyOps(psi, list(range(L // 2)), Cup.T, trail=F)
    dmrgb.applyOps(psi, list(range(L // 2)), Cdn.T, trail=F)
    ref = om.hubbard_half_filling_mps(L)
    for a, b in zip(psi.tensors, ref):
        assert np.array_equal(a, b)
