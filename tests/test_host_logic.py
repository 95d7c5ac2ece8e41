"""Host-side containers and set-up (no GPU): product states, the seeded random MPS and its gauge,
block-form densification, parameter mapping."""
import numpy as np

from oracle import models as om


def test_random_mps_is_right_canonical(dmrgb):
    psi = dmrgb.randMPS(2, 10, 8, seed=2)
    for A in psi.tensors[1:]:
        a, d, b = A.shape
        M = A.reshape(a, d * b)
        assert np.max(np.abs(M @ M.T - np.eye(a))) < 1e-12
    assert abs(np.linalg.norm(psi.tensors[0]) - 1.0) < 1e-12


def test_neel_state(dmrgb):
    psi = dmrgb.neelMPS(6)
    ref = om.neel_mps(6)
    for a, b in zip(psi.tensors, ref):
        assert np.array_equal(a, b)


def test_block_form_densifies(dmrgb):
    psi = dmrgb.MPS()
    psi.sectors = [[((0,), 1)], [((1,), 1), ((-1,), 1)], [((0,), 2)]]
    psi.phys = [[(1,), (-1,)], [(1,), (-1,)]]
    # site 0: (ka=0, s=0)->q=1 (sector 0 of bond 1), (ka=0,s=1)->q=-1 (sector 1)
    psi.blocks = [np.array([0.6, 0.8]), np.array([1.0, 2.0, 3.0, 4.0])]
    A0 = psi[0]
    assert A0.shape == (1, 2, 2) and A0[0, 0, 0] == 0.6 and A0[0, 1, 1] == 0.8
    A1 = psi[1]                                   # (q=1, s=dn) -> 0 and (q=-1, s=up) -> 0
    assert A1.shape == (2, 2, 2)
    assert A1[0, 1, 0] == 1.0 and A1[0, 1, 1] == 2.0 and A1[1, 0, 0] == 3.0 and A1[1, 0, 1] == 4.0
    psi.materialize()
    assert psi.bond_labels[1] == [(1,), (-1,)]


def test_params_mapping(dmrgb):
    p = dmrgb.make_params(maxm=45, minm=3, cutoff=1e-9, krylov=8, precision="fp64")
    assert (p.maxm, p.minm, p.krylov) == (45, 3, 8) and p.cutoff == 1e-9


def test_dmrg_rejects_other_methods(dmrgb):
    import pytest
    with pytest.raises(ValueError, match="not defined"):
        dmrgb.dmrg(dmrgb.neelMPS(4), dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 4), method="2S")
