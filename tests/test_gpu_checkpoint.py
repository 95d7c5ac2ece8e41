"""Checkpoint / resume of a device state (the persistence of ``largeMPS`` / ``loadMPS``,
``lib/MPS/largeMPS.jl:19-81``).

A checkpoint round trip is exact (sectors, centre, every block bit for bit). A run of 2 sweeps,
checkpointed, loaded into a new state and continued for 2 sweeps gives the same sweep energies,
truncation errors and final tensors, bit for bit, as 4 uninterrupted sweeps (the environments
rebuilt after the load are the same deterministic function of the tensors as the ones the sweep
leaves). A corrupted byte, a truncated file and an MPO of another length are rejected with an
error, not a device fault.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(dmrgb, L=16):
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    return mpo, dmrgb.neelMPS(L)


def test_checkpoint_round_trip_is_exact(dmrgb, ctx, tmp_path):
    mpo, psi = _setup(dmrgb)
    dmrgb.dmrg(psi, mpo, m=32, sweeps=2, cutoff=1e-12, ctx=ctx)
    path = dmrgb.largeMPS(psi, tmp_path / "psi.ckp")
    back = dmrgb.loadMPS(path, mpo, ctx=ctx)
    assert back.oc == psi.oc
    assert back.sectors == psi.sectors
    for a, b in zip(psi.blocks, back.blocks):
        assert np.array_equal(a, b)


def test_resume_equals_uninterrupted_run(dmrgb, ctx, tmp_path):
    mpo, psi_a = _setup(dmrgb)
    dmrgb.dmrg(psi_a, mpo, m=32, sweeps=4, cutoff=1e-12, ctx=ctx)
    mpo_b, psi_b = _setup(dmrgb)
    dmrgb.dmrg(psi_b, mpo_b, m=32, sweeps=2, cutoff=1e-12, ctx=ctx)
    path = dmrgb.largeMPS(psi_b, tmp_path / "half.ckp")
    psi_c = dmrgb.loadMPS(path, mpo_b, ctx=ctx)
    dmrgb.dmrg(psi_c, mpo_b, m=32, sweeps=2, cutoff=1e-12, ctx=ctx)
    for sa, sc in zip(psi_a.sweep_stats[2:], psi_c.sweep_stats):
        assert sa["energy"] == sc["energy"]
        assert sa["max_truncerr"] == sc["max_truncerr"]
    assert psi_c.sectors == psi_a.sectors
    for a, c in zip(psi_a.blocks, psi_c.blocks):
        assert np.array_equal(a, c)


def test_corrupt_truncated_and_mismatched_checkpoints_are_rejected(dmrgb, ctx, tmp_path):
    mpo, psi = _setup(dmrgb)
    dmrgb.dmrg(psi, mpo, m=16, sweeps=1, ctx=ctx)
    path = dmrgb.largeMPS(psi, tmp_path / "ok.ckp")
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.ckp"
    raw[len(raw) // 2] ^= 0x40
    bad.write_bytes(bytes(raw))
    with pytest.raises(dmrgb.DmrgError, match="checksum"):
        dmrgb.loadMPS(bad, mpo, ctx=ctx)
    short = tmp_path / "short.ckp"
    short.write_bytes(path.read_bytes()[:100])
    with pytest.raises(dmrgb.DmrgError):
        dmrgb.loadMPS(short, mpo, ctx=ctx)
    other = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 12).with_qn(dmrgb.SPIN_QN)
    with pytest.raises(dmrgb.DmrgError, match="length"):
        dmrgb.loadMPS(path, other, ctx=ctx)
