"""Split-precision forms (Heff and environment GEMMs on tcgen05 as 3 TF32 products or as 9 BF16
products) against the plain FP64 form.

One Heff application agrees with FP64 to FP32 accuracy (the split products accumulate in FP32,
relative 1e-5 here), in the direct form (small lists) and the image-fed form (large lists, with the
MPO mixing fused into the pack of the second GEMM's operand); whole DMRG runs from the same start
agree in energy within 1e-8, the reported energy of a sweep being the FP64 Rayleigh quotient of
the final Ritz vector.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _heff(dmrgb, dev, iL, x, precision):
    y = np.zeros_like(x, order="F")
    dp = C.POINTER(C.c_double)
    code = dmrgb.lib().dmrg_heff_apply(dev.h, dev.dmpo.h, iL, np.asfortranarray(x).ctypes.data_as(dp),
                                       y.ctypes.data_as(dp), precision)
    assert code == 0, dmrgb.lib().dmrg_last_error(dev.ctx.h)
    return y


FORMS = [1, 2]        # DMRG_PREC_3XTF32, DMRG_PREC_BF16X9


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("qn", [False, True])
def test_split_heff_matches_fp64(dmrgb, ctx, qn, form):
    L, iL = 12, 5
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    if qn:
        mpo = mpo.with_qn(dmrgb.SPIN_QN)
        psi = dmrgb.neelMPS(L)
        dmrgb.dmrg(psi, mpo, m=48, sweeps=2, cutoff=1e-12, ctx=ctx)
        psi.materialize()
        psi._dev = None
        psi.oc = iL
    else:
        psi = dmrgb.randMPS(2, L, 40, seed=3, oc=iL)
    Lenv, _ = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    dev = Lenv.dev
    d = (C.c_int * 4)()
    assert dmrgb.lib().dmrg_twosite_dims(dev.h, dev.dmpo.h, iL, d) == 0
    x = np.random.default_rng(2).standard_normal(tuple(d))
    y64 = _heff(dmrgb, dev, iL, x, 0)
    y32 = _heff(dmrgb, dev, iL, x, form)
    scale = np.max(np.abs(y64))
    assert np.max(np.abs(y32 - y64)) <= 1e-5 * scale


@pytest.mark.parametrize("form", FORMS)
def test_split_heff_image_form_matches_fp64(dmrgb, ctx, form):
    """Bond dimension 384 either side: every Heff GEMM list is above 1 GFLOP and takes the
    image-fed form (operand windows converted once into chunk images of their split parts; the
    mixing summed inside the pack of the second GEMM's operand). The second GEMM accumulates
    K = d w m = 3840 products in FP32 (ten times the first test's), so the bound is relative 5e-5
    here (measured 1.3e-5)."""
    L, iL = 20, 9
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, 384, seed=8, oc=iL)
    Lenv, _ = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    dev = Lenv.dev
    d = (C.c_int * 4)()
    assert dmrgb.lib().dmrg_twosite_dims(dev.h, dev.dmpo.h, iL, d) == 0
    assert tuple(d) == (384, 2, 2, 384)
    x = np.random.default_rng(9).standard_normal(tuple(d))
    y64 = _heff(dmrgb, dev, iL, x, 0)
    y32 = _heff(dmrgb, dev, iL, x, form)
    assert np.max(np.abs(y32 - y64)) <= 5e-5 * np.max(np.abs(y64))


@pytest.mark.parametrize("form", FORMS)
def test_split_heff_cached_environment_images(dmrgb, ctx, form):
    """The applications of one plan after its first reuse the environment images the first packed
    (as a bond step's Lanczos iterations do): the fourth application of a plan gives the first's
    result bit for bit, at the image-fed size of the test above."""
    L, iL = 20, 9
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, 384, seed=8, oc=iL)
    Lenv, _ = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    dev = Lenv.dev
    d = (C.c_int * 4)()
    assert dmrgb.lib().dmrg_twosite_dims(dev.h, dev.dmpo.h, iL, d) == 0
    x = np.asfortranarray(np.random.default_rng(10).standard_normal(tuple(d)))
    dp = C.POINTER(C.c_double)
    y1 = np.zeros_like(x, order="F")
    y4 = np.zeros_like(x, order="F")
    for y, reps in ((y1, 1), (y4, 4)):
        code = dmrgb.lib().dmrg_test_heff_apply_repeat(dev.h, dev.dmpo.h, iL, x.ctypes.data_as(dp),
                                                       y.ctypes.data_as(dp), form, reps)
        assert code == 0, dmrgb.lib().dmrg_last_error(dev.ctx.h)
    assert np.array_equal(y1, y4)
    assert np.array_equal(y1, _heff(dmrgb, dev, iL, x, form))


@pytest.mark.parametrize("form", ["3xtf32", "bf16x9"])
def test_split_dmrg_energy_within_1e8_of_fp64(dmrgb, ctx, form):
    L = 16
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L).with_qn(dmrgb.SPIN_QN)
    ramp = [16, 32, 64, 64, 64, 64]
    e = {}
    for prec in ("fp64", form):
        psi = dmrgb.neelMPS(L)
        e[prec] = dmrgb.dmrg(psi, mpo, m=ramp, cutoff=1e-12, precision=prec, ctx=ctx)
    assert abs(e[form] - e["fp64"]) <= 1e-8
    from oracle import ed, models as om
    ref = ed.sparse_ground_energy(om.make_mpo([om.heisenberg_bulk()] * L, 2))
    assert abs(e[form] - ref) <= 1e-8 * abs(ref)


def test_split_dense_lanczos_k(dmrgb, ctx):
    L = 14
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    e = {}
    for prec in ("fp64", "3xtf32"):
        psi = dmrgb.randMPS(2, L, 16, seed=11)
        e[prec] = dmrgb.dmrg(psi, mpo, m=[32, 64, 64, 64], cutoff=1e-12, krylov=8, precision=prec,
                             ctx=ctx)
    from oracle import ed, models as om
    ref = ed.sparse_ground_energy(om.make_mpo([om.heisenberg_bulk()] * L, 2))
    assert abs(e["3xtf32"] - e["fp64"]) <= 1e-8
    assert abs(e["3xtf32"] - ref) <= 1e-8 * abs(ref)


def test_heff_timing_hook_reports_every_form(dmrgb, ctx):
    psi = dmrgb.randMPS(2, 12, 64, seed=5, oc=5)
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, 12)
    Lenv, _ = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    dev = Lenv.dev
    for prec in (0, 1, 2):
        sec, fl = C.c_double(), C.c_double()
        assert dmrgb.lib().dmrg_test_heff_time(dev.h, dev.dmpo.h, 5, prec, 3, C.byref(sec),
                                               C.byref(fl)) == 0
        assert sec.value > 0 and fl.value > 0
    # an unknown precision code is refused
    assert dmrgb.lib().dmrg_test_heff_time(dev.h, dev.dmpo.h, 5, 7, 1, C.byref(sec),
                                           C.byref(fl)) == dmrgb._lib.ERR_ARG


@pytest.mark.parametrize("form", ["3xtf32", "bf16x9"])
def test_split_environment_updates_match_fp64(dmrgb, ctx, form):
    """The environment updates of a split-precision sweep (fp64_final = 0: every update on the
    tensor cores) agree with an FP64 rebuild from the same site tensors to FP32 accuracy: relative
    5e-5 after a chain of 13 updates (each product accumulates up to K ~ 1300 terms in FP32,
    ~2^-24 K relative, and the chain compounds 13 of them; measured 0.8e-5 to 1.7e-5 depending on
    the site tensors' rounding)."""
    L = 14
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, 128, seed=5)
    dev = dmrgb.DeviceState(psi, mpo.device(ctx))
    dev.env_build()
    dev.sweep(dmrgb.make_params(maxm=256, cutoff=1e-14, precision=form, fp64_final=0))
    assert dev.oc == 0
    R32 = [dev.env(i, False) for i in range(1, L)]
    dev.env_build()                                  # FP64, from the same site tensors
    for i, R in zip(range(1, L), R32):
        R64 = dev.env(i, False)
        assert np.max(np.abs(R - R64)) <= 5e-5 * np.max(np.abs(R64)), f"Renv[{i}]"


def test_split_sweep_in_image_form_matches_fp64_from_the_same_state(dmrgb, ctx):
    """Dense L=20 chain at bond dimension 384: the middle bonds' Heff lists (2.3 GFLOP) take the
    image-fed form, so a split sweep runs it inside the captured Krylov step, with the
    environments' images packed once per bond step, the mixing fused into the pack and the
    environment updates on the tensor cores. From one FP64-converged state, a sweep in each split
    form ends within 1e-8 (relative) of the FP64 sweep's energy."""
    L, m = 20, 384
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    psi = dmrgb.randMPS(2, L, m, seed=3)
    dmrgb.dmrg(psi, mpo, m=m, sweeps=3, cutoff=0.0, ctx=ctx)
    start, oc = [np.array(psi[i]) for i in range(L)], psi.oc
    e = {}
    for prec in ("fp64", "3xtf32", "bf16x9"):
        p = dmrgb.MPS([a.copy() for a in start], oc=oc)
        e[prec] = dmrgb.dmrg(p, mpo, m=m, sweeps=1, cutoff=0.0, precision=prec, ctx=ctx)
    for prec in ("3xtf32", "bf16x9"):
        assert abs(e[prec] - e["fp64"]) <= 1e-8 * abs(e["fp64"]), (prec, e)
