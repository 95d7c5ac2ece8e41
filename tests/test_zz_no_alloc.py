"""The allocation-free Heff entry point against the regular one (through the C ABI).

dmrg_heff_apply_noalloc exists for callers that cannot allocate device memory where they apply the
effective Hamiltonian (a host framework whose allocator owns the free HBM, a solver loop that must
not call the allocator). It computes the same FP64 product as dmrg_heff_apply, with every
intermediate in a fixed array inside the library; this test checks two calls in a row against
the regular entry point (tolerance 1e-13 relative: same kernels, same order) and that a two-site
space beyond the fixed maximum is refused with DMRG_ERR_BUDGET. Device vectors come from torch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(dmrgb, ctx, L, m, qn, seed, oc):
    mpo = dmrgb.makeMPO(dmrgb.heisenbergMPO, 2, L)
    if qn:
        mpo = mpo.with_qn(dmrgb.SPIN_QN)
        psi = dmrgb.neelMPS(L)
        dmrgb.dmrg(psi, mpo, m=m, sweeps=2, cutoff=1e-12, ctx=ctx)   # grow a U(1) state
        psi.materialize()
        psi._dev = None
        psi.oc = oc          # environments are rebuilt for this centre
    else:
        psi = dmrgb.randMPS(2, L, m, seed=seed, oc=oc)
    Lenv, _ = dmrgb.makeEnv(psi, mpo, ctx=ctx)
    return Lenv.dev


def _noalloc(dmrgb, dev, iL, x):
    import torch
    xin = torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).cuda()
    yout = torch.full_like(xin, float("nan"))
    torch.cuda.synchronize()
    code = dmrgb.lib().dmrg_heff_apply_noalloc(dev.h, dev.dmpo.h, iL, xin.data_ptr(),
                                               yout.data_ptr(), 0)
    y = yout.cpu().numpy().reshape(x.shape, order="F")
    return code, y


@pytest.mark.parametrize("qn", [False, True])
def test_noalloc_matches_regular_heff_twice(dmrgb, ctx, qn):
    L, iL = 10, 4
    dev = _state(dmrgb, ctx, L, 16, qn, seed=4, oc=iL)
    rng = np.random.default_rng(9)
    dims = _dims(dmrgb, dev, iL)
    for call in range(2):                      # two calls in a row share the scratch array
        # both entry points read only the QN-allowed blocks of the input
        x = rng.standard_normal(dims)
        y_ref = dev.heff(iL, np.asfortranarray(x))
        code, y = _noalloc(dmrgb, dev, iL, x)
        assert code == 0, dmrgb.lib().dmrg_last_error(ctx.h)
        scale = max(np.max(np.abs(y_ref)), 1e-300)
        assert np.max(np.abs(y - y_ref)) <= 1e-13 * scale, f"call {call}"


def test_noalloc_in_place(dmrgb, ctx):
    """psi_in and psi_out may be one buffer: the input is read completely before the output is
    written, so the result equals the regular entry point's."""
    import torch
    L, iL = 10, 4
    dev = _state(dmrgb, ctx, L, 16, True, seed=4, oc=iL)
    x = np.random.default_rng(3).standard_normal(_dims(dmrgb, dev, iL))
    y_ref = dev.heff(iL, np.asfortranarray(x))
    buf = torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).cuda()
    torch.cuda.synchronize()
    code = dmrgb.lib().dmrg_heff_apply_noalloc(dev.h, dev.dmpo.h, iL, buf.data_ptr(),
                                               buf.data_ptr(), 0)
    assert code == 0, dmrgb.lib().dmrg_last_error(ctx.h)
    y = buf.cpu().numpy().reshape(x.shape, order="F")
    assert np.max(np.abs(y - y_ref)) <= 1e-13 * max(np.max(np.abs(y_ref)), 1e-300)


def _dims(dmrgb, dev, iL):
    import ctypes as C
    d = (C.c_int * 4)()
    assert dmrgb.lib().dmrg_twosite_dims(dev.h, dev.dmpo.h, iL, d) == 0
    return tuple(d)


def test_noalloc_refuses_spaces_beyond_its_maximum(dmrgb, ctx):
    L, iL = 18, 8
    dev = _state(dmrgb, ctx, L, 256, False, seed=5, oc=iL)
    x = np.zeros(_dims(dmrgb, dev, iL))
    code, _ = _noalloc(dmrgb, dev, iL, x)
    assert code == dmrgb._lib.ERR_BUDGET
    assert b"fixed maximum" in dmrgb.lib().dmrg_last_error(ctx.h)
