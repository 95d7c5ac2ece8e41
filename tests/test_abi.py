"""The C ABI library: it loads, exports every entry point that include/dmrg_b200.h declares, and
fails cleanly (status codes, messages) where no GPU is present. No compute call runs here."""
import ctypes as C
import re
from pathlib import Path

import pytest

HEADER = Path(__file__).resolve().parents[1] / "include" / "dmrg_b200.h"


def declared():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"DMRG_API\s+[\w\s\*]+?\b(dmrg_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(dmrgb):
    names = declared()
    assert len(names) >= 25
    lib = C.CDLL(str(dmrgb._lib.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    # and the Python binding covers them all with signatures
    assert set(names) <= set(dmrgb._lib.SIGNATURES)


def test_abi_version_and_defaults(dmrgb):
    lib = dmrgb.lib()
    assert lib.dmrg_abi_version() == 3
    p = dmrgb._lib.Params()
    lib.dmrg_params_default(C.byref(p))
    assert (p.minm, p.krylov, p.maxm, p.precision) == (2, 2, 0, 0)
    assert p.betatest == 1e-10
    # algvars defaults (algs/optimizeMPS.jl:527-528): energy convergence test, goal 0 (never stops)
    assert (p.cvgE, p.goal) == (1, 0.0)
    assert (p.tune, p.graph) == (1, 0)
    # the ctypes mirrors have the C layout: 80-byte params, stats end with the convergence fields
    assert C.sizeof(dmrgb._lib.Params) == 80
    # the 3S noise schedule (algs/optimizeMPS.jl:528-532)
    nz = dmrgb._lib.Noise()
    lib.dmrg_noise_default(C.byref(nz))
    assert (nz.noise, nz.noise_goal, nz.noise_incr) == (1.0, 0.3, 0.01)
    assert C.sizeof(dmrgb._lib.Noise) == 32


def test_null_handles_are_rejected(dmrgb):
    lib = dmrgb.lib()
    assert lib.dmrg_ctx_destroy(None) == dmrgb._lib.ERR_ARG
    assert lib.dmrg_state_destroy(None) == dmrgb._lib.ERR_ARG
    assert lib.dmrg_mpo_destroy(None) == dmrgb._lib.ERR_ARG
    assert lib.dmrg_sweep(None, None, None, None) == dmrgb._lib.ERR_ARG
    assert lib.dmrg_sweep3s(None, None, None, None, None) == dmrgb._lib.ERR_ARG
    assert lib.dmrg_tdvp(None, None, None, 0.0, 1, None) == dmrgb._lib.ERR_ARG


def test_context_without_gpu_reports_nocuda(dmrgb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    code = dmrgb.lib().dmrg_ctx_create(0, 0, C.byref(h))
    assert code == dmrgb._lib.ERR_NOCUDA
    assert b"no CUDA device" in dmrgb.lib().dmrg_last_error(None)
    with pytest.raises(dmrgb.DmrgError):
        dmrgb.Context(0)


def test_julia_binding_calls_only_declared_entry_points():
    """No Julia runtime exists here, so the shim's ccalls are checked as text: every symbol it
    calls is declared in the header, and its struct mirrors have the C field counts."""
    jl = (HEADER.parents[1] / "dmrjtensor.jl_b200" / "julia" / "DMRJtensorB200.jl").read_text()
    called = set(re.findall(r"ccall\(\(:(dmrg_\w+), libdmrg\)", jl))
    assert {"dmrg_sweep", "dmrg_sweep3s", "dmrg_tdvp", "dmrg_mps_upload_blocks"} <= called
    assert called <= set(declared())
    txt = HEADER.read_text()

    def c_fields(name):
        body = re.search(r"typedef struct " + name + r" \{(.*?)\} " + name + ";", txt, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        return len(re.findall(r"\b(?:int|double|size_t)\s+\w+", body))

    def jl_fields(name):
        body = re.search(r"mutable struct " + name + r"\n(.*?)\nend", jl, re.S).group(1)
        return len([ln for ln in body.splitlines() if "::" in ln])

    assert jl_fields("Params") == c_fields("dmrg_params")
    assert jl_fields("Noise") == c_fields("dmrg_noise")
    assert jl_fields("SweepStats") == c_fields("dmrg_sweep_stats")
