"""ctypes binding of libdmrgb200.so (the C ABI declared in include/dmrg_b200.h).

The library is required: importing this module without the built ``libdmrgb200.so`` raises,
and every call that needs a GPU raises when the library reports no CUDA device. There is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libdmrgb200.so"

OK, ERR_ARG, ERR_SHAPE, ERR_QN, ERR_OOM, ERR_BUDGET, ERR_TIMEOUT, ERR_CUDA, ERR_STATE, ERR_NOCUDA = range(10)
PREC = {"fp64": 0, "3xtf32": 1, "bf16x9": 2}

ERRNAMES = {1: "ERR_ARG", 2: "ERR_SHAPE", 3: "ERR_QN", 4: "ERR_OOM", 5: "ERR_BUDGET",
            6: "ERR_TIMEOUT", 7: "ERR_CUDA", 8: "ERR_STATE", 9: "ERR_NOCUDA"}


class Params(C.Structure):
    _fields_ = [("maxm", C.c_int), ("minm", C.c_int), ("cutoff", C.c_double),
                ("krylov", C.c_int), ("precision", C.c_int), ("svnbond", C.c_int),
                ("degen_rtol", C.c_double), ("betatest", C.c_double), ("fp64_final", C.c_int),
                ("profile", C.c_int), ("cvgE", C.c_int), ("tune", C.c_int),
                ("goal", C.c_double), ("graph", C.c_int), ("halfsweep", C.c_int)]


class SweepStats(C.Structure):
    _fields_ = [("energy", C.c_double), ("max_truncerr", C.c_double), ("biggest_m", C.c_int),
                ("n_matvec", C.c_int), ("entropy", C.c_double), ("seconds", C.c_double),
                ("heff_flops", C.c_double), ("heff_seconds", C.c_double),
                ("env_flops", C.c_double), ("env_seconds", C.c_double),
                ("eig_seconds", C.c_double), ("vec_seconds", C.c_double),
                ("d_top", C.c_double * 8), ("gemm_flops", C.c_double),
                ("gemm_seconds", C.c_double), ("gemm_launches", C.c_int), ("eig_max_n", C.c_int),
                ("host_seconds", C.c_double), ("wait_seconds", C.c_double),
                ("converged", C.c_int), ("graph_launches", C.c_int), ("cvg_check", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "d_top"}
        d["d_top"] = list(self.d_top)
        return d


class Noise(C.Structure):
    _fields_ = [("noise", C.c_double), ("noise_goal", C.c_double), ("noise_incr", C.c_double),
                ("reserved", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("hbm_budget_bytes", C.c_size_t),
                ("unbatched", C.c_int), ("reserved", C.c_int * 7)]


class Request(C.Structure):
    _fields_ = [("L", C.c_int), ("nsym", C.c_int),
                ("d", C.POINTER(C.c_int)), ("wl", C.POINTER(C.c_int)), ("wr", C.POINTER(C.c_int)),
                ("W", C.POINTER(C.POINTER(C.c_double))), ("phys_qn", C.POINTER(C.POINTER(C.c_int))),
                ("ml", C.POINTER(C.c_int)), ("mr", C.POINTER(C.c_int)),
                ("A", C.POINTER(C.POINTER(C.c_double))), ("oc", C.c_int), ("sweeps", C.c_int),
                ("params", Params)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(4)


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("error", C.c_int), ("energy", C.c_double),
                ("max_truncerr", C.c_double), ("entropy", C.c_double), ("biggest_m", C.c_int),
                ("sweeps_done", C.c_int), ("queue_seconds", C.c_double),
                ("run_seconds", C.c_double), ("footprint_bytes", C.c_size_t)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DmrgError(RuntimeError):
    """Raised for every non-zero status returned by the library."""

    def __init__(self, code, msg):
        super().__init__(f"{ERRNAMES.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_IP = C.POINTER(C.c_int)
_DP = C.POINTER(C.c_double)
_DPP = C.POINTER(_DP)
_IPP = C.POINTER(_IP)

SIGNATURES = {
    "dmrg_abi_version": (C.c_int, []),
    "dmrg_kernel_launches": (C.c_longlong, []),
    "dmrg_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(_P)]),
    "dmrg_ctx_destroy": (C.c_int, [_P]),
    "dmrg_last_error": (C.c_char_p, [_P]),
    "dmrg_ctx_memory": (C.c_int, [_P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "dmrg_ctx_tuner": (C.c_int, [_P, _IP, _IP, _IP]),
    "dmrg_mpo_upload": (C.c_int, [_P, C.c_int, C.c_int, _IP, _IP, _IP, _DPP, _IPP, _IPP,
                                  C.POINTER(_P)]),
    "dmrg_mpo_destroy": (C.c_int, [_P]),
    "dmrg_mps_upload": (C.c_int, [_P, _P, _IP, _IP, _DPP, _IPP, C.c_int, C.POINTER(_P)]),
    "dmrg_mps_upload_blocks": (C.c_int, [_P, _P, _IP, _IPP, _IPP, _DPP, C.c_int, C.POINTER(_P)]),
    "dmrg_state_destroy": (C.c_int, [_P]),
    "dmrg_state_oc": (C.c_int, [_P, _IP]),
    "dmrg_bond_info": (C.c_int, [_P, C.c_int, _IP, _IP, _IP]),
    "dmrg_site_size": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int64)]),
    "dmrg_mps_download_blocks": (C.c_int, [_P, C.c_int, _DP]),
    "dmrg_mps_download": (C.c_int, [_P, C.c_int, _DP, _IP, _IP]),
    "dmrg_env_build": (C.c_int, [_P, _P]),
    "dmrg_lupdate": (C.c_int, [_P, _P, C.c_int]),
    "dmrg_rupdate": (C.c_int, [_P, _P, C.c_int]),
    "dmrg_env_get": (C.c_int, [_P, C.c_int, C.c_int, _DP, _IP]),
    "dmrg_state_save": (C.c_int, [_P, C.c_char_p]),
    "dmrg_state_load": (C.c_int, [_P, _P, C.c_char_p, C.POINTER(_P)]),
    "dmrg_expect": (C.c_int, [_P, _P, _DP]),
    "dmrg_env_step": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _DP,
                                _DP, _DP, _DP, _DP]),
    "dmrg_correlationmatrix": (C.c_int, [_P, C.c_int, _DP, _DP, _DP, _DP]),
    "dmrg_correlation": (C.c_int, [_P, C.c_int, C.c_int, _IP, _DP, _IP, _IP, _DP, _DP]),
    "dmrg_mps_download_all_blocks": (C.c_int, [_P, _DP, C.POINTER(C.c_int64)]),
    "dmrg_bonds_info": (C.c_int, [_P, _IP, _IP, _IP]),
    "dmrg_heff_apply": (C.c_int, [_P, _P, C.c_int, _DP, _DP, C.c_int]),
    "dmrg_heff_apply_noalloc": (C.c_int, [_P, _P, C.c_int, C.c_void_p, C.c_void_p, C.c_int]),
    "dmrg_twosite_dims": (C.c_int, [_P, _P, C.c_int, _IP]),
    "dmrg_sweep": (C.c_int, [_P, _P, C.POINTER(Params), C.POINTER(SweepStats)]),
    "dmrg_params_default": (None, [C.POINTER(Params)]),
    "dmrg_noise_default": (None, [C.POINTER(Noise)]),
    "dmrg_sweep3s": (C.c_int, [_P, _P, C.POINTER(Params), C.POINTER(Noise), C.POINTER(SweepStats)]),
    "dmrg_tdvp": (C.c_int, [_P, _P, C.POINTER(Params), C.c_double, C.c_int, C.POINTER(SweepStats)]),
    "dmrg_test_gemm": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _DP, C.c_int,
                                 _DP, C.c_int, _DP, C.c_int]),
    "dmrg_test_eigh": (C.c_int, [_P, C.c_int, _IP, _DP, _DP]),
    "dmrg_test_syevt": (C.c_int, [_P, C.c_int, _IP, _IP, _DP, _DP, _DP]),
    "dmrg_test_heff_time": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _DP, _DP]),
    "dmrg_test_heff_apply_repeat": (C.c_int, [_P, _P, C.c_int, _DP, _DP, C.c_int, C.c_int]),
    "dmrg_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(_P)]),
    "dmrg_server_submit": (C.c_int, [_P, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "dmrg_server_poll": (C.c_int, [_P, C.c_longlong, C.c_int, C.POINTER(Result)]),
    "dmrg_server_fetch_site": (C.c_int, [_P, C.c_longlong, C.c_int, _DP, _IP, _IP, _IP, _IP]),
    "dmrg_server_release": (C.c_int, [_P, C.c_longlong]),
    "dmrg_server_destroy": (C.c_int, [_P]),
    "dmrg_server_last_error": (C.c_char_p, [_P]),
    "dmrg_server_stats": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
}

_lib = None


def lib():
    """The loaded library (loaded on first use; raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with dmrjtensor.jl_b200/build.py "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, ctx=None):
    if code != OK:
        msg = lib().dmrg_last_error(ctx)
        raise DmrgError(code, msg.decode() if msg else "")
