"""dmrjtensor_b200 -- a B200-native DMRG engine, drop-in for DMRJtensor.jl's
``dmrg(psi, mpo; m, sweeps, cutoff, method)`` path (two-site and 3S), its ``makeEnv``/``Lupdate``/
``Rupdate`` API, and ``tdvp``/``tdvp_twosite`` with real prefactors.

The compute runs in ``libdmrgb200.so`` (hand-written sm_100a kernels behind a C ABI,
``include/dmrg_b200.h``); this package is the host-side mirror of the reference interface.
Import it with :func:`load` from the repository root when the directory name is not importable.
"""
from ._lib import DmrgError, PREC, lib
from .models import (HUBBARD_QN, SPIN_QN, XXZ, cylinder_bonds, fermionOps, heisenbergCylinderMPO,
                     heisenbergMPO, hubbardMPO, makeMPO, spinOps, tfiMPO)
from .state import (MPO, MPS, Context, DeviceMPO, DeviceState, Env, Lupdate, Rupdate, applyOps,
                    correlation, correlationmatrix, default_context, dmrg, expect, largeMPS, loadMPS,
                    make_params, makeEnv, mpo_product, neelMPS, product_MPS, randMPS, tdvp,
                    tdvp_twosite)
from .serving import Server, ServerError



def kernel_launches():
    """Kernel launches issued by libdmrgb200.so in this process."""
    return int(lib().dmrg_kernel_launches())


__all__ = [
    "kernel_launches",
    "DmrgError", "PREC", "lib", "HUBBARD_QN", "SPIN_QN", "XXZ", "cylinder_bonds", "fermionOps",
    "heisenbergCylinderMPO", "heisenbergMPO", "hubbardMPO", "makeMPO", "spinOps", "tfiMPO", "MPO",
    "MPS", "Context", "DeviceMPO", "DeviceState", "Env", "Lupdate", "Rupdate", "applyOps",
    "default_context", "dmrg", "make_params", "makeEnv", "neelMPS", "product_MPS", "randMPS",
    "expect", "mpo_product", "correlation", "correlationmatrix", "largeMPS", "loadMPS", "tdvp", "tdvp_twosite",
    "Server", "ServerError",
]
