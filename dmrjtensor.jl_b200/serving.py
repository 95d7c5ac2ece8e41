"""Serving: many independent ``dmrg`` solves on one GPU (``dmrg_server_*`` in the C ABI).

``Server.submit(psi, mpo, m=..., sweeps=..., cutoff=...)`` queues what one call of
``dmrg(psi, mpo; m, minm, sweeps, cutoff)`` (``algs/DMRG.jl:549-588``) computes and returns a
ticket at once; ``poll``/``result`` report it. Up to ``slots`` solves run at the same time, each
in its own context and CUDA stream, admitted first come first served while their worst-case
device footprints fit in ``hbm_budget`` bytes. Inside their sweeps the solves' Heff applications
share grouped launches (``batched=False`` gives every solve its own). A solve's result is the
same alone and in a mix.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Request, Result, ServerConfig, lib
from .state import MPO, MPS, _int_arr, _ptr_array, make_params


class ServerError(_lib.DmrgError):
    pass


class Server:
    def __init__(self, device=0, slots=4, hbm_budget=0, batched=True):
        cfg = ServerConfig()
        cfg.device, cfg.slots, cfg.hbm_budget_bytes = int(device), int(slots), int(hbm_budget)
        cfg.unbatched = 0 if batched else 1
        h = C.c_void_p()
        code = lib().dmrg_server_create(C.byref(cfg), C.byref(h))
        if code != _lib.OK:
            raise ServerError(code, "dmrg_server_create failed (no device, or bad slot count)")
        self.h = h
        self.slots = slots

    def _check(self, code):
        if code != _lib.OK:
            msg = lib().dmrg_server_last_error(self.h)
            raise ServerError(code, msg.decode() if msg else "")

    def stats(self):
        """(shared Heff launches, Heff applications they carried) since the server started."""
        a, b = C.c_longlong(), C.c_longlong()
        self._check(lib().dmrg_server_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def submit(self, psi: MPS, mpo: MPO, m=0, sweeps=1, minm=2, cutoff=0.0, krylov=2,
               SvNbond=0, degen_rtol=0.0, precision="fp64"):
        """Queue one solve; returns its ticket. ``psi`` is copied (dense-equivalent tensors)."""
        L = len(mpo)
        if psi.tensors is None:
            psi.materialize()
        As = [np.asfortranarray(a, dtype=float) for a in psi.tensors]
        Ws = [np.asfortranarray(w, dtype=float) for w in mpo.W]
        d = [w.shape[1] for w in Ws]
        keep = [As, Ws]
        r = Request()
        r.L, r.nsym = L, mpo.nsym
        r.d, r.wl, r.wr = _int_arr(d), _int_arr([w.shape[0] for w in Ws]), \
            _int_arr([w.shape[3] for w in Ws])
        r.W = _ptr_array(Ws, C.c_double)
        if mpo.nsym:
            phys = [np.asarray(mpo.qlabels[i], dtype=np.int32).reshape(-1) for i in range(L)]
            keep.append(phys)
            r.phys_qn = _ptr_array(phys, C.c_int)
        r.ml, r.mr = _int_arr([a.shape[0] for a in As]), _int_arr([a.shape[2] for a in As])
        r.A = _ptr_array(As, C.c_double)
        r.oc, r.sweeps = int(psi.oc), int(sweeps)
        r.params = make_params(m, minm, cutoff, krylov, precision, SvNbond, degen_rtol)
        t = C.c_longlong()
        self._check(lib().dmrg_server_submit(self.h, C.byref(r), C.byref(t)))
        del keep
        return t.value

    def poll(self, ticket, wait_ms=0):
        """Status and statistics of a ticket (``status``: 0 queued, 1 running, 2 done,
        3 failed), waiting up to ``wait_ms`` ms (negative: until it finishes)."""
        res = Result()
        self._check(lib().dmrg_server_poll(self.h, int(ticket), int(wait_ms), C.byref(res)))
        out = res.as_dict()
        if out["status"] == _lib.REQ_FAILED:
            msg = lib().dmrg_server_last_error(self.h)
            out["message"] = msg.decode() if msg else ""
        return out

    def result(self, ticket, fetch=True):
        """Waits for the ticket; returns (statistics, final MPS or None). Raises if it failed."""
        st = self.poll(ticket, -1)
        if st["status"] != _lib.REQ_DONE:
            raise ServerError(st["error"], st.get("message", "solve failed"))
        if not fetch:
            return st, None
        tensors, oc = [], C.c_int()
        i = 0
        while True:
            ml, d, mr = C.c_int(), C.c_int(), C.c_int()
            code = lib().dmrg_server_fetch_site(self.h, int(ticket), i, None, C.byref(ml),
                                                C.byref(d), C.byref(mr), C.byref(oc))
            if code != _lib.OK:
                break
            a = np.zeros((ml.value, d.value, mr.value), order="F")
            self._check(lib().dmrg_server_fetch_site(
                self.h, int(ticket), i, a.ctypes.data_as(C.POINTER(C.c_double)), None, None,
                None, None))
            tensors.append(np.array(a))
            i += 1
        return st, MPS(tensors, oc=oc.value)

    def release(self, ticket):
        self._check(lib().dmrg_server_release(self.h, int(ticket)))

    def close(self):
        if self.h:
            lib().dmrg_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
