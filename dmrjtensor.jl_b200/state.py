"""MPS / MPO containers and the device-backed drop-in for the reference's two-site path.

``dmrg(psi, mpo; m, minm, sweeps, cutoff)`` mirrors ``algs/DMRG.jl:549-588`` (method "twosite"):
it returns the energy of the last bond step and updates ``psi`` in place (tensors and ``oc``).
``makeEnv``/``Lupdate``/``Rupdate`` mirror ``lib/Env/makeEnv.jl:196-246`` and
``lib/MPO_MPS/{L,R}update.jl`` on device-resident environments.

Indices are 0-based here (site ``i`` is the reference's site ``i+1``; ``psi.oc`` is ``oc-1``).
All arithmetic happens in libdmrgb200.so on the GPU; nothing here computes a contraction.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import Params, SweepStats, check, lib

# ------------------------------------------------------------------ context


class Context:
    """One CUDA stream on one device, with an optional HBM budget (bytes, 0 = none)."""

    def __init__(self, device=0, hbm_budget=0):
        h = C.c_void_p()
        code = lib().dmrg_ctx_create(int(device), C.c_size_t(int(hbm_budget)), C.byref(h))
        check(code, None)
        self.h = h
        self.device = device

    def tuner(self):
        """FP64 GEMM tile autotuner: (signatures seen, decided, won by 32 x 32 tiles)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().dmrg_ctx_tuner(self.h, C.byref(a), C.byref(b), C.byref(c)), self.h)
        return a.value, b.value, c.value

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        check(lib().dmrg_ctx_memory(self.h, C.byref(a), C.byref(b)), self.h)
        return a.value, b.value

    def close(self):
        if self.h:
            lib().dmrg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None or _default_ctx.h is None:
        _default_ctx = Context(0)
    return _default_ctx


def _ptr_array(arrs, ctype):
    P = C.POINTER(ctype)
    out = (P * len(arrs))()
    for i, a in enumerate(arrs):
        out[i] = a.ctypes.data_as(P) if a is not None else None
    return out


def _int_arr(vals):
    return (C.c_int * len(vals))(*[int(v) for v in vals])


# ------------------------------------------------------------------ host containers


class MPO:
    """``W[i]``: array [wl, d, d, wr] (ket = index 1, bra = index 2). ``qlabels``: per-site list
    of physical charges (tuples) or None for a dense MPO (``makeqMPO`` = :meth:`with_qn`)."""

    def __init__(self, tensors, qlabels=None):
        self.W = [np.asarray(w, dtype=float) for w in tensors]
        self.qlabels = qlabels
        self._dev = {}

    def __len__(self):
        return len(self.W)

    def __getitem__(self, i):
        return self.W[i]

    @property
    def nsym(self):
        return 0 if self.qlabels is None else len(self.qlabels[0][0])

    def with_qn(self, Qlabels):
        """``makeqMPO(Qlabels, mpo)``: the same operator with physical charges attached
        (``Qlabels`` repeats over the sites, ``lib/MPO/makeqMPO.jl:23-84``)."""
        ql = [list(map(tuple, Qlabels[i % len(Qlabels)])) if isinstance(Qlabels[0], list)
              else list(map(tuple, Qlabels)) for i in range(len(self))]
        return MPO(self.W, ql)

    def device(self, ctx=None):
        ctx = ctx or default_context()
        key = id(ctx)
        if key not in self._dev:
            self._dev[key] = DeviceMPO(self, ctx)
        return self._dev[key]


class MPS:
    """Matrix product state ``psi[i]``: [ml, d, mr]. Dense tensors, or QN block form.

    ``bond_labels[b]`` (optional) gives the charge of every state of bond b. After a device run
    with charges the state is held in block form (``sectors``, ``blocks``) like a Qtens; ``psi[i]``
    always returns the dense-equivalent tensor."""

    def __init__(self, tensors=None, oc=0, bond_labels=None):
        self.tensors = [np.asarray(a, dtype=float) for a in tensors] if tensors is not None else None
        self.oc = int(oc)
        self.bond_labels = bond_labels
        self.sectors = None     # L+1 lists of (qn tuple, dim)
        self.blocks = None      # L flat arrays (canonical block order)
        self.phys = None        # per-site physical labels when in block form
        self.sweep_stats = []
        self._dev = None

    def __len__(self):
        return len(self.tensors) if self.tensors is not None else len(self.blocks)

    def __getitem__(self, i):
        if self.tensors is None:
            return self._dense_site(i)
        return self.tensors[i]

    def __setitem__(self, i, A):
        self.materialize()
        self.tensors[i] = np.asarray(A, dtype=float)
        self._dev = None

    def _dense_site(self, i):
        Bl, Br, p = self.sectors[i], self.sectors[i + 1], self.phys[i]
        ml, mr = sum(d for _, d in Bl), sum(d for _, d in Br)
        out = np.zeros((ml, len(p), mr), order="F")
        ol = np.cumsum([0] + [d for _, d in Bl])
        orr = np.cumsum([0] + [d for _, d in Br])
        rq = {q: k for k, (q, _) in enumerate(Br)}
        off = 0
        data = self.blocks[i]
        for ka, (qa, da) in enumerate(Bl):
            for s, ps in enumerate(p):
                kb = rq.get(tuple(x + y for x, y in zip(qa, ps)))
                if kb is None:
                    continue
                db = Br[kb][1]
                blk = data[off:off + da * db].reshape((da, db), order="F")
                out[ol[ka]:ol[ka] + da, s, orr[kb]:orr[kb] + db] = blk
                off += da * db
        return out

    def materialize(self):
        """Convert block form into dense-equivalent tensors (with their bond labels)."""
        if self.tensors is not None:
            return self
        L = len(self.blocks)
        self.tensors = [self._dense_site(i) for i in range(L)]
        self.bond_labels = [[q for q, d in sec for _ in range(d)] for sec in self.sectors]
        self.sectors = self.blocks = None
        return self


def product_MPS(states, d, oc=0):
    """Product state with site i in basis state ``states[i]`` (``MPS(initTensor)`` pattern of
    ``test/dmrg_test.jl:55-58``)."""
    out = []
    for s in states:
        A = np.zeros((1, d, 1))
        A[0, s, 0] = 1.0
        out.append(A)
    return MPS(out, oc=oc)


def neelMPS(L):
    """Neel product state: up on odd (1-based) sites, down on even ones."""
    return product_MPS([0 if i % 2 == 0 else 1 for i in range(L)], 2)


def applyOps(psi, sites, op, trail=None):
    """``applyOps!`` (``lib/MPO_MPS/applyMPO.jl:21-34``) on a dense host MPS (initial states)."""
    psi.materialize()
    for p in sites:
        psi.tensors[p] = np.einsum("st,atb->asb", op, psi.tensors[p])
        if trail is not None:
            for j in range(p):
                psi.tensors[j] = np.einsum("st,atb->asb", trail, psi.tensors[j])
    psi._dev = None
    return psi


def randMPS(d, L, m, seed=0, oc=0):
    """Seeded random MPS: bond dim min(d^k, d^(L-k), m), entries standard normal, each tensor
    normalised, then moved to a right-canonical form with centre ``oc`` (the seeded stand-in for
    ``randMPS``, ``lib/MPS/randMPS.jl:27-56``; the gauge moves are exact QR/LQ, host-side set-up)."""
    rng = np.random.default_rng(seed)
    dims = [min(d ** k, d ** (L - k), m) for k in range(L + 1)]
    T = []
    for i in range(L):
        A = rng.standard_normal((dims[i], d, dims[i + 1]))
        T.append(A / np.linalg.norm(A))
    for i in range(L - 1, oc, -1):            # LQ from the right
        a, dd, b = T[i].shape
        Q, R = np.linalg.qr(T[i].reshape(a, dd * b).T)
        T[i] = Q.T.reshape(Q.shape[1], dd, b)
        T[i - 1] = np.tensordot(T[i - 1], R.T, axes=(2, 0))
    for i in range(0, oc):                    # QR from the left
        a, dd, b = T[i].shape
        Q, R = np.linalg.qr(T[i].reshape(a * dd, b))
        T[i] = Q.reshape(a, dd, Q.shape[1])
        T[i + 1] = np.tensordot(R, T[i + 1], axes=(1, 0))
    T[oc] = T[oc] / np.linalg.norm(T[oc])
    return MPS(T, oc=oc)


# ------------------------------------------------------------------ device handles


class DeviceMPO:
    def __init__(self, mpo: MPO, ctx: Context):
        self.ctx = ctx
        self.mpo = mpo
        L = len(mpo)
        nsym = mpo.nsym
        Ws = [np.asfortranarray(w) for w in mpo.W]
        d = [w.shape[1] for w in Ws]
        wl = [w.shape[0] for w in Ws]
        wr = [w.shape[3] for w in Ws]
        self._keep = [Ws]
        if nsym:
            phys = [np.asarray(mpo.qlabels[i], dtype=np.int32).reshape(-1) for i in range(L)]
            self._keep.append(phys)
            pq = _ptr_array(phys, C.c_int)
        else:
            pq = None
        h = C.c_void_p()
        check(lib().dmrg_mpo_upload(ctx.h, L, nsym, _int_arr(d), _int_arr(wl), _int_arr(wr),
                                    _ptr_array(Ws, C.c_double), pq, None, C.byref(h)), ctx.h)
        self.h = h
        self.L, self.nsym, self.d = L, nsym, d

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib().dmrg_mpo_destroy(self.h)
        except Exception:
            pass


class DeviceState:
    """A device-resident MPS plus its environments (``dmrg_state``)."""

    def __init__(self, psi: MPS, dmpo: DeviceMPO):
        self.ctx = dmpo.ctx
        self.dmpo = dmpo
        L = len(psi)
        if len(dmpo.mpo) != L:
            raise ValueError("MPS and MPO lengths differ")
        h = C.c_void_p()
        if psi.tensors is None:
            nsym = dmpo.nsym
            nsec = _int_arr([len(s) for s in psi.sectors])
            qn = [np.asarray([q for q, _ in s], dtype=np.int32).reshape(-1) for s in psi.sectors]
            dims = [np.asarray([dd for _, dd in s], dtype=np.int32) for s in psi.sectors]
            data = [np.ascontiguousarray(b, dtype=float) for b in psi.blocks]
            self._keep = (qn, dims, data)
            check(lib().dmrg_mps_upload_blocks(self.ctx.h, dmpo.h, nsec,
                                               _ptr_array(qn, C.c_int) if nsym else None,
                                               _ptr_array(dims, C.c_int),
                                               _ptr_array(data, C.c_double), psi.oc, C.byref(h)),
                  self.ctx.h)
        else:
            As = [np.asfortranarray(a) for a in psi.tensors]
            ml = _int_arr([a.shape[0] for a in As])
            mr = _int_arr([a.shape[2] for a in As])
            bq = None
            keep = [As]
            if psi.bond_labels is not None and dmpo.nsym:
                lab = [np.asarray(b, dtype=np.int32).reshape(-1) for b in psi.bond_labels]
                keep.append(lab)
                bq = _ptr_array(lab, C.c_int)
            self._keep = keep
            check(lib().dmrg_mps_upload(self.ctx.h, dmpo.h, ml, mr, _ptr_array(As, C.c_double),
                                        bq, psi.oc, C.byref(h)), self.ctx.h)
        self.h = h
        self.L = L

    # -- queries
    @property
    def oc(self):
        v = C.c_int()
        check(lib().dmrg_state_oc(self.h, C.byref(v)), self.ctx.h)
        return v.value

    def bond(self, b):
        n = C.c_int()
        check(lib().dmrg_bond_info(self.h, b, C.byref(n), None, None), self.ctx.h)
        ns = self.dmpo.nsym
        q = (C.c_int * max(n.value * max(ns, 1), 1))()
        dd = (C.c_int * max(n.value, 1))()
        check(lib().dmrg_bond_info(self.h, b, C.byref(n), q, dd), self.ctx.h)
        return [(tuple(q[k * ns:(k + 1) * ns]), dd[k]) for k in range(n.value)]

    def bonds(self):
        """Every bond's sectors [(charges, dim), ...], bond 0 first (one call)."""
        L, ns = self.L, self.dmpo.nsym
        nsec = np.zeros(L + 1, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        check(lib().dmrg_bonds_info(self.h, nsec.ctypes.data_as(ip), None, None), self.ctx.h)
        tot = int(nsec.sum())
        q = np.zeros(max(tot * ns, 1), dtype=np.int32)
        dd = np.zeros(max(tot, 1), dtype=np.int32)
        check(lib().dmrg_bonds_info(self.h, nsec.ctypes.data_as(ip), q.ctypes.data_as(ip),
                                    dd.ctypes.data_as(ip)), self.ctx.h)
        ql, dl = q.tolist(), dd.tolist()
        out, k = [], 0
        for b in range(L + 1):
            out.append([(tuple(ql[(k + j) * ns:(k + j + 1) * ns]), dl[k + j])
                        for j in range(int(nsec[b]))])
            k += int(nsec[b])
        return out

    def all_site_blocks(self):
        """Every site's blocks (one call, one device synchronisation)."""
        sizes = np.zeros(self.L, dtype=np.int64)
        sp = C.POINTER(C.c_int64)
        check(lib().dmrg_mps_download_all_blocks(self.h, None, sizes.ctypes.data_as(sp)),
              self.ctx.h)
        flat = np.empty(max(int(sizes.sum()), 1))
        check(lib().dmrg_mps_download_all_blocks(self.h, flat.ctypes.data_as(C.POINTER(C.c_double)),
                                                 sizes.ctypes.data_as(sp)), self.ctx.h)
        cuts = np.cumsum(sizes)[:-1]
        return [a.copy() for a in np.split(flat[:int(sizes.sum())], cuts)]

    def site_blocks(self, i):
        n = C.c_int64()
        check(lib().dmrg_site_size(self.h, i, C.byref(n)), self.ctx.h)
        out = np.empty(n.value)
        check(lib().dmrg_mps_download_blocks(self.h, i, out.ctypes.data_as(C.POINTER(C.c_double))),
              self.ctx.h)
        return out

    def site_dense(self, i):
        ml, mr = C.c_int(), C.c_int()
        check(lib().dmrg_mps_download(self.h, i, None, C.byref(ml), C.byref(mr)), self.ctx.h)
        out = np.zeros((ml.value, self.dmpo.d[i], mr.value), order="F")
        check(lib().dmrg_mps_download(self.h, i, out.ctypes.data_as(C.POINTER(C.c_double)), None,
                                      None), self.ctx.h)
        return out

    def download_into(self, psi: MPS, blocks=None):
        """Write the device MPS back into ``psi`` (block form when charges are present)."""
        use_blocks = (self.dmpo.nsym > 0) if blocks is None else blocks
        if use_blocks:
            psi.sectors = self.bonds()
            psi.blocks = self.all_site_blocks()
            psi.phys = [list(map(tuple, self.dmpo.mpo.qlabels[i])) if self.dmpo.nsym
                        else [()] * self.dmpo.d[i] for i in range(self.L)]
            psi.tensors = None
            psi.bond_labels = None
        else:
            psi.tensors = [self.site_dense(i) for i in range(self.L)]
            psi.bond_labels = ([[q for q, d in self.bond(b) for _ in range(d)]
                                for b in range(self.L + 1)] if self.dmpo.nsym else None)
            psi.sectors = psi.blocks = None
        psi.oc = self.oc
        psi._dev = self

    # -- checkpoints
    def save(self, path):
        """Checkpoint of the device state in one file (``dmrg_state_save``)."""
        check(lib().dmrg_state_save(self.h, os.fsencode(str(path))), self.ctx.h)

    @classmethod
    def load(cls, path, dmpo: DeviceMPO):
        """The device state of a checkpoint (``dmrg_state_load``); environments are not built."""
        self = cls.__new__(cls)
        self.ctx, self.dmpo, self._keep = dmpo.ctx, dmpo, ()
        h = C.c_void_p()
        check(lib().dmrg_state_load(self.ctx.h, dmpo.h, os.fsencode(str(path)), C.byref(h)),
              self.ctx.h)
        self.h = h
        self.L = len(dmpo.mpo)
        return self

    # -- environments and contractions
    def env_build(self):
        check(lib().dmrg_env_build(self.h, self.dmpo.h), self.ctx.h)

    def lupdate(self, i):
        check(lib().dmrg_lupdate(self.h, self.dmpo.h, i), self.ctx.h)

    def rupdate(self, i):
        check(lib().dmrg_rupdate(self.h, self.dmpo.h, i), self.ctx.h)

    def env(self, i, left):
        dims = (C.c_int * 3)()
        check(lib().dmrg_env_get(self.h, i, 1 if left else 0, None, dims), self.ctx.h)
        out = np.zeros(tuple(dims), order="F")
        check(lib().dmrg_env_get(self.h, i, 1 if left else 0,
                                 out.ctypes.data_as(C.POINTER(C.c_double)), dims), self.ctx.h)
        return out

    def heff(self, iL, psi2, precision="fp64"):
        dims = (C.c_int * 4)()
        check(lib().dmrg_twosite_dims(self.h, self.dmpo.h, iL, dims), self.ctx.h)
        x = np.asfortranarray(psi2, dtype=float)
        if x.shape != tuple(dims):
            raise ValueError(f"two-site vector has shape {x.shape}, expected {tuple(dims)}")
        y = np.zeros(tuple(dims), order="F")
        check(lib().dmrg_heff_apply(self.h, self.dmpo.h, iL, x.ctypes.data_as(C.POINTER(C.c_double)),
                                    y.ctypes.data_as(C.POINTER(C.c_double)),
                                    _lib.PREC[precision]), self.ctx.h)
        return y

    def sweep(self, params: Params):
        st = SweepStats()
        check(lib().dmrg_sweep(self.h, self.dmpo.h, C.byref(params), C.byref(st)), self.ctx.h)
        return st.as_dict()

    def tdvp(self, params: Params, prefactor: float, twosite: bool = True):
        """One call of tdvp_twosite (or tdvp) on the resident state; the environments must be
        built for its current tensors."""
        st = SweepStats()
        check(lib().dmrg_tdvp(self.h, self.dmpo.h, C.byref(params), float(prefactor),
                              1 if twosite else 0, C.byref(st)), self.ctx.h)
        return st.as_dict()

    def sweep3s(self, params: Params, noise: "_lib.Noise"):
        """One single-site sweep with subspace expansion; ``noise.noise`` (alpha) is updated."""
        st = SweepStats()
        check(lib().dmrg_sweep3s(self.h, self.dmpo.h, C.byref(params), C.byref(noise),
                                 C.byref(st)), self.ctx.h)
        d = st.as_dict()
        d["noise"] = noise.noise
        return d

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib().dmrg_state_destroy(self.h)
        except Exception:
            pass


def make_params(maxm=0, minm=2, cutoff=0.0, krylov=2, precision="fp64", svnbond=0,
                degen_rtol=0.0, betatest=1e-10, fp64_final=1, profile=0, goal=0.0, cvgE=True,
                tune=True, graph=False, halfsweep=False):
    p = Params()
    lib().dmrg_params_default(C.byref(p))
    p.maxm, p.minm, p.cutoff = int(maxm), int(minm), float(cutoff)
    p.krylov = int(krylov)
    p.precision = _lib.PREC[precision] if isinstance(precision, str) else int(precision)
    p.svnbond, p.degen_rtol, p.betatest, p.fp64_final = int(svnbond), float(degen_rtol), \
        float(betatest), int(fp64_final)
    p.profile = int(profile)
    p.goal, p.cvgE = float(goal), 1 if cvgE else 0
    p.tune = 1 if tune else 0
    p.graph = 1 if graph else 0
    p.halfsweep = 1 if halfsweep else 0
    return p


# ------------------------------------------------------------------ the drop-in

def dmrg(psi: MPS, mpo: MPO, m=None, maxm=None, minm=2, sweeps=1, cutoff=0.0, silent=True,
         method="twosite", krylov=2, precision="fp64", SvNbond=0, degen_rtol=0.0, goal=0.0,
         cvgE=True, noise=1.0, noise_goal=0.3, noise_incr=0.01, halfsweep=False, ctx=None,
         download=True):
    """DMRG on the GPU: ``dmrg(psi, mpo; m, minm, sweeps, cutoff, method)`` of
    ``algs/DMRG.jl:549-588``. ``method="twosite"`` (default) runs ``dmrg_twosite``;
    ``method="3S"`` runs ``dmrg3S`` (``algs/DMRG.jl:655-671``: single-site steps with subspace
    expansion weighted by ``noise``, adapted by ``alpha_update`` with ``noise_goal`` and
    ``noise_incr``; Krylov dimension ``max(2, krylov)``).
    ``maxm`` is accepted as an alias of ``m``; ``m`` may also be a per-sweep list (a bond-dimension
    ramp). Returns the energy of the last bond step and updates ``psi`` (tensors, ``oc``) in
    place; per-sweep records go to ``psi.sweep_stats``.
    ``goal > 0`` stops after the first sweep whose energy (``cvgE``) or centre entropy changed by
    less than ``goal`` (``dmrgcvg``, ``algs/DMRG.jl:610-652``; the first sweep is compared with
    the starting energy <psi|H|psi>).
    ``halfsweep=True`` makes every sweep one direction only (L-1 bond steps), as the reference's
    ``halfsweep`` does (``algs/DMRG.jl:253``).
    ``download=False`` leaves the result on the device (``psi`` keeps a handle to it)."""
    if method not in ("twosite", "3S"):
        raise ValueError(f"DMRG method ({method}) not defined")
    mm = m if m is not None else (maxm if maxm is not None else 0)
    sched = list(mm) if np.ndim(mm) else [int(mm)] * int(sweeps)
    dmpo = mpo.device(ctx)
    dev = psi._dev if (psi._dev is not None and psi._dev.dmpo is dmpo) else DeviceState(psi, dmpo)
    dev.env_build()
    energy = 0.0
    stats = []
    nz = None
    if method == "3S":
        nz = _lib.Noise()
        lib().dmrg_noise_default(C.byref(nz))
        nz.noise, nz.noise_goal, nz.noise_incr = float(noise), float(noise_goal), float(noise_incr)
    for n, mcur in enumerate(sched):
        p = make_params(mcur, minm, cutoff, krylov, precision, SvNbond, degen_rtol, goal=goal,
                        cvgE=cvgE, halfsweep=halfsweep)
        st = dev.sweep(p) if nz is None else dev.sweep3s(p, nz)
        energy = st["energy"]
        stats.append(st)
        if not silent:
            print(f"Sweep {n + 1} (back and forth): {st['seconds']:.5f} sec")
            print(f"Largest truncation = {st['max_truncerr']}, m = {st['biggest_m']}")
            print(f"Energy at sweep {n + 1} is {energy:.12f}\n")
        if st["converged"]:
            if not silent:
                what = "energy" if cvgE else "entropy"
                print(f"The {what} for DMRG converged to a difference of {st['cvg_check']} "
                      f"after {n + 1} sweeps!\n")
            break
    psi.sweep_stats = stats
    if download:
        dev.download_into(psi)
    else:
        psi._dev = dev
        psi.oc = dev.oc
    return energy


# ------------------------------------------------------------------ time evolution

def _bond_dims(psi: MPS):
    if psi.tensors is not None:
        return [a.shape[2] for a in psi.tensors]
    return [sum(d for _, d in sec) for sec in psi.sectors[1:]]


def _tdvp(psi, mpo, m, minm, cutoff, origj, r, prefactor, twosite, precision, ctx, download):
    pre = complex(prefactor)
    if pre.imag != 0.0:
        raise ValueError("complex prefactor: real-time evolution needs complex tensors, which "
                         "this engine does not hold (a real prefactor evolves in imaginary time)")
    mm = max(_bond_dims(psi)) if m is None else int(m)
    dmpo = mpo.device(ctx)
    dev = psi._dev if (psi._dev is not None and psi._dev.dmpo is dmpo) else DeviceState(psi, dmpo)
    L = len(psi)
    if not origj and 0 < dev.oc < L - 1:
        raise ValueError("origj=false from an interior centre (leftward first) is not available")
    dev.env_build()    # makeEnv(psi, psi, mpo) at the start of every call (algs/time.jl:214,291)
    rec = dev.tdvp(make_params(mm, minm, cutoff, r, precision), pre.real, twosite)
    psi.sweep_stats = [rec]
    if download:
        dev.download_into(psi)
    else:
        psi._dev = dev
        psi.oc = dev.oc
    return rec["energy"]


def tdvp_twosite(psi: MPS, mpo: MPO, m=None, minm=2, cutoff=0.0, origj=True, r=2, prefactor=1.0,
                 precision="fp64", ctx=None, download=True):
    """``tdvp_twosite(psi, mpo; m, minm, cutoff, origj, r, prefactor)`` (``algs/time.jl:288-363``)
    on the GPU: one half sweep of two-site TDVP steps, each applying exp(tau H) (tau =
    prefactor / (L-1) / 2) by a Krylov exponential with ``r`` vectors to the two-site tensor and
    then to the site left as centre, with a truncated move between. ``m`` defaults to the largest
    bond dimension of ``psi``. Real prefactors only (imaginary-time evolution). Returns En of the
    last Krylov call; ``psi`` is updated in place."""
    return _tdvp(psi, mpo, m, minm, cutoff, origj, r, prefactor, True, precision, ctx, download)


def tdvp(psi: MPS, mpo: MPO, m=None, minm=2, cutoff=0.0, origj=True, r=2, prefactor=1.0,
         precision="fp64", ctx=None, download=True):
    """``tdvp(psi, mpo; m, minm, cutoff, origj, r, prefactor)`` (``algs/time.jl:211-286``) on the
    GPU: single-site TDVP steps (the site by exp(tau H1), tau = prefactor / L / 2, then the bond
    matrix by exp(tau H0) through the zero-site Heff). One call is one half sweep of L-1 steps
    (the reference's L-th step would read past the chain's end). Real prefactors only."""
    return _tdvp(psi, mpo, m, minm, cutoff, origj, r, prefactor, False, precision, ctx, download)


# ------------------------------------------------------------------ measurements

def _measure_state(psi: MPS, ctx=None):
    """The device state of ``psi``: its resident handle, or an upload against an identity MPO
    that carries the state's physical charges (block form) or none (dense tensors)."""
    if psi._dev is not None and (ctx is None or psi._dev.ctx is ctx):
        return psi._dev
    L = len(psi)
    if psi.tensors is None:
        d = [len(p) for p in psi.phys]
        ql = [list(map(tuple, p)) for p in psi.phys] if psi.phys and len(psi.phys[0][0]) else None
    else:
        d = [a.shape[1] for a in psi.tensors]
        ql = None
    ident = MPO([np.eye(di).reshape(1, di, di, 1) for di in d], ql)
    dev = DeviceState(psi, ident.device(ctx))
    psi._dev = dev
    return dev


def mpo_product(*Hs: MPO) -> MPO:
    """The MPO of the operator product H1 H2 ... Hn, Hn acting on the ket first (the order of
    ``expect(psi, H1, ..., Hn)``, ``lib/MPO_MPS/expect.jl:19-45``): per site
    W[(w1,w2), s, t, (w1',w2')] = sum_u W1[w1, u, t, w1'] W2[w2, s, u, w2'] (s ket, t bra)."""
    out = Hs[0]
    for H in Hs[1:]:
        if len(H) != len(out):
            raise ValueError("MPOs of different lengths")
        Ws = []
        for A, B in zip(out.W, H.W):
            W = np.einsum("auth,bsuk->absthk", A, B)
            a, b, d1, d2, h, k = W.shape
            Ws.append(W.reshape(a * b, d1, d2, h * k))
        out = MPO(_prune_bonds(Ws), out.qlabels)
    return out


def _prune_bonds(Ws):
    """Drops MPO bond states with no weight on one side (an all-zero column of the left site or
    row of the right site): they contribute nothing, and the charge labels of the makeqMPO rule
    are defined only for states that carry weight."""
    Ws = [w.copy() for w in Ws]
    changed = True
    while changed:
        changed = False
        for i in range(len(Ws) - 1):
            keep = np.any(Ws[i] != 0, axis=(0, 1, 2)) & np.any(Ws[i + 1] != 0, axis=(1, 2, 3))
            if not keep.any():
                keep[0] = True          # the zero operator: keep one state
            if not keep.all():
                Ws[i] = Ws[i][..., keep]
                Ws[i + 1] = Ws[i + 1][keep]
                changed = True
    return Ws


def expect(psi: MPS, *H: MPO, ctx=None):
    """``expect(psi, H...)`` (``lib/MPO_MPS/expect.jl:47-56``): <psi|H1 H2 ... Hn|psi> on the
    device, not normalised (as in the reference); several MPOs are multiplied on the host first
    (:func:`mpo_product`). The MPOs may differ from the one the state was solved with but must
    share its sites and physical charges. The state's centre is not moved."""
    if not H:
        raise ValueError("expect needs at least one MPO")
    H = H[0] if len(H) == 1 else mpo_product(*H)
    dev = psi._dev if psi._dev is not None and (ctx is None or psi._dev.ctx is ctx) else None
    dh = H.device(dev.ctx if dev is not None else ctx)
    if dev is None:
        dev = DeviceState(psi, dh)
        psi._dev = dev
    v = C.c_double()
    check(lib().dmrg_expect(dev.h, dh.h, C.byref(v)), dev.ctx.h)
    return v.value


def correlationmatrix(psi: MPS, Cc, Ca, trail=None, ctx=None):
    """``correlationmatrix(psi, Cc, Ca; trail)`` (``lib/MPO_MPS/correlationmatrix.jl:21-83``):
    ``rho[i,j] = <psi|(Cc F)_i F_{i+1}..F_{j-1} Ca_j|psi> / <psi|psi>`` for i < j, mirrored below
    the diagonal, ``rho[i,i] = <psi|(Cc Ca)_i|psi> / <psi|psi>``; operators are d x d arrays
    O[bra, ket]. Runs on the device and leaves the centre where it is (the reference moves it to
    each site; the values agree for a normalised state)."""
    dev = _measure_state(psi, ctx)
    ops = [np.asfortranarray(np.asarray(o, dtype=float)) for o in (Cc, Ca)]
    d = ops[0].shape[0]
    for o in ops:
        if o.shape != (d, d):
            raise ValueError("operators must be square and of one size")
    F = None
    if trail is not None and np.size(trail):
        F = np.asfortranarray(np.asarray(trail, dtype=float))
        if F.shape != (d, d):
            raise ValueError("trail must have the operators' size")
    L = dev.L
    rho = np.zeros((L, L), order="F")
    dp = C.POINTER(C.c_double)
    check(lib().dmrg_correlationmatrix(dev.h, d, ops[0].ctypes.data_as(dp),
                                       ops[1].ctypes.data_as(dp),
                                       F.ctypes.data_as(dp) if F is not None else None,
                                       rho.ctypes.data_as(dp)), dev.ctx.h)
    return rho


def correlation(psi: MPS, *ops, sites=None, trail=(), ctx=None):
    """``correlation(psi, ops...; sites, trail)`` (``lib/MPO_MPS/correlation.jl:73-237``) on the
    device: ``omega[i_1, ..., i_n] = <psi|O(1) ... O(L)|psi>``, not normalised, with operator g at
    its i_g-th position and, at each site, the product A_1 A_2 ... A_n of what the operators put
    there (operator g's factor on its sites, its trail on every site left of it, the identity
    elsewhere). An operator is a d x d array O[bra, ket] or a list of them on consecutive sites.
    ``sites`` (1-based, as in the reference): one sequence of start sites per operator, default
    ``1:L``; the last ``len - 1`` entries of a multi-site operator's sequence are not used as
    starts. ``trail``: a d x d array for every operator, or one per operator (cycled), or
    ``()``. Equal to the reference's result when every sequence is ``1:k``, for one or two
    operators; with three or more the reference reuses stale right environments across position
    combinations, and this returns the definition above."""
    if not ops:
        raise ValueError("correlation needs at least one operator")
    dev = _measure_state(psi, ctx)
    L = dev.L
    factors, lens = [], []
    for o in ops:
        fs = list(o) if isinstance(o, (list, tuple)) else [o]
        lens.append(len(fs))
        factors.extend(np.asarray(f, dtype=float) for f in fs)
    d = factors[0].shape[0]
    for f in factors:
        if f.shape != (d, d):
            raise ValueError("operators must be square and of one size")
    n = len(lens)
    if sites is None:
        sites = [range(1, L + 1)] * n
    if len(sites) != n:
        raise ValueError("one sequence of sites per operator")
    starts = [[int(x) - 1 for x in sq] for sq in sites]
    base = [len(sq) - (k - 1) for sq, k in zip(starts, lens)]
    if min(base) < 1:
        raise ValueError("an operator has no start site")
    trails = None
    if trail is not None and not (isinstance(trail, (list, tuple)) and len(trail) == 0):
        tl = list(trail) if isinstance(trail, (list, tuple)) else [trail]
        trails = np.concatenate([np.asarray(tl[g % len(tl)], dtype=float).reshape(d, d)
                                 .ravel(order="F") for g in range(n)])
    opbuf = np.concatenate([f.ravel(order="F") for f in factors])
    lenbuf = np.asarray(lens, dtype=np.int32)
    nsbuf = np.asarray([len(sq) for sq in starts], dtype=np.int32)
    stbuf = np.asarray([x for sq in starts for x in sq], dtype=np.int32)
    omega = np.zeros(base, order="F")
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    check(lib().dmrg_correlation(dev.h, d, n, lenbuf.ctypes.data_as(ip), opbuf.ctypes.data_as(dp),
                                 nsbuf.ctypes.data_as(ip), stbuf.ctypes.data_as(ip),
                                 trails.ctypes.data_as(dp) if trails is not None else None,
                                 omega.ctypes.data_as(dp)), dev.ctx.h)
    return omega


# ------------------------------------------------------------------ checkpoints

def largeMPS(psi: MPS, path, mpo: MPO = None, ctx=None):
    """Writes ``psi`` to the checkpoint file ``path`` and returns the path: the persistence of
    ``largeMPS(psi)`` (``lib/MPS/largeMPS.jl:19-33``) in one file rather than one per tensor. The
    device state ``psi`` holds is written directly; otherwise ``psi`` is uploaded for ``mpo`` (or,
    without one, for an identity MPO carrying its physical charges)."""
    if psi._dev is not None:
        dev = psi._dev
    elif mpo is not None:
        dev = DeviceState(psi, mpo.device(ctx))
        psi._dev = dev
    else:
        dev = _measure_state(psi, ctx)
    dev.save(path)
    return path


def loadMPS(path, mpo: MPO, ctx=None):
    """``loadMPS`` (``lib/MPS/largeMPS.jl:60-79``): the MPS of a checkpoint, resident on the device
    for ``mpo`` (same sites and charges as when it was written) and downloaded into the returned
    object. A following ``dmrg(psi, mpo, ...)`` rebuilds the environments and continues exactly
    as an uninterrupted run would."""
    dev = DeviceState.load(path, mpo.device(ctx))
    psi = MPS()
    dev.download_into(psi)
    return psi


class Env:
    """Device-backed environment list (``environment{W}``, ``lib/types.jl:113-115``):
    ``Lenv[i]`` downloads the dense-equivalent [m, w, m] tensor of site i."""

    def __init__(self, dev: DeviceState, left: bool):
        self.dev, self.left = dev, left

    def __getitem__(self, i):
        return self.dev.env(i, self.left)

    def __len__(self):
        return self.dev.L


def makeEnv(psi: MPS, mpo: MPO, ctx=None):
    """``makeEnv(psi, mpo)`` (``lib/Env/makeEnv.jl:196-221,244-246``): returns ``(Lenv, Renv)``
    built on the device for the centre ``psi.oc``."""
    dmpo = mpo.device(ctx)
    dev = psi._dev if (psi._dev is not None and psi._dev.dmpo is dmpo) else DeviceState(psi, dmpo)
    psi._dev = dev
    dev.env_build()
    return Env(dev, True), Env(dev, False)


def _env_step(left, env, dual, psi, W, ctx=None):
    """One dense environment step on the device (``dmrg_env_step``)."""
    ctx = ctx or default_context()
    A = np.asfortranarray(np.asarray(psi, dtype=float))
    B = np.asfortranarray(np.asarray(dual, dtype=float)) if dual is not None else A
    Wf = np.asfortranarray(np.asarray(W, dtype=float))
    E = np.asfortranarray(np.asarray(env, dtype=float))
    if A.ndim != 3 or B.shape != A.shape or Wf.ndim != 4 or E.ndim != 3:
        raise ValueError("env step: environment [m,w,m], sites [ml,d,mr], MPO [wl,d,d,wr]")
    ml, d, mr = A.shape
    wl, wr = Wf.shape[0], Wf.shape[3]
    if Wf.shape[1:3] != (d, d):
        raise ValueError("MPO physical dimensions differ from the site's")
    want = (ml, wl, ml) if left else (mr, wr, mr)
    if E.shape != want:
        raise ValueError(f"environment has shape {E.shape}, expected {want}")
    out = np.zeros((mr, wr, mr) if left else (ml, wl, ml), order="F")
    dp = C.POINTER(C.c_double)
    check(lib().dmrg_env_step(ctx.h, 1 if left else 0, ml, d, mr, wl, wr, E.ctypes.data_as(dp),
                              B.ctypes.data_as(dp), A.ctypes.data_as(dp), Wf.ctypes.data_as(dp),
                              out.ctypes.data_as(dp)), ctx.h)
    return out


def Lupdate(*args, ctx=None):
    """Both forms of the reference's left update (``lib/MPO_MPS/Lupdate.jl:17-37``):

    * ``Lupdate(Lenv, dualpsi, psi, mpo)`` with dense tensors returns the next left environment
      ``L'[a',w',b'] = conj(dualpsi[a,t,a']) L[a,w,b] W[w,s,t,w'] psi[b,s,b']``, computed on the
      device;
    * ``Lupdate(i, Lenv, psi, mpo)`` (the reference's ``Lupdate!``) updates the device-resident
      environment list of :func:`makeEnv`: ``Lenv[i+1]`` from ``Lenv[i]`` and the state's site i.
    """
    if isinstance(args[0], (int, np.integer)):
        args[1].dev.lupdate(int(args[0]))
        return None
    L, dual, psi, W = args
    return _env_step(True, L, dual, psi, W, ctx)


def Rupdate(*args, ctx=None):
    """Both forms of the reference's right update (``lib/MPO_MPS/Rupdate.jl:17-37``):
    ``Rupdate(Renv, dualpsi, psi, mpo)`` returns ``R[b,w,a] = psi[b,s,b'] W[w,s,t,w']
    conj(dualpsi[a,t,a']) R'[b',w',a']``; ``Rupdate(i, Renv, psi, mpo)`` (``Rupdate!``) updates
    ``Renv[i-1]`` of a device-resident list."""
    if isinstance(args[0], (int, np.integer)):
        args[1].dev.rupdate(int(args[0]))
        return None
    R, dual, psi, W = args
    return _env_step(False, R, dual, psi, W, ctx)
