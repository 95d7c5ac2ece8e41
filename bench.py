#!/usr/bin/env python3
"""Two-site DMRG sweep benchmark on B200 (one process per GPU; N GPUs run independent replicas).

Workload (the headline configuration): spin-1/2 Heisenberg chain, L = 100, J = 1, open ends,
U(1) block-sparse (Sz_total = 0), MPO bond dimension 5, Neel product start, cutoff 1e-10,
maxm ramped 64 -> 1024 over 12 sweeps (64, 82, 105, 135, 173, 222, 284, 364, 467, 598, 766, 1024).
The first 11 ramp sweeps prepare the state (untimed); a "step" is one full sweep (2(L-1) two-site
bond steps with their environment updates) at maxm = 1024. W warm-up steps, then K timed steps.
The resident MPS + environments are smaller than the 126 MB L2, so L2 is flushed (a 256 MB
device write, outside the device-timed region) before every timed sweep.

Reported: value = sweeps/s over all ranks (device-timed, state resident in HBM); e2e = the same
through the public ``dmrg(psi, mpo; m, sweeps=1)`` call with the MPS in host memory (upload,
environment build, sweep, download inside the timed region); roofline of the dominant kernel
(the grouped FP64 GEMM) against the FP64 GEMM peak measured here with cuBLAS; and the CPU oracle
timed on the device's own state (the oracle's sweep() on the host cores).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
RAMP = [64, 82, 105, 135, 173, 222, 284, 364, 467, 598, 766, 1024]
L_CHAIN = 100
CUTOFF = 1e-10
METRIC = "sweep s & Heff TFLOP/s, chosen vs plain FP64 at |dE|<=1e-8; solves/s, p99 latency"


def load_pkg():
    if "dmrjtensor_b200" in sys.modules:
        return sys.modules["dmrjtensor_b200"]
    pkg_dir = ROOT / "dmrjtensor.jl_b200"
    spec = importlib.util.spec_from_file_location(
        "dmrjtensor_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dmrjtensor_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------ clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "samples": len(rows), "reasons": sorted(reasons)}


# ------------------------------------------------------------------ workload

def ramp_schedule(nsweeps):
    """maxm of the untimed ramp sweeps: the whole 64 -> 766 ramp by default, or nsweeps of its
    values spread over it (first and last kept) for short profiling runs."""
    full = RAMP[:-1]
    if nsweeps is None or nsweeps >= len(full):
        return full
    if nsweeps <= 1:
        return full[-1:]
    return [full[round(i * (len(full) - 1) / (nsweeps - 1))] for i in range(nsweeps)]


def nvtx(op, name=None):
    try:
        import torch
        if op == "push":
            torch.cuda.nvtx.range_push(name)
        else:
            torch.cuda.nvtx.range_pop()
    except Exception:
        pass


def build_workload(pkg):
    mpo = pkg.makeMPO(pkg.heisenbergMPO, 2, L_CHAIN).with_qn(pkg.SPIN_QN)
    psi = pkg.neelMPS(L_CHAIN)
    return mpo, psi


def params(pkg, m, args, profile=0, precision=None, tune=True):
    return pkg.make_params(maxm=m, minm=2, cutoff=CUTOFF, krylov=args.krylov,
                           precision=precision or args.precision, profile=profile, tune=tune)


def graph_report(pkg, ctx, dev, mfin, args, flush):
    """The Lanczos step as one CUDA graph per bond step against plain launches: the headline state
    (2-vector Krylov step) and the dense L=20 chain of the benchmark's small configuration (maxm
    100, Krylov 8, after its 10 sweeps), device time per sweep (best of 3) in each mode."""
    out = {}
    for name, tune_graph in (("plain_launches", False), ("graph", True)):
        ms = []
        for _ in range(3):
            flush()
            st = dev.sweep(pkg.make_params(maxm=mfin, minm=2, cutoff=CUTOFF, krylov=args.krylov,
                                           precision=args.precision, graph=tune_graph))
            ms.append(st["seconds"] * 1e3)
        out.setdefault("heisenberg_l100_u1", {})[name + "_ms"] = min(ms)
    L = 20
    mpo = pkg.makeMPO(pkg.heisenbergMPO, 2, L)
    small = pkg.DeviceState(pkg.randMPS(2, L, 10, seed=20), mpo.device(ctx))
    small.env_build()
    for _ in range(10):
        small.sweep(pkg.make_params(maxm=100, cutoff=1e-12, krylov=8))
    for name, g in (("plain_launches", False), ("graph", True)):
        ms = []
        for _ in range(3):
            st = small.sweep(pkg.make_params(maxm=100, cutoff=1e-12, krylov=8, graph=g))
            ms.append(st["seconds"] * 1e3)
        out.setdefault("heisenberg_l20_dense_krylov8", {})[name + "_ms"] = min(ms)
    for v in out.values():
        v["speedup"] = v["plain_launches_ms"] / v["graph_ms"]
    return out


def autotune_report(pkg, ctx, dev, mfin, args, flush):
    """Tile autotuner on the resident state: profiled sweeps with the tuned tile shapes and with
    fixed 64 x 64 tiles (the numbers are identical; the GEMM device time and the sweep time are
    compared), plus the tuner's table size."""
    rec = {}
    for name, tune in (("fixed_64x64", False), ("tuned", True)):
        ms, gs, en = [], [], []
        for _ in range(3):
            flush()
            st = dev.sweep(params(pkg, mfin, args, profile=1, tune=tune))
            ms.append(st["seconds"] * 1e3)
            gs.append(st["gemm_seconds"] * 1e3)
            en.append(st["energy"])
        rec[name] = {"sweep_ms": min(ms), "heff_gemm_ms": min(gs)}
    sig, decided, small = ctx.tuner()
    rec.update({"signatures": sig, "decided": decided, "won_by_32x32": small,
                "gemm_speedup": rec["fixed_64x64"]["heff_gemm_ms"] / rec["tuned"]["heff_gemm_ms"]})
    return rec


def fp64_gemm_peak(device):
    """cuBLAS DGEMM 8192^3 on this GPU (best of 5): the FP64 tensor-pipe roofline denominator."""
    import torch
    dev = torch.device("cuda", device)
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


class L2Flush:
    """Writes a 256 MB device buffer (twice the 126 MB L2) and waits for it: called between timed
    sweeps, outside their device-timed region, so that no sweep starts with a warm L2 (the
    resident state of the headline workload is smaller than L2)."""

    def __init__(self, device):
        import torch
        self.torch = torch
        self.buf = torch.empty(256 << 20, dtype=torch.uint8, device=torch.device("cuda", device))

    def __call__(self):
        self.buf.fill_(1)
        self.torch.cuda.synchronize(self.buf.device)


def host_block_bytes(psi):
    return int(sum(b.size for b in psi.blocks) * 8)


# ------------------------------------------------------------------ CPU oracle sample

def oracle_qmps(sectors, blocks, phys):
    """The oracle's block tensors A[a(+1), s(+1), b(-1)] of an MPS given in the library's block
    form (bond sectors, per-site flat block data in canonical order, physical charges)."""
    sys.path.insert(0, str(ROOT))
    from oracle import qtensor as oq
    out = []
    for i, data in enumerate(blocks):
        Bl, Br = sectors[i], sectors[i + 1]
        ia = oq.Index([q for q, _ in Bl], [d for _, d in Bl], +1)
        isx = oq.Index(phys[i], [1] * len(phys[i]), +1)
        ib = oq.Index([q for q, _ in Br], [d for _, d in Br], -1)
        rq = {q: k for k, (q, _) in enumerate(Br)}
        T = oq.QTensor([ia, isx, ib], {}, tuple(0 for _ in phys[i][0]))
        off = 0
        for ka, (qa, da) in enumerate(Bl):
            for si, ps in enumerate(phys[i]):
                kb = rq.get(tuple(x + y for x, y in zip(qa, ps)))
                if kb is None:
                    continue
                db = Br[kb][1]
                T.blocks[(ka, si, kb)] = np.asarray(data[off:off + da * db]).reshape(
                    (da, db), order="F").reshape(da, 1, db).copy()
                off += da * db
        out.append(T)
    return out


def oracle_workload():
    """The oracle's copy of the headline workload: Heisenberg L=100, U(1), Neel start."""
    sys.path.insert(0, str(ROOT))
    from oracle import models as om
    q = [[(1,), (-1,)]] * L_CHAIN
    return (om.to_qmps(om.neel_mps(L_CHAIN), q),
            om.to_qmpo(om.make_mpo([om.heisenberg_bulk()] * L_CHAIN, 2), q))


class OracleSweeps:
    """The oracle's own sweep loop (algs/optimizeMPS.jl:790-835 restated in numpy) on a state:
    environments built once, then one ``sweep()`` call per timed step at maxm 1024."""

    def __init__(self, psi, mpo, krylov, oc=0, j=1):
        from oracle import dmrg as od
        self.od = od
        self.psi, self.mpo, self.oc, self.j = psi, mpo, oc, j
        self.Lenv, self.Renv = od.make_env(psi, mpo, oc)
        self.P = od.Params(L_CHAIN, RAMP[-1], 2, CUTOFF, krylov, "rho")

    def sweep(self, maxm=RAMP[-1]):
        self.P.maxm = maxm
        t0 = time.perf_counter()
        self.oc, self.j = self.od.sweep(self.psi, self.mpo, self.Lenv, self.Renv, self.oc, self.j,
                                        self.P)
        return time.perf_counter() - t0


def serving_requests(pkg, nreq, seed=5, rate=20.0):
    """The serving workload: transverse-field Ising chains H = -sum Z Z - h sum X with h ~ U[0.5,
    1.5], L in {16, 32, 64, 128}, maxm in {64, 128, 256, 512}, |+...+> start, Poisson arrival
    gaps at `rate` per second (all from default_rng(seed))."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, nreq)
    hs = rng.uniform(0.5, 1.5, nreq)
    Ls = rng.choice([16, 32, 64, 128], nreq)
    ms = rng.choice([64, 128, 256, 512], nreq)
    reqs = []
    for h, L, m in zip(hs, Ls, ms):
        mpo = pkg.makeMPO(pkg.tfiMPO(h=float(h)), 2, int(L))
        psi = pkg.MPS([np.full((1, 2, 1), 1 / math.sqrt(2)) for _ in range(int(L))], oc=0)
        reqs.append((psi, mpo, int(m)))
    return reqs, gaps


def run_serving(pkg, device, nreq, rate=20.0, slots=16, seed=5, saturate=False, precision="fp64",
                batched=True):
    """Serving workload: requests submitted at their Poisson arrival times (or all at once when
    `saturate`, which measures capacity instead of offered load) to a server with `slots`
    concurrent solves (16: measured capacity flattens there, 35 solves/s with or without shared
    launches, while 8 slots with shared launches lose a quarter) and a 150 GB budget; returns solves/s over the whole run (first submission
    to last completion), the latency percentiles (submit to completion) and how many solves the
    shared Heff launches carried on average."""
    reqs, gaps = serving_requests(pkg, nreq, seed, rate)
    lat = []
    with pkg.Server(device=device, slots=slots, hbm_budget=150 * 10**9, batched=batched) as srv:
        t0 = time.perf_counter()
        tick = []
        arrival = t0
        for (psi, mpo, m), g in zip(reqs, gaps):
            if not saturate:
                arrival += g
                now = time.perf_counter()
                if arrival > now:
                    time.sleep(arrival - now)
            tick.append((srv.submit(psi, mpo, m=m, sweeps=6, cutoff=CUTOFF, precision=precision),
                         time.perf_counter()))
        for t, ts in tick:
            st = srv.poll(t, -1)
            if st["status"] != 2:
                raise RuntimeError(f"served solve failed: {st}")
            lat.append(st["queue_seconds"] + st["run_seconds"])
        t1 = time.perf_counter()
        batches, carried = srv.stats()
    lat.sort()
    pct = lambda q: lat[min(len(lat) - 1, int(math.ceil(q * len(lat))) - 1)]
    return {"workload": "TFI chains, h~U[0.5,1.5], L in {16,32,64,128}, maxm in {64,128,256,512}, "
                        "6 sweeps, cutoff 1e-10, |+...+> start, " +
                        ("all submitted at once (capacity)" if saturate else "Poisson arrivals"),
            "requests": nreq, "arrival_rate_per_s": None if saturate else rate, "slots": slots,
            "precision": precision, "shared_heff_launches": batched,
            "solves_per_s": nreq / (t1 - t0), "p50_latency_s": pct(0.50),
            "p99_latency_s": pct(0.99), "mean_latency_s": statistics.mean(lat),
            "solves_per_shared_launch": (carried / batches) if batches else None}


def run_measurements(pkg, ctx, dev, mpo, energy, cpu=True, m_small=64):
    """``expect(psi, H)``, ``correlationmatrix`` and the two-point ``correlation`` on the device:
    on the resident maxm-1024 state of the sweep workload, and on the same chain after a short
    maxm-64 run where the CPU oracle (dense; centre-moving for the matrix, the reference's loop
    for ``correlation`` over the first 20 sites) finishes in seconds and is timed beside the
    device on identical tensors."""
    Sp, Sm, Sz = pkg.spinOps()[:3]
    psi = pkg.MPS()
    psi._dev = dev
    pkg.expect(psi, mpo, ctx=ctx)                    # untimed warm-up (allocations, descriptors)
    pkg.correlationmatrix(psi, Sz, Sz, ctx=ctx)
    n0 = pkg.kernel_launches()
    t = time.perf_counter()
    E = pkg.expect(psi, mpo, ctx=ctx)
    t_exp = time.perf_counter() - t
    n1 = pkg.kernel_launches()
    t = time.perf_counter()
    rho = pkg.correlationmatrix(psi, Sz, Sz, ctx=ctx)
    t_zz = time.perf_counter() - t
    n2 = pkg.kernel_launches()
    t = time.perf_counter()
    rho_pm = pkg.correlationmatrix(psi, Sp, Sm, ctx=ctx)
    t_pm = time.perf_counter() - t
    n3 = pkg.kernel_launches()
    t = time.perf_counter()
    om_pm = pkg.correlation(psi, Sp, Sm, ctx=ctx)
    t_corr = time.perf_counter() - t
    n4 = pkg.kernel_launches()
    out = {"state": f"heisenberg L={L_CHAIN} U(1), maxm {RAMP[-1]} (resident)",
           "expect_seconds": t_exp, "expect_launches": n1 - n0,
           "expect_rel_diff_vs_sweep_energy": abs(E - energy) / abs(energy),
           "correlationmatrix_zz_seconds": t_zz, "correlationmatrix_pm_seconds": t_pm,
           "correlationmatrix_launches": n2 - n1,
           "zz_max_abs_row_sum": float(np.max(np.abs(rho.sum(axis=1)))),
           "correlation_pm_seconds": t_corr, "correlation_pm_launches": n4 - n3,
           "correlation_pm_max_abs_diff_vs_correlationmatrix":
               float(np.max(np.abs(om_pm - rho_pm)))}
    small = pkg.neelMPS(L_CHAIN)
    pkg.dmrg(small, mpo, m=m_small, sweeps=2, cutoff=CUTOFF, ctx=ctx)
    pkg.correlationmatrix(small, Sz, Sz, ctx=ctx)    # untimed warm-up
    t = time.perf_counter()
    E_s = pkg.expect(small, mpo, ctx=ctx)
    t_exp_s = time.perf_counter() - t
    t = time.perf_counter()
    rho_s = pkg.correlationmatrix(small, Sz, Sz, ctx=ctx)
    t_zz_s = time.perf_counter() - t
    first = range(1, 21)
    t = time.perf_counter()
    om_s = pkg.correlation(small, Sp, Sm, sites=(first, first), ctx=ctx)
    t_corr_s = time.perf_counter() - t
    cmp = {"state": f"heisenberg L={L_CHAIN} U(1) after 2 sweeps at maxm {m_small}",
           "device_expect_seconds": t_exp_s, "device_correlationmatrix_zz_seconds": t_zz_s,
           "device_correlation_pm_20x20_seconds": t_corr_s}
    if cpu:
        from oracle import measure as omeas, models as omod
        dense = [np.array(small[i]) for i in range(L_CHAIN)]
        ompo = omod.make_mpo([omod.heisenberg_bulk()] * L_CHAIN, 2)
        t = time.perf_counter()
        E_o = omeas.expect_value(dense, ompo)
        t_exp_o = time.perf_counter() - t
        t = time.perf_counter()
        rho_o = omeas.correlationmatrix(dense, small.oc, Sz, Sz)
        t_zz_o = time.perf_counter() - t
        t = time.perf_counter()
        om_o = omeas.correlation(dense, (Sp, Sm), sites=[list(range(20))] * 2)
        t_corr_o = time.perf_counter() - t
        cmp.update({"oracle_expect_seconds": t_exp_o, "oracle_correlationmatrix_zz_seconds": t_zz_o,
                    "oracle_correlation_pm_20x20_seconds": t_corr_o,
                    "oracle_cores": cpu_threads(), "abs_dE": abs(E_s - E_o),
                    "max_abs_drho": float(np.max(np.abs(rho_s - rho_o))),
                    "max_abs_domega": float(np.max(np.abs(om_s - om_o)))})
    out["vs_oracle"] = cmp
    return out


def geometric_ramp(m0, m1, n):
    """n maxm values from m0 to m1, geometric, rounded."""
    return [int(round(m0 * (m1 / m0) ** (i / (n - 1)))) for i in range(n)]


# The two large benchmark configurations, full size: the Hubbard chain (N, 2Sz) at half filling
# with maxm up to 2048 over 10 sweeps, and the Heisenberg 4x16 cylinder with maxm up to 4096 over
# 8 sweeps; both from their product starts.
CONFIGS = {
    "c3": {"workload": "hubbard L=32 t=1 U=4 mu=0 U(1)xU(1) (N=32, Sz=0), half-filling product "
                       "start, maxm 64->2048 over 10 sweeps, cutoff 1e-10",
           "schedule": geometric_ramp(64, 2048, 10), "cutoff": 1e-10,
           "forms": ("fp64", "3xtf32")},
    "c4": {"workload": "heisenberg 4x16 open cylinder (periodic W=4, snake order) U(1) Sz=0, Neel "
                       "start, maxm 64->4096 over 8 sweeps, cutoff 1e-9",
           "schedule": geometric_ramp(64, 4096, 8), "cutoff": 1e-9,
           "forms": ("fp64", "3xtf32", "bf16x9")},
}


def config_inputs(pkg, which):
    sys.path.insert(0, str(ROOT))
    from oracle import models as om
    if which == "c3":
        L = 32
        mpo = pkg.makeMPO(lambda i: pkg.hubbardMPO(mu=0.0, HubU=4.0, t=1.0), 4, L)
        return (pkg.MPS([np.array(a) for a in om.hubbard_half_filling_mps(L)], oc=0),
                mpo.with_qn(pkg.HUBBARD_QN))
    return pkg.neelMPS(64), pkg.heisenbergCylinderMPO(4, 16).with_qn(pkg.SPIN_QN)


def config_leg(pkg, ctx, which, fp64_peak, tf32_peak, bf16_peak, tmpdir):
    """One large configuration at full size, plain FP64 and split 3xTF32: (1) the whole sweep
    schedule from the product start in each form (device time, final energies); (2) the same state
    (the plain run's final MPS, checkpointed) swept once more in each form, the second of two
    sweeps timed, with the phase breakdown and Heff/environment TFLOP/s of a profiled sweep."""
    cfg = CONFIGS[which]
    sched, cutoff = cfg["schedule"], cfg["cutoff"]
    psi0, mpo = config_inputs(pkg, which)
    dmpo = mpo.device(ctx)
    ckpt = str(Path(tmpdir) / f"{which}.ckp")
    out = {"workload": cfg["workload"], "schedule": sched}
    forms = cfg["forms"]
    for form in forms:
        dev = pkg.DeviceState(psi0, dmpo)
        dev.env_build()
        st = [dev.sweep(pkg.make_params(maxm=m, minm=2, cutoff=cutoff, precision=form))
              for m in sched]
        out[form] = {"run_seconds": sum(s["seconds"] for s in st),
                     "last_sweep_seconds": st[-1]["seconds"], "energy": st[-1]["energy"],
                     "biggest_m": max(s["biggest_m"] for s in st),
                     "eig_max_n": max(s["eig_max_n"] for s in st),
                     "max_truncerr_last": st[-1]["max_truncerr"]}
        if form == "fp64":
            dev.save(ckpt)
        del dev
    for form in forms[1:]:
        out[f"run_speedup_{form}"] = out["fp64"]["run_seconds"] / out[form]["run_seconds"]
        out[f"run_abs_dE_{form}"] = abs(out["fp64"]["energy"] - out[form]["energy"])
    same = {}
    for form in forms:
        rec = {}
        for rep in range(2):
            dev = pkg.DeviceState.load(ckpt, dmpo)
            dev.env_build()
            if rep == 1:    # a profiler can select exactly this sweep's launches
                nvtx("push", f"{which}_same_state_{form}")
            s = dev.sweep(pkg.make_params(maxm=sched[-1], minm=2, cutoff=cutoff, precision=form))
            if rep == 1:
                nvtx("pop")
            rec = {"sweep_seconds": s["seconds"], "energy": s["energy"],
                   "host_seconds": s["host_seconds"], "wait_seconds": s["wait_seconds"]}
            del dev
        dev = pkg.DeviceState.load(ckpt, dmpo)
        dev.env_build()
        p = dev.sweep(pkg.make_params(maxm=sched[-1], minm=2, cutoff=cutoff, precision=form,
                                      profile=1))
        del dev
        rec["phases_profiled"] = {k: p[k] for k in ("heff_seconds", "env_seconds", "eig_seconds",
                                                     "vec_seconds")}
        rec["heff_tflops"] = p["heff_flops"] / p["heff_seconds"] / 1e12 if p["heff_seconds"] else None
        rec["env_tflops"] = p["env_flops"] / p["env_seconds"] / 1e12 if p["env_seconds"] else None
        rec["heff_gemm_tflops"] = (p["gemm_flops"] / p["gemm_seconds"] / 1e12
                                   if p["gemm_seconds"] else None)
        rec["eig_max_n"] = p["eig_max_n"]
        same[form] = rec
    g64 = same["fp64"]["heff_gemm_tflops"]
    same["roofline"] = {"fp64_heff_gemm": {"achieved": g64, "peak": fp64_peak, "unit": "TFLOP/s",
                                           "frac": g64 / fp64_peak if (g64 and fp64_peak) else None}}
    ceilings = {"3xtf32": (tf32_peak / 3 if tf32_peak else None, "TF32 peak / 3"),
                "bf16x9": (bf16_peak / 9 if bf16_peak else None, "BF16 peak / 9")}
    for form in forms[1:]:
        same[f"speedup_{form}"] = same["fp64"]["sweep_seconds"] / same[form]["sweep_seconds"]
        same[f"abs_dE_{form}"] = abs(same["fp64"]["energy"] - same[form]["energy"])
        g = same[form]["heff_gemm_tflops"]
        ceil, how = ceilings[form]
        same["roofline"][f"{form}_heff_gemm"] = {
            "achieved": g, "peak": ceil, "unit": f"TFLOP/s (algorithmic; ceiling = {how})",
            "frac": g / ceil if (g and ceil) else None}
    out["same_state_sweep"] = same
    return out


def measured_bf16_peak():
    """Dense BF16 TFLOP/s of this pool's B200s (burst), from MEASURED_PEAKS.json when present."""
    f = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(f.read_text())["bf16_tflops"])
    except Exception:
        return 1590.0   # earlier measurement on this pool (fallback)


def tf32_gemm_peak(device):
    """cuBLAS TF32 GEMM (FP32 operands, TF32 tensor cores) 8192^3 on this GPU, best of 5."""
    import torch
    dev = torch.device("cuda", device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device=dev)
    b = torch.randn(n, n, dtype=torch.float32, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def heff_forms(pkg, ctx, m=1024, L=22, reps=5, tf32_peak=None, bf16_peak=None):
    """Heff at the dense-equivalent size of the headline workload at maxm 1024 (dense random MPS,
    bond dimension 1024 either side of the centre bond): device time per application in the plain
    FP64 form and the 3xTF32 / BF16x9 tensor-core forms, algorithmic TFLOP/s of each, and each
    split form's fraction of its algorithmic ceiling (TF32 peak / 3, BF16 peak / 9). The timed
    applications follow a warm-up one with the same plan, as the Lanczos iterations of a bond step
    follow its first: the environments' chunk images are packed by the warm-up and reused."""
    import ctypes as C
    lib = pkg.lib()
    mpo = pkg.makeMPO(pkg.heisenbergMPO, 2, L)
    iL = L // 2 - 1
    psi = pkg.randMPS(2, L, m, seed=1, oc=iL)
    dev = pkg.DeviceState(psi, mpo.device(ctx))
    dev.env_build()
    out = {"workload": f"dense Heisenberg L={L}, random MPS with m={m} at bond {iL + 1} "
                       f"(two-site vector {m}x2x2x{m}); Heff at sites {iL},{iL + 1}"}
    for name, code in (("fp64", 0), ("3xtf32", 1), ("bf16x9", 2)):
        sec, fl = C.c_double(), C.c_double()
        pkg._lib.check(lib.dmrg_test_heff_time(dev.h, dev.dmpo.h, iL, code, reps, C.byref(sec),
                                               C.byref(fl)), ctx.h)
        out["flops_per_apply"] = fl.value
        out[name] = {"seconds": sec.value, "tflops": fl.value / sec.value / 1e12}
    out["speedup_3xtf32"] = out["fp64"]["seconds"] / out["3xtf32"]["seconds"]
    out["speedup_bf16x9"] = out["fp64"]["seconds"] / out["bf16x9"]["seconds"]
    for name, peak, k in (("3xtf32", tf32_peak, 3), ("bf16x9", bf16_peak, 9)):
        if peak:
            out[name]["ceiling_tflops"] = peak / k
            out[name]["frac_of_ceiling"] = out[name]["tflops"] / (peak / k)
    return out


def method_legs(pkg, ctx, dev, args):
    """The 3S sweep (dmrg3S) and TDVP (tdvp_twosite, real prefactor) rows: the device against the
    oracle on the same start (L=100 Heisenberg U(1) from the Neel state, capped bond dimension so
    that the dense-with-charges oracle finishes in seconds), then the device alone on the headline
    state (the ramped maxm-1024 two-site state). Times are device-timed per sweep / per call
    (the oracle's with perf_counter on the host cores)."""
    from oracle import dmrg3s as o3, models as om, tdvp as ot
    L, sp = L_CHAIN, [(1,), (-1,)]
    mpo = pkg.makeMPO(pkg.heisenbergMPO, 2, L).with_qn(pkg.SPIN_QN)
    ompo = om.make_mpo([om.heisenberg_bulk()] * L, 2)
    start = om.neel_mps(L)
    labels = om.mps_bond_labels(start, [sp] * L)
    out = {}
    # 3S at maxm 128, 6 sweeps
    psi = pkg.neelMPS(L)
    pkg.dmrg(psi, mpo, m=128, sweeps=6, cutoff=CUTOFF, method="3S", ctx=ctx)
    t = time.perf_counter()
    e3, recs, _ = o3.dmrg3s(start, ompo, [sp] * L, labels, m=128, sweeps=6, cutoff=CUTOFF)
    t3 = time.perf_counter() - t
    d3 = psi.sweep_stats
    out["dmrg3s_m128_6sweeps"] = {
        "device_seconds_per_sweep": statistics.mean(x["seconds"] for x in d3),
        "oracle_seconds_per_sweep": t3 / 6, "oracle_cores": cpu_threads(),
        "energy_device": d3[-1]["energy"], "energy_oracle": e3,
        "abs_dE": abs(d3[-1]["energy"] - e3),
        "noise_device": d3[-1]["noise"], "noise_oracle": recs[-1]["noise"],
        "biggest_m": d3[-1]["biggest_m"]}
    # tdvp_twosite at maxm 64, 2 calls, prefactor -1 (imaginary time)
    psi = pkg.neelMPS(L)
    dt = []
    for _ in range(2):
        en = pkg.tdvp_twosite(psi, mpo, m=64, cutoff=CUTOFF, prefactor=-1.0, ctx=ctx)
        dt.append(psi.sweep_stats[-1]["seconds"])
    t = time.perf_counter()
    orecs, _ = ot.tdvp(start, ompo, [sp] * L, labels, calls=2, prefactor=-1.0, m=64,
                       cutoff=CUTOFF, twosite=True)
    tt = time.perf_counter() - t
    out["tdvp_twosite_m64_2calls"] = {
        "device_seconds_per_call": statistics.mean(dt), "oracle_seconds_per_call": tt / 2,
        "En_device": en, "En_oracle": orecs[-1][0], "abs_dEn": abs(en - orecs[-1][0])}
    # the headline state: 3S sweeps and TDVP calls at maxm 1024
    p = params(pkg, RAMP[-1], args)
    nz = pkg._lib.Noise()
    pkg.lib().dmrg_noise_default(pkg._lib.C.byref(nz))
    dev.sweep3s(p, nz)
    st3 = [dev.sweep3s(p, nz) for _ in range(max(args.steps, 1))]
    out["dmrg3s_headline_state_maxm1024"] = {
        "seconds_per_sweep": statistics.mean(x["seconds"] for x in st3),
        "energy": st3[-1]["energy"], "biggest_m": st3[-1]["biggest_m"],
        "heff_flops_per_sweep": st3[-1]["heff_flops"], "noise": st3[-1]["noise"]}
    stt = []
    for _ in range(2):
        dev.env_build()
        stt.append(dev.tdvp(p, -0.1, True))
    out["tdvp_twosite_headline_state_maxm1024"] = {
        "seconds_per_call": statistics.mean(x["seconds"] for x in stt),
        "En": stt[-1]["energy"], "biggest_m": stt[-1]["biggest_m"],
        "max_truncerr": stt[-1]["max_truncerr"], "prefactor": -0.1}
    return out


def eig_only(pkg, ctx, n, k, reps=3):
    """One density-matrix eigensolve of an n x n block keeping k vectors through the library's
    kernel hook (dmrg_test_syevt): a synthetic DMRG-like density matrix M M^T with column scales
    exp(-c / 12), seed 7. The case the eigensolver captures use; prints device-visible seconds
    per call and the residual of the returned pairs."""
    import ctypes as C
    rng = np.random.default_rng(7)
    M = rng.standard_normal((n, 2 * n)) * np.exp(-np.arange(2 * n) / 12.0)
    rho = M @ M.T
    dp = C.POINTER(C.c_double)
    times = []
    for _ in range(reps):
        A = np.asfortranarray(rho.copy())
        w = np.zeros(n)
        U = np.zeros((n, k), order="F")
        t0 = time.perf_counter()
        pkg._lib.check(pkg.lib().dmrg_test_syevt(ctx.h, 1, (C.c_int * 1)(n), (C.c_int * 1)(k),
                                                 A.ctypes.data_as(dp), w.ctypes.data_as(dp),
                                                 U.ctypes.data_as(dp)), ctx.h)
        times.append(time.perf_counter() - t0)
    res = float(np.max(np.abs(rho @ U - U * w[:k])) / w[0])
    return {"n": n, "keep": k, "seconds_per_call_host": min(times), "residual": res}


def cpu_threads():
    try:
        import threadpoolctl
        info = threadpoolctl.threadpool_info()
        return max([i.get("num_threads", 1) for i in info] or [os.cpu_count() or 1])
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ arms

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def reduce_max(dist, x):
    """Max of a float over all ranks (the slowest replica sets the whole-job time)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(world, steps, tmax):
    """Whole-job throughput of N independent replicas: N * K sweeps in the slowest rank's time."""
    return world * steps / tmax


def workload_config(args, world):
    """The `config` of both arms' JSON lines."""
    return {"workload": "heisenberg L=100 U(1) Sz=0, maxm 1024 sweep (two-site), after the "
                        "64->1024 ramp", "krylov": args.krylov, "cutoff": CUTOFF,
            "precision": args.precision, "l2": "flushed before every timed sweep (256 MB write)",
            "parallelism": f"replicas x{world}"}


def run_reference(args, world, rank):
    """The CPU arm: the oracle (numpy/scipy restatement of the reference's two-site path; the
    reference itself is Julia and cannot run here) on the host cores. It ramps the same Neel start
    through the same 64 -> 766 maxm schedule (untimed), then times W warm-up and K measured full
    sweeps at maxm 1024, one oracle ``sweep()`` call per step -- the unit the device arm times."""
    if rank != 0:
        return
    n_steps = args.steps_ref if args.steps_ref is not None else args.steps
    n_warm = args.warmup_ref if args.warmup_ref is not None else args.warmup
    psi, mpo = oracle_workload()
    run = OracleSweeps(psi, mpo, args.krylov)
    t_ramp = time.perf_counter()
    for m in ramp_schedule(args.ramp_sweeps):
        run.sweep(m)
    t_ramp = time.perf_counter() - t_ramp
    for _ in range(n_warm):
        run.sweep()
    times = [run.sweep() for _ in range(n_steps)]
    sweep_s = statistics.mean(times)
    cores = cpu_threads()
    value = 1.0 / sweep_s
    desc = (f"oracle sweep() (numpy/scipy, OpenBLAS threads {cores}) on its own ramped state: "
            f"{n_steps} full sweeps at maxm {RAMP[-1]} after the untimed 64->766 ramp")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sweeps/s",
           "n_gpus": args.gpus, "steps": n_steps, "warmup": n_warm,
           "ms_per_step": sweep_s * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args, world),
           "energy": run.P.energy, "ramp_seconds": t_ramp,
           "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": cores, "kind": "port",
                            "sample": desc},
           "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def cpu_baseline_on_state(dev, krylov, nsweeps=2):
    """The oracle timed on the device arm's own resident state (downloaded block by block): the
    same sweep at maxm 1024 on the host cores. Returns the cpu_baseline record and the oracle's
    energy after those sweeps."""
    sectors = [dev.bond(b) for b in range(L_CHAIN + 1)]
    blocks = [dev.site_blocks(i) for i in range(L_CHAIN)]
    phys = [[(1,), (-1,)]] * L_CHAIN
    psi = oracle_qmps(sectors, blocks, phys)
    _, mpo = oracle_workload()
    run = OracleSweeps(psi, mpo, krylov, oc=dev.oc, j=1 if dev.oc == 0 else -1)
    times = [run.sweep() for _ in range(nsweeps)]
    t = statistics.mean(times)
    return ({"value": 1.0 / t, "unit": "sweeps/s", "cores": cpu_threads(), "kind": "port",
             "sample": f"oracle sweep() at maxm {RAMP[-1]} on the device's resident state, "
                       f"{nsweeps} full sweeps timed (mean)", "seconds_per_sweep": t},
            run.P.energy)


def run_ours(args, world, rank, local, dist):
    pkg = load_pkg()
    ctx = pkg.Context(local)
    mpo, psi0 = build_workload(pkg)
    dmpo = mpo.device(ctx)
    dev = pkg.DeviceState(psi0, dmpo)
    dev.env_build()
    t_setup = time.perf_counter()
    for m in ramp_schedule(args.ramp_sweeps):
        dev.sweep(params(pkg, m, args))
    t_setup = time.perf_counter() - t_setup
    mfin = RAMP[-1]
    for _ in range(args.warmup):
        dev.sweep(params(pkg, mfin, args))
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    n0 = pkg.kernel_launches()
    nvtx("push", "timed_sweeps")     # lets a profiler select exactly the timed launches
    t0 = time.perf_counter()
    flush = L2Flush(local)
    stats = []
    for _ in range(args.steps):
        flush()
        stats.append(dev.sweep(params(pkg, mfin, args)))
    wall = time.perf_counter() - t0
    nvtx("pop")
    launches = pkg.kernel_launches() - n0
    clocks = sampler.stop() if rank == 0 else None
    dev_s = sum(s["seconds"] for s in stats)
    tmax = reduce_max(dist, dev_s)
    value = aggregate_value(world, args.steps, tmax)
    sweep_s = dev_s / args.steps
    energy = stats[-1]["energy"]
    # one extra profiled sweep (CUDA events around every phase and every Heff GEMM launch; not
    # part of the timed steps): phase breakdown and per-launch timing of the dominant kernel
    prof = dev.sweep(params(pkg, mfin, args, profile=1))
    tuner = autotune_report(pkg, ctx, dev, mfin, args, flush)
    graphs = graph_report(pkg, ctx, dev, mfin, args, flush)
    heff_flops = prof["heff_flops"]
    heff_sec = prof["heff_seconds"]
    # chosen form on the same resident state: Heff GEMMs as 3xTF32 on the tensor cores (FP64
    # Krylov, eigensolver and environments; FP64 energy of the final Ritz vector)
    chosen = None
    if args.chosen:
        for _ in range(args.warmup):
            dev.sweep(params(pkg, mfin, args, precision="3xtf32"))
        if dist:
            dist.barrier()
        st_c = []
        for _ in range(args.steps):
            flush()
            st_c.append(dev.sweep(params(pkg, mfin, args, precision="3xtf32")))
        tc = reduce_max(dist, sum(x["seconds"] for x in st_c))
        prof_c = dev.sweep(params(pkg, mfin, args, profile=1, precision="3xtf32"))
        chosen = {"form": "3xtf32: Heff GEMMs as three TF32 products on tcgen05 (FP32 accumulate "
                          "in TMEM); Krylov, density matrix, eigensolver, environments FP64; "
                          "sweep energy = FP64 Rayleigh quotient of the final Ritz vector",
                  "value": aggregate_value(world, args.steps, tc), "unit": "sweeps/s",
                  "ms_per_step": tc / args.steps * 1e3,
                  "energy": st_c[-1]["energy"],
                  "abs_dE_vs_plain": abs(st_c[-1]["energy"] - energy),
                  "heff_tflops": (prof_c["heff_flops"] / prof_c["heff_seconds"] / 1e12
                                  if prof_c["heff_seconds"] > 0 else None)}
    cpu = None
    if not args.no_cpu and rank == 0:
        # the oracle on this very state: the same sweeps on the host cores, energies side by side
        cpu, e_oracle = cpu_baseline_on_state(dev, args.krylov, nsweeps=args.cpu_sweeps)
        e_dev = [dev.sweep(params(pkg, mfin, args))["energy"] for _ in range(args.cpu_sweeps)][-1]
        cpu.update({"oracle_energy": e_oracle, "device_energy_same_sweeps": e_dev,
                    "abs_dE_device_vs_oracle": abs(e_dev - e_oracle)})
    sectors = [dev.bond(b) for b in range(L_CHAIN + 1)]
    if args.dump_sectors:
        Path(args.dump_sectors).write_text(json.dumps(
            {"what": "bond sectors (2Sz, dim) after the ramp of the L=100 Heisenberg U(1) workload "
                     "at maxm 1024", "sectors": [[[list(q), d] for q, d in b] for b in sectors]}))
    # e2e through the public API with a host MPS
    e2e = None
    if args.e2e_steps > 0:
        psi_host = pkg.MPS()
        dev.download_into(psi_host)
        psi_host._dev = None
        e2e_times = []
        for _ in range(args.e2e_steps):
            psi_host._dev = None
            t1 = time.perf_counter()
            pkg.dmrg(psi_host, mpo, m=mfin, sweeps=1, cutoff=CUTOFF, krylov=args.krylov,
                     precision=args.precision, ctx=ctx)
            e2e_times.append(time.perf_counter() - t1)
            psi_host._dev = None
        nbytes = host_block_bytes(psi_host)
        e2e = {"value": 1.0 / statistics.mean(e2e_times), "unit": "sweeps/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "seconds_per_step": statistics.mean(e2e_times)}
    meas = (run_measurements(pkg, ctx, dev, mpo, energy, cpu=not args.no_cpu)
            if args.measure else None)
    serving = None
    if args.serve_requests > 0:
        serving = {"poisson_fp64": run_serving(pkg, local, args.serve_requests),
                   "capacity_fp64": run_serving(pkg, local, args.serve_saturate, saturate=True),
                   "capacity_fp64_own_launches": run_serving(pkg, local, args.serve_saturate,
                                                             saturate=True, batched=False),
                   "capacity_3xtf32": run_serving(pkg, local, args.serve_saturate, saturate=True,
                                                  precision="3xtf32")}
    methods = method_legs(pkg, ctx, dev, args) if args.methods else None
    if rank != 0:
        return
    peak = fp64_gemm_peak(local)
    tf32_peak = tf32_gemm_peak(local)
    bf16_peak = measured_bf16_peak()
    heff_large = (heff_forms(pkg, ctx, tf32_peak=tf32_peak, bf16_peak=bf16_peak)
                  if args.chosen else None)
    configs = {}
    if args.configs:
        with tempfile.TemporaryDirectory() as td:
            for which in args.configs.split(","):
                configs[which] = config_leg(pkg, ctx, which, peak, tf32_peak, bf16_peak, td)
    g_ach = prof["gemm_flops"] / prof["gemm_seconds"] / 1e12 if prof["gemm_seconds"] > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "gemm_f64_traffic.json"
    if tfile.exists():
        # DRAM bytes per Heff GEMM launch of this workload, from the committed ncu capture
        traffic = json.loads(tfile.read_text()).get("dram_bytes_per_heff_launch")
    out = {
        "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sweep_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args, world),
        "energy": energy,
        "sweep_seconds": sweep_s,
        "device_bytes_in_use": ctx.memory()[0],
        "heff_tflops": heff_flops / heff_sec / 1e12 if heff_sec > 0 else None,
        "phase_seconds_profiled_sweep": {k: prof[k] for k in
                                         ("seconds", "heff_seconds", "env_seconds",
                                          "eig_seconds", "vec_seconds")},
        "host_seconds_per_step": statistics.mean(s["host_seconds"] for s in stats),
        "host_wait_seconds_per_step": statistics.mean(s["wait_seconds"] for s in stats),
        "eig_max_n": max(s["eig_max_n"] for s in stats),
        "n_matvec_per_sweep": stats[-1]["n_matvec"],
        "setup_seconds_ramp": t_setup,
        "wall_seconds_timed": wall,
        "gpu_launches": launches,
        "roofline": {"bound": "tensor", "kernel": "k_gemm_f64 (grouped FP64 DMMA GEMM)",
                     "achieved": g_ach, "peak": peak, "unit": "TFLOP/s",
                     "frac": (g_ach / peak) if (g_ach and peak) else None, "traffic": traffic,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in "
                                    "MEASURED_PEAKS.json)",
                     "launches": prof["gemm_launches"],
                     "mean_launch_us": prof["gemm_seconds"] / max(prof["gemm_launches"], 1) * 1e6},
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "serving": serving,
        "measurements": meas,
        "chosen": chosen,
        "heff_forms_m1024": heff_large,
        "tf32_gemm_peak_tflops": tf32_peak,
        "autotune": tuner,
        "graph": graphs,
        "configs": configs,
        "methods": methods,
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "3xtf32", "bf16x9"])
    ap.add_argument("--krylov", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--dump-sectors", default=None)
    ap.add_argument("--configs", default="c3,c4",
                    help="large configurations to run at full size, plain and split ('' = none)")
    ap.add_argument("--cpu-sweeps", type=int, default=2,
                    help="oracle sweeps timed on the device state for cpu_baseline")
    ap.add_argument("--steps-ref", type=int, default=None,
                    help="reference arm: timed samples (default: --steps)")
    ap.add_argument("--warmup-ref", type=int, default=None,
                    help="reference arm: warm-up samples (default: --warmup)")
    ap.add_argument("--no-chosen", dest="chosen", action="store_false",
                    help="skip the split-precision (3xTF32) sweeps")
    ap.add_argument("--heff-only", action="store_true",
                    help="only time the plain and split Heff at the m=1024 dense-equivalent size")
    ap.add_argument("--eig-only", default=None, metavar="N,K",
                    help="only one N x N density-matrix eigensolve keeping K vectors (the "
                         "eigensolver captures' case)")
    ap.add_argument("--no-methods", dest="methods", action="store_false",
                    help="skip the 3S and TDVP legs")
    ap.add_argument("--no-measure", dest="measure", action="store_false",
                    help="skip the expect / correlationmatrix measurement")
    ap.add_argument("--serve-requests", type=int, default=200,
                    help="requests of the Poisson serving measurement (0: skip serving)")
    ap.add_argument("--serve-saturate", type=int, default=200,
                    help="requests of the capacity runs (all submitted at once)")
    ap.add_argument("--serve-only", action="store_true",
                    help="only the serving measurements (--serve-requests Poisson arrivals, FP64 "
                         "and 3xTF32, plus the capacity runs)")
    ap.add_argument("--ramp-sweeps", type=int, default=None,
                    help="untimed ramp sweeps before the timed ones (default: the full 11-sweep "
                         "ramp); fewer only for profiler runs")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.serve_only:
            pkg = load_pkg()
            out = {}
            for prec in ("fp64", "3xtf32"):
                out[f"poisson_{prec}"] = run_serving(pkg, local, args.serve_requests,
                                                     precision=prec)
                out[f"capacity_{prec}"] = run_serving(pkg, local, args.serve_saturate,
                                                      saturate=True, precision=prec)
            print(json.dumps({"serving": out}))
        elif args.eig_only:
            n, k = (int(x) for x in args.eig_only.split(","))
            pkg = load_pkg()
            print(json.dumps({"eig_only": eig_only(pkg, pkg.Context(local), n, k)}))
        elif args.heff_only:
            # the plain and split Heff forms alone (the kernel-profiling case)
            pkg = load_pkg()
            print(json.dumps({"heff_forms_m1024": heff_forms(
                pkg, pkg.Context(local), tf32_peak=tf32_gemm_peak(local),
                bf16_peak=measured_bf16_peak())}))
        else:
            run_ours(args, world, rank, local, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
