"""Writes tests/golden/config_parity.json: the oracle's converged invariants on the benchmark
configurations at a capped bond dimension, for the device parity tests (test infrastructure).

Run from the repository root: ``python tests/golden/make_config_fixtures.py [name ...]``.
Every case starts from a deterministic product state and a deterministic MPO, so the device
test rebuilds the identical input. Each runs the configuration's maxm schedule (capped), then
continues at the cap until the energy of a sweep moved by less than 1e-10 (dmrgcvg's goal test),
with Lanczos of Krylov dimension 8 and full re-orthogonalisation (near-exact bond solves, so the
runs converge in a few sweeps). Cases:
  * heisenberg_l100_u1_cap128: spin-1/2 Heisenberg chain L=100, U(1) (2Sz), Neel start
    (test/dmrg_test.jl:55-58), the 64 -> 1024 maxm ramp of 12 sweeps capped at 128, cutoff 1e-10;
  * hubbard_l32_u1xu1_m256: Hubbard chain L=32, t=1, U=4, mu=0, (N, 2Sz) charges, half-filling
    start of test/dmrg_test.jl:62-75, maxm 256, cutoff 1e-10;
  * cylinder_4x16_u1_m256: Heisenberg on the 4x16 open cylinder (periodic in W=4, snake order),
    U(1), Neel start in snake order, maxm 256, cutoff 1e-9.
The comparison is made at convergence on purpose. The density-matrix eigenvalues at the
truncation cut are ~1e-11 and are resolved only to ~1e-15 absolute by any FP64 eigensolver, so on
a trajectory that is still moving, two correct implementations occasionally keep different states
at a near-tie and their intermediate energies part at the 1e-7 level; both still converge to the
same fixed point, where the energy (1e-10), truncation error and entropy (1e-8) are compared.
Weights equal to 1e-6 relative (SU(2) multiplets spread over several charge sectors) are kept
or dropped together (degen_rtol).
"""
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import dmrg as od, models as om  # noqa: E402

OUT = Path(__file__).resolve().parent / "config_parity.json"
SPIN = [(1,), (-1,)]
HUB = [(0, 0), (1, 1), (1, -1), (2, 0)]
C2_RAMP = [64, 82, 105, 135, 173, 222, 284, 364, 467, 598, 766, 1024]

CASES = {
    "heisenberg_l100_u1_cap128": dict(model="heisenberg", L=100,
                                      schedule=[min(m, 128) for m in C2_RAMP] + [128] * 28,
                                      cutoff=1e-10, degen_rtol=1e-6, krylov=8, goal=1e-10),
    "hubbard_l32_u1xu1_m256": dict(model="hubbard", L=32, schedule=[256] * 30, cutoff=1e-10,
                                   degen_rtol=1e-6, mu=0.0, U=4.0, t=1.0, krylov=8, goal=1e-10),
    "cylinder_4x16_u1_m256": dict(model="cylinder", W=4, Lx=16, L=64, schedule=[256] * 30,
                                  cutoff=1e-9, degen_rtol=1e-6, krylov=8, goal=1e-10),
}


def inputs(case):
    if case["model"] == "heisenberg":
        L = case["L"]
        q = [SPIN] * L
        return om.to_qmps(om.neel_mps(L), q), om.to_qmpo(om.make_mpo([om.heisenberg_bulk()] * L, 2), q)
    if case["model"] == "hubbard":
        L = case["L"]
        q = [HUB] * L
        bulk = om.hubbard_bulk(t=case["t"], mu=case["mu"], U=case["U"])
        return (om.to_qmps(om.hubbard_half_filling_mps(L), q),
                om.to_qmpo(om.make_mpo([bulk] * L, 4), q))
    L = case["L"]
    q = [SPIN] * L
    mpo = om.prune_mpo(om.make_mpo(om.cylinder_heisenberg_bulks(case["W"], case["Lx"]), 2))
    return om.to_qmps(om.neel_mps(L), q), om.to_qmpo(mpo, q)


def run(name):
    case = CASES[name]
    psi, mpo = inputs(case)
    t0 = time.perf_counter()
    E, info = od.dmrg(psi, mpo, m=max(case["schedule"]), sweeps=len(case["schedule"]),
                      cutoff=case["cutoff"], krylov=case["krylov"], trunc="rho",
                      degen_rtol=case["degen_rtol"], maxm_schedule=case["schedule"],
                      goal=case["goal"])
    recs = [{k: r[k] for k in ("energy", "maxtrunc", "entropy", "biggestm", "maxm")}
            for r in info["sweeps"]]
    return {"case": case, "sweeps": recs, "energy": E, "oracle_seconds": time.perf_counter() - t0}


def main(names):
    for n in names or list(CASES):
        rec = run(n)
        data = json.loads(OUT.read_text()) if OUT.exists() else {}
        data[n] = rec
        OUT.write_text(json.dumps(data, indent=1, sort_keys=True))
        print(n, rec["energy"], len(rec["sweeps"]), f"{rec['oracle_seconds']:.1f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
