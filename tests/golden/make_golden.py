"""Regenerate the golden fixtures of the oracle tests from the reference's own
test outputs (run in a checkout that has the reference sources mounted):

  ranf_test.reference            -> ranf_test.json   (RNG known answers)
  work/out.quick-test.reference  -> quick_test.json  (%it/%Favg/%Fmax/%fa records
                                                      of one 4^4 HMC trajectory)
  work/out.test.reference        -> test20.json      (%it/%fa/%mc records of 20
                                                      trajectories, work/input.test)
  work/out.smp.reference         -> smp.json         (%fa record and seed of the SMP
                                                      benchmark, work/input.smp)
  work/out.mpp.reference         -> mpp.json         (%fa and %mc records and seed of
                                                      the MPP benchmark, work/input.mpp)

Usage: python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_ranf(path):
    sections, cur = [], None
    for line in open(path):
        s = line.strip()
        if not s:
            continue
        if s.endswith(":"):
            cur = {"title": s, "records": []}
            sections.append(cur)
            continue
        i, seed, x = s.split()
        cur["records"].append([int(i), int(seed), x])
    return sections


def parse_quick(path):
    out = {}
    for line in open(path):
        s = line.strip()
        if s.startswith("%it"):
            f = s.split()
            out["it"] = {"traj": int(f[1]), "f1": int(f[2]), "f2": int(f[3])}
        elif s.startswith("%Favg") or s.startswith("%Fmax"):
            f = s.split()
            out[f[0][1:]] = {"traj": int(f[1]), "values": [float(v) for v in f[2:6]],
                             "names": ["F_gauge", "F_det", "F_F1", "F_F2"]}
        elif s.startswith("%fa"):
            f = s.split()
            out["fa"] = {"traj": int(f[1]), "e": int(f[2]), "plaq_energy": float(f[3]), "exp_mdh": float(f[4]),
                         "cg_calls": int(f[5]), "cg_it_tot": int(f[6]), "cg_it_max": int(f[7])}
        elif s.startswith("Seed") and re.match(r"Seed\s+\d+$", s) and int(s.split()[1]) != 0:
            out["final_seed"] = int(s.split()[1])
        elif s.startswith("Program"):
            out["program"] = s
    out["input"] = {"lattice": [4, 4, 4, 4], "bc_fermions": [1, 1, 1, -1], "beta": 5.0, "kappa": 0.13,
                    "csw": 2.3327, "h": 0.0, "hmc_model": "C", "hmc_rho": 0.1, "hmc_trajectory_length": 0.2,
                    "hmc_steps": 10, "hmc_m_scale": 3, "start": "cold", "seed": "default", "solver_rest": 1e-5,
                    "solver_maxiter": 1000, "solver_mre_vectors": 7, "force_accept": True}
    return out


def parse_test20(path):
    """The %it, %fa and %mc records (mc.F90) and the final seed of the
    20-trajectory test: 10 force-accepted trajectories, then 10 with the
    Metropolis test."""
    recs, seed = [], None
    for line in open(path):
        f = line.split()
        if not f:
            continue
        if f[0] == "%it":
            recs.append({"traj": int(f[1]), "f1": int(f[2]), "f2": int(f[3])})
        elif f[0] == "%fa":
            recs[-1].update(kind="fa", plaq_energy=float(f[3]), exp_mdh=float(f[4]), accepted=1,
                            cg_calls=int(f[5]), cg_it_tot=int(f[6]), cg_it_max=int(f[7]))
        elif f[0] == "%mc":
            recs[-1].update(kind="mc", plaq_energy=float(f[4]), exp_mdh=float(f[5]), accepted=int(f[6]),
                            cg_calls=int(f[7]), cg_it_tot=int(f[8]), cg_it_max=int(f[9]))
        elif f[0] == "Seed" and len(f) == 2 and int(f[1]) != 0:
            seed = int(f[1])
    return {"source": "work/out.test.reference:39-81 (work/input.test; BQCD 3.0.1, libd3)",
            "records": recs, "final_seed": seed,
            "tolerance": "floats printed with 10 decimals may differ in the last or second-last digit "
                         "(README:235-262)"}


def parse_bench(path, source):
    """The %fa (and %mc) records, final seed and total time of a benchmark
    job (one force-accepted trajectory, then Metropolis ones; CG capped at
    100 iterations)."""
    out = {"source": source, "mc": []}
    for line in open(path):
        f = line.split()
        if not f:
            continue
        if f[0] == "%fa":
            out["fa"] = {"plaq_energy": float(f[3]), "exp_mdh": float(f[4]), "cg_calls": int(f[5]),
                         "cg_it_tot": int(f[6]), "cg_it_max": int(f[7])}
        elif f[0] == "%mc":
            out["mc"].append({"traj": int(f[1]), "plaq_energy": float(f[4]), "exp_mdh": float(f[5]),
                              "accepted": int(f[6]), "cg_calls": int(f[7]), "cg_it_tot": int(f[8]),
                              "cg_it_max": int(f[9])})
        elif f[0] == "Seed" and len(f) == 2 and int(f[1]) != 0:
            out["final_seed"] = int(f[1])
        elif f[0] == "CPU-Time":
            out["cpu_time_s"], out["cpus"] = float(f[1]), int(f[4])
        elif f[0] == "TOTAL" and len(f) >= 3:
            out["total_s"] = float(f[2])
        elif f[0] in ("CG", "MTDAGMT", "D_TOTAL") and len(f) == 7:
            # timing_write bins (timing.F90): calls, seconds, Mflop/s mean/min/max, Gflop/s total
            out.setdefault("timing", {})[f[0]] = {"calls": int(f[1]), "seconds": float(f[2]),
                                                  "gflops_total": float(f[6])}
    return out


def main(root):
    ranf = parse_ranf(os.path.join(root, "ranf_test.reference"))
    with open(os.path.join(HERE, "ranf_test.json"), "w") as f:
        json.dump({"source": "ranf_test.reference (ranf_test.F90:26-93)", "sections": ranf}, f, indent=0)
    quick = parse_quick(os.path.join(root, "work", "out.quick-test.reference"))
    quick["source"] = "work/out.quick-test.reference:39-45,50 (work/input.quick-test)"
    with open(os.path.join(HERE, "quick_test.json"), "w") as f:
        json.dump(quick, f, indent=1)
    for name, lines in (("smp", "39,43,45,58-59,74,90"), ("mpp", "41,45,49,50,63-64,79,95")):
        rec = parse_bench(os.path.join(root, "work", "out.%s.reference" % name),
                          "work/out.%s.reference:%s (work/input.%s)" % (name, lines, name))
        with open(os.path.join(HERE, "%s.json" % name), "w") as f:
            json.dump(rec, f, indent=1)
    t20 = parse_test20(os.path.join(root, "work", "out.test.reference"))
    with open(os.path.join(HERE, "test20.json"), "w") as f:
        json.dump(t20, f, indent=1)
    print("wrote", len(ranf), "ranf sections,", sorted(quick), "and", len(t20["records"]), "trajectories")


if __name__ == "__main__":
    # the reference checkout: first argument, else $BQCD_REFERENCE
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BQCD_REFERENCE")
    if not src:
        sys.exit("usage: make_golden.py <reference checkout>  (or set BQCD_REFERENCE)")
    main(src)
