"""Benchmark of the M^+M CG hot path on B200 (one JSON line on rank 0).

Workload (the 32^3 x 64 configuration): clover-Wilson, c_sw = 1.9192,
kappa = 0.13, antiperiodic in t; links = seeded hot start (BQCD's ranf, default
seed) + conf_relax cooling sweeps until the plaquette reaches 0.55 (one sweep
does it), all generated on the device; b =
ran_gauss_volh(12, b, 1/2, EVEN) (unit-variance complex).  A step is one solve
of M~^+M~ x = b from x = 0 to a true FP64 |r|/|b| < 1e-10:
  value   mixed-precision CG (int16 sloppy fields, FP64 reliable updates), s
  fp64    the all-FP64 CG on the same system (same kernels, FP64 storage)
  e2e     the reference-facing C-ABI call with host arrays in pinned memory:
          links (flipped, as at BQCD's call sites), clover A and A^-1, b and x
          uploaded and x downloaded inside the timed region
Every field is larger than the 126 MB L2 (spinor 201 MB FP64, links 1.2 GB),
so no L2 flush is needed between steps.

--impl reference times the CPU restatement of the reference's CG (OpenMP, all
host threads) on a bounded sample of iterations of the same system.
Multi-GPU (torchrun): independent replicas, one solve per GPU, no collective in
the data path; the step time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "bqcd-r399-quda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "M†M CG time-to-1e-10 at 32^3x64: mixed vs FP64 (1 B200); D-slash HBM GB/s"
KAPPA, CSW, COOL = 0.13, 1.9192, 10
# The 32^3x64 configuration asks for hot-start links smoothed "by 10 steps of
# seeded cooling to plaquette ~0.55".  One sweep of BQCD's conf_relax (a full
# Cabibbo-Marinari minimisation) already takes a hot start to 0.61, and ten
# sweeps reach 0.98, a nearly free field on which kappa = 0.13 is beyond the
# critical hopping parameter (FP64 CG then needs ~30,000 iterations).  The
# benchmark therefore cools until the plaquette first reaches the stated
# value; --cool N forces N sweeps.
PLAQ_TARGET = 0.55


# nominal HBM3e bandwidth of an HGX B200 (8 TB/s on DGX): the second
# denominator beside the measured copy bandwidth
NOMINAL_HBM_GBS = 7700.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.out:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if _has_cuda() else "gloo", timeout=datetime.timedelta(seconds=300),
                                device_id=None)
        pg = dist
    return world, rank, local, pg


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def barrier(pg, local):
    if pg is not None:
        import torch
        if _has_cuda():
            torch.cuda.set_device(local)
        pg.barrier()


def allmax(pg, v, local):
    if pg is None:
        return v
    import torch
    dev = torch.device("cuda", local) if _has_cuda() else torch.device("cpu")
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def lattice_of(args, default):
    return tuple(int(x) for x in (args.lattice or default).split(","))


def start_config(bq, L, device, cool):
    """Hot start, then conf_relax sweeps.  cool < 0: sweep until the plaquette
    (<Re Tr P>/3) first reaches PLAQ_TARGET, at most COOL sweeps."""
    lat = bq.Lattice(L, (1, 1, 1, -1), device=device)
    lat.ranset(0)
    lat.conf_hot()
    sweeps = 0
    if cool >= 0:
        lat.conf_relax(cool)
        sweeps = cool
    else:
        while sweeps < COOL and 1.0 - lat.plaq_energy() < PLAQ_TARGET:
            lat.conf_relax(1)
            sweeps += 1
    lat.sweeps = sweeps
    return lat


def build_system(bq, L, device, seed_skip, cool):
    """start_config, the clover term, one Gaussian right-hand side."""
    lat = start_config(bq, L, device, cool)
    lat.clover_init(CSW * KAPPA)
    lat.ranset(0, seed_skip)
    hb = lat.field()
    lat.field_gauss(hb, 0.5)
    hx = lat.field()
    return lat, hb, hx


# DRAM bytes (read + write) of one k_pass1<int16> launch per output site, from
# one ncu capture at 32x32x32x32 (dram__bytes_read.sum + dram__bytes_write.sum
# = 205.6 + 5.2 MB for 524288 sites); traffic grows with the number of
# sites, so the per-launch figure at another volume is this times volh
TRAFFIC_PER_SITE_INT16 = 402.0


def stencil_bytes_per_site(prec, rec12=True):
    """Algorithmic bytes of one mtil first-half pass (D_oe + Ainv_oo) per odd
    output site: read the input spinor once, 8 links, one clover block, write
    one spinor.  int16 fields carry one 4-byte norm per spinor/clover site.
    FP64 links are read as 12 reals (96 B) when the context holds SU(3)
    links, as every benchmark system here does (the device generators keep
    them unitary), else as 18 reals (144 B)."""
    if prec == 0:
        s, gl, c = 192, (96 if rec12 else 144), 576
    elif prec == 1:
        s, gl, c = 96, 48, 288            # FP32, 12-real links
    else:
        s, gl, c = 52, 24, 148            # int16 + norm, 12-real links
    return 2 * s + 8 * gl + c


def run_ours(args):
    import numpy as np
    import bqcdg as bq

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "32,32,32,64")
    peak, peak_kind = peaks()
    lat, hb, hx = build_system(bq, L, local, 1000003 * rank, args.cool)
    para = bq.HmcPara(kappa=KAPPA, csw=CSW)
    zero = np.zeros((lat.volh, 3, 4), np.complex128)
    plaq = 1.0 - lat.plaq_energy()

    def solve(prec, timek=False):
        lat.field_set(hx, zero)
        return lat.solve_dev(hx, hb, para, precision=prec, tol=args.tol, relative=True, time_kernels=timek)

    # warm-up (untimed): both solvers, builds the sloppy copies
    for _ in range(args.warmup):
        solve(bq.PREC_HALF)
    fp64_warm = solve(bq.PREC_DOUBLE)

    # timed region: K mixed-precision solves
    barrier(pg, local)
    infos = []
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            infos.append(solve(bq.PREC_HALF, timek=True))
        wall = time.perf_counter() - t0
    dev_s = sum(i.seconds for i in infos)
    step_s = allmax(pg, dev_s / args.steps, local)
    ok = all(i.converged for i in infos)

    # FP64 baseline solves (same system, same kernels in FP64)
    fp64 = [solve(bq.PREC_DOUBLE, timek=True) for _ in range(max(1, args.fp64_steps))]
    fp64_s = allmax(pg, sum(i.seconds for i in fp64) / len(fp64), local)

    # roofline of the dominant stencil kernel, from the CUDA events of the timed solves
    st_ms = sum(i.stencil_ms for i in infos) / max(1, sum(i.stencil_launches for i in infos))
    st_bytes = stencil_bytes_per_site(2) * lat.volh
    st_gbs = st_bytes / (st_ms * 1e-3) / 1e9
    f64_ms = sum(i.stencil_ms for i in fp64) / max(1, sum(i.stencil_launches for i in fp64))
    f64_gbs = stencil_bytes_per_site(0, rec12=True) * lat.volh / (f64_ms * 1e-3) / 1e9

    # e2e through the reference-facing call (host arrays, transfers timed)
    e2e = None
    if not args.no_e2e:
        # the host side of BQCD's call: links (flipped), clover A and A^-1, b and
        # the initial guess x, staged in pinned host memory
        import torch
        keep = []

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.complex128, pin_memory=_has_cuda())
            keep.append(t)
            v = t.numpy()
            v[...] = a
            return v

        u_host = pinned(lat.get_gauge(flipped=True))
        a_host, i_host = (pinned(c) for c in lat.get_clover()[:2])
        b_host = pinned(lat.field_get(hb))
        x_host = pinned(np.zeros_like(b_host))
        e2e_t, e2e_ok = [], True
        n_e2e = args.e2e_steps if args.e2e_steps > 0 else args.steps
        for k in range(1 + n_e2e):           # one untimed call, then the timed ones
            x_host[...] = 0.0
            barrier(pg, local)
            t0 = time.perf_counter()
            lat.load_gauge(u_host, flipped=True)
            lat.load_clover_solver(a_host, i_host)      # A even and A^-1 odd: what the solver reads
            x, einfo = lat.solve(x_host, b_host, para, precision=bq.PREC_HALF, tol=args.tol, inplace=True)
            dt = time.perf_counter() - t0
            if k > 0:
                e2e_t.append(allmax(pg, dt, local))
                e2e_ok = e2e_ok and bool(einfo.converged)
        h2d = u_host.nbytes + a_host.nbytes // 2 + i_host.nbytes // 2 + b_host.nbytes + x_host.nbytes
        e2e = {"value": sum(e2e_t) / len(e2e_t), "unit": "s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(x.nbytes), "converged": e2e_ok, "steps": len(e2e_t),
               "min_s": min(e2e_t), "max_s": max(e2e_t)}
        lat.clover_init(CSW * KAPPA)   # all six clover parts again (the lean upload kept two)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(lat, hb, L, fp64[0].niter, args.cpu_seconds)

    if rank == 0:
        it = infos[-1]
        flops_site_iter = 4 * 1824          # 4 clover D-slash applications per M^+M, 1824 flop each
        gflops = flops_site_iter * lat.volh * it.niter / step_s / 1e9
        out = {
            "metric": METRIC,
            "value": round(step_s, 6),
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(step_s * 1e3, 3),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64 (int16/f32 sloppy iterations)",
            "data": "synthetic: device hot start (BQCD ranf, default seed) + %d conf_relax cooling sweep(s) "
                    "(plaquette %.4f), Gaussian b" % (lat.sweeps, plaq),
            "config": solve_config(L, lat.sweeps, plaq, lat.volh, world),
            "mixed": {"time_s": step_s, "iterations": it.niter, "reliable_updates": it.reliable_updates,
                      "true_rel_residual": (it.true_rtr / it.b2) ** 0.5, "converged": ok,
                      "gflops": round(gflops, 1), "wall_s_per_step": wall / args.steps},
            "fp64": {"time_s": fp64_s, "steps": len(fp64), "iterations": fp64[0].niter,
                     "true_rel_residual": (fp64[0].true_rtr / fp64[0].b2) ** 0.5,
                     "dslash_gbs": round(f64_gbs, 1), "dslash_frac": round(f64_gbs / peak, 4),
                     "dslash_frac_nominal": round(f64_gbs / NOMINAL_HBM_GBS, 4),
                     "dslash_bytes_per_site": stencil_bytes_per_site(0, rec12=True),
                     "dslash_kernel": "k_pass1<F64> (12-real SU(3) links)"},
            "speedup_mixed_vs_fp64": round(fp64_s / step_s, 3),
            "roofline": {"bound": "hbm", "achieved": round(st_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(st_gbs / peak, 4), "traffic": int(TRAFFIC_PER_SITE_INT16 * lat.volh),
                         "frac_nominal": round(st_gbs / NOMINAL_HBM_GBS, 4), "nominal_peak": NOMINAL_HBM_GBS,
                         "kernel": "k_pass1<F16> (D_oe + Ainv_oo, int16 fields)",
                         "bytes_per_launch": st_bytes, "avg_launch_ms": round(st_ms, 5), "peak_kind": peak_kind},
            "e2e": e2e,
            "gpu_launches": int(sum(i.kernel_launches for i in infos)),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


def cpu_baseline(lat, hb, L, fp64_iters, seconds):
    """The oracle's FP64 CG (restated cg.F90, OpenMP on all host threads) on a
    bounded sample of iterations of the same system; time-to-solution scaled
    by the FP64 iteration count of the same algorithm."""
    import numpy as np
    from oracle import oracle as O
    g = O.Geom(L, (1, 1, 1, -1))
    u = lat.get_gauge(flipped=True)
    a, ai, b = lat.get_clover()
    bvec = lat.field_get(hb)
    x = np.zeros_like(bvec)
    # one iteration to size the sample
    t0 = time.perf_counter()
    g.cg("mtdagmt", x, bvec, u, (a, ai, b), KAPPA, CSW * KAPPA, 0.0, 0.0, rest=0.0, maxiter=1, log=2)
    t1 = time.perf_counter() - t0
    n = max(2, min(200, int(seconds / max(t1, 1e-6))))
    t0 = time.perf_counter()
    g.cg("mtdagmt", x, bvec, u, (a, ai, b), KAPPA, CSW * KAPPA, 0.0, 0.0, rest=0.0, maxiter=n, log=2)
    dt = time.perf_counter() - t0
    per_iter = dt / n
    return {"value": per_iter * fp64_iters, "unit": "s", "cores": O.threads(), "kind": "port",
            "sample": "%d FP64 CG iterations (cg.F90 restated, M~^+M~ at %s) = %.2f s; %.4f s/iteration x %d "
                      "iterations of the FP64 GPU CG" % (n, "x".join(map(str, L)), dt, per_iter, fp64_iters)}


def solve_config(L, sweeps, plaq, volh, world):
    """The config object of the default line, shared by both arms."""
    return {"workload": "M^+M CG to true |r|/|b|<1e-10, lattice %s, kappa %.4f, c_sw %.4f, bc t -1"
                        % ("x".join(map(str, L)), KAPPA, CSW),
            "lattice": list(L), "volh": volh, "sweeps": sweeps, "plaquette": round(plaq, 6),
            "parallelism": "replicas x%d" % world, "l2": "inputs larger than L2 (no flush)"}


def run_reference(args):
    """The reference's CG path on the host cores: the oracle's FP64 CG (a C
    restatement of cg.F90 over mtdagmt and the D21/clover routines, OpenMP on
    all host threads) on the same system as the GPU arm, built on the host by
    the same generators.  One full solve from x = 0 to |r|/|b| < 1e-10 is
    timed, and its true residual recomputed with the oracle's operator: that
    solve is the line's value.  The K timed steps (after W warm-up ones) are
    bounded samples of the same CG, each a fixed number of iterations scaled
    to the measured iteration count; they are reported beside the value as
    a check of its per-iteration cost.  Under torchrun only rank 0 works."""
    import numpy as np
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    L = lattice_of(args, "32,32,32,64")
    g = O.Geom(L, (1, 1, 1, -1))
    O.ranset(0)
    u = g.hot()
    sweeps = 0
    if args.cool >= 0:
        g.relax(u, args.cool)
        sweeps = args.cool
    else:
        while sweeps < COOL and 1.0 - g.sg(u) / (6.0 * 2 * g.volh) < PLAQ_TARGET:
            g.relax(u, 1)
            sweeps += 1
    plaq = 1.0 - g.sg(u) / (6.0 * 2 * g.volh)
    clov = g.clover_init(u, CSW * KAPPA)
    g.flip_bc(u)
    O.ranset(0)
    b = g.gauss_spinor(0, 0.5)
    b2 = float(np.vdot(b, b).real)
    # the stopping rule of the GPU arm: |r|^2 <= tol^2 |b|^2 on the iterated
    # residual (cg.F90:111 with rest = tol^2 |b|^2), then the true residual
    rest = np.float32(args.tol ** 2 * b2)
    t0 = time.perf_counter()
    x, iters, rtr, rc = g.cg("mtdagmt", np.zeros_like(b), b, u, clov, KAPPA, CSW * KAPPA, 0.0, 0.0, rest=rest,
                             maxiter=args.ref_maxiter, log=2)
    full = time.perf_counter() - t0
    ax = g.op("mtdagmt", x, u, clov, KAPPA, CSW * KAPPA)
    true_rel = float(np.linalg.norm(b - ax) / np.sqrt(b2))
    converged = rtr <= rest
    per_iter_full = full / max(1, iters)
    n = max(10, min(iters, int(args.ref_sample_seconds / max(per_iter_full, 1e-9))))
    samples = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        g.cg("mtdagmt", np.zeros_like(b), b, u, clov, KAPPA, CSW * KAPPA, 0.0, 0.0, rest=0.0, maxiter=n, log=2)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            samples.append(dt / n * iters)
    cfg = solve_config(L, sweeps, plaq, g.volh, world)
    out = {"metric": METRIC, "value": round(full, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(full * 1e3, 1), "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic: host hot start (BQCD ranf, default seed) + %d conf_relax cooling sweep(s) "
                   "(plaquette %.4f), Gaussian b" % (sweeps, plaq),
           "impl": "reference", "config": cfg,
           "full_solve": {"seconds": round(full, 4), "iterations": iters, "converged": bool(converged),
                          "iterated_rel_residual": float(np.sqrt(max(rtr, 0.0) / b2)),
                          "true_rel_residual": true_rel, "s_per_iteration": per_iter_full},
           "sampled_steps": {"iterations_per_sample": n, "scaled_s": [round(v, 3) for v in samples],
                             "mean_scaled_s": round(sum(samples) / len(samples), 4)},
           "cpu_baseline": {"value": round(full, 4), "unit": "s", "cores": O.threads(), "kind": "port",
                            "sample": "one full FP64 CG solve (cg.F90 restated, M~^+M~ at %s) from x = 0: %d "
                                      "iterations, true |r|/|b| %.2e, %.1f s; then %d timed samples of %d "
                                      "iterations each, scaled to %d iterations (mean %.1f s)"
                                      % ("x".join(map(str, L)), iters, true_rel, full, len(samples), n, iters,
                                         sum(samples) / len(samples))},
           "e2e": {"value": round(full, 4), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_hmc(args):
    """Optional workload: full HMC trajectories at 24^3x48 (clover-Wilson
    N_f = 2, Hasenbusch with two pseudofermions: kappa 0.1355, shift kappa
    0.13 as rho = kappa/kappa_shift - 1 in BQCD's W = M~ + rho; beta 5.29,
    c_sw 1.9192; trajectory length 1 in 20 outer x 5 inner leapfrog steps,
    BQCD's only integrator; mixed-precision solves), every field resident on
    the device.  The synthetic start (hot start + cooling) is brought towards
    equilibrium by forced-accept pure-gauge trajectories first.  One step =
    one trajectory; the value is seconds per trajectory."""
    import numpy as np
    import bqcdg as bq
    from bqcdg.hmc import Hmc, quenched_trajectory

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "24,24,24,48")
    kappa, kshift, beta = 0.1355, 0.13, 5.29
    lat, hb, _ = build_system(bq, L, local, 1000003 * rank, args.cool)
    therm = []
    for _ in range(args.therm):
        acc, dh, plaq = quenched_trajectory(lat, beta, 1.0, 50, force_accept=True)
        therm.append(round(plaq, 5))
    b2 = lat.field_cdot(hb, hb).real   # |phi|^2 scale of a unit-variance field
    hmc = Hmc(lat, beta=beta, kappa=kappa, csw=CSW, rho=kappa / kshift - 1, traj_length=1.0, ntau=20, m_scale=5,
              model="C", rest=1e-20 * b2, maxiter=100000, solver="mixed")
    # dynamical thermalisation: forced-accept N_f = 2 trajectories of the
    # same algorithm, which bring the configuration to the fermionic
    # equilibrium, where dH is O(1)
    therm_dyn = []
    for k in range(args.therm_dyn):
        rec = hmc.trajectory(force_accept=True)
        therm_dyn.append({"dh": round(rec["dh"], 3), "plaq": round(1.0 - rec["plaq_energy"], 5)})
        print("hmc: thermalisation %d dH %.3f plaquette %.5f" % (k, rec["dh"], 1.0 - rec["plaq_energy"]),
              file=sys.stderr, flush=True)
    recs = []
    for k in range(args.warmup + args.steps):
        barrier(pg, local)
        t0 = time.perf_counter()
        rec = hmc.trajectory()
        rec["seconds"] = allmax(pg, time.perf_counter() - t0, local)
        print("hmc: trajectory %d dH %.4f accepted %d %.2f s" % (k, rec["dh"], rec["accepted"], rec["seconds"]),
              file=sys.stderr, flush=True)
        if k >= args.warmup:
            recs.append(rec)
    if rank == 0:
        secs = [r["seconds"] for r in recs]
        out = {"metric": "HMC trajectory time at %s (N_f=2 clover, Hasenbusch, 20/5 nested leapfrog)"
                         % "x".join(map(str, L)),
               "value": round(sum(secs) / len(secs), 3), "unit": "s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(1e3 * sum(secs) / len(secs), 1),
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64 (int16/f32 sloppy solves)", "data": "synthetic: hot start + %d conf_relax sweep(s), "
               "then %d forced-accept pure-gauge trajectories (plaquettes %s), then %d forced-accept N_f=2 "
               "trajectories of the measured algorithm" % (lat.sweeps, args.therm, therm, args.therm_dyn),
               "config": {"workload": "HMC model C, lattice %s, kappa %.4f, kappa_shift %.2f (rho %.5f), c_sw %.4f, "
                                      "beta %.2f, tau 1, 20x5 steps" % ("x".join(map(str, L)), kappa, kshift,
                                                                      kappa / kshift - 1, CSW, beta),
                          "parallelism": "replicas x%d" % world},
               "trajectories": [{k: r[k] for k in ("accepted", "dh", "plaq_energy", "it_f1", "it_f2", "cg_calls",
                                                   "cg_it_max", "seconds")} for r in recs],
               "acceptance": sum(1 for r in recs if r["accepted"]) / len(recs),
               "dh_mean": sum(r["dh"] for r in recs) / len(recs),
               "dh_abs_max": max(abs(r["dh"]) for r in recs),
               "exp_minus_dh_mean": sum(math.exp(-r["dh"]) for r in recs) / len(recs),
               "thermalisation_dynamical": therm_dyn}
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


def run_batch(args):
    """Optional workload: 16 right-hand sides at 48^3x96, kappa 0.1355 (the
    default workload's action; its gauge construction followed by the
    pure-gauge thermalisation of the hmc workload): the 12
    spin-colour point sources at the origin plus 4 Gaussian vectors, solved
    to true |r|/|b| < 1e-10 as one batched CG: 16 independent CG recurrences
    whose stencil passes share one launch (FP32 iterations, FP64 reliable
    updates, autotuned right-hand sides per thread), against
    sequential single-RHS solves of the same systems.  The sequential time is
    one point-source and one Gaussian solve scaled to 12 + 4; both arms run
    the same precision and stopping rule."""
    import numpy as np
    import bqcdg as bq

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "48,48,48,96")
    from bqcdg.hmc import quenched_trajectory
    kappa = 0.1355
    lat, hb, hx = build_system(bq, L, local, 1000003 * rank, args.cool)
    # the cooled start is smoother than an equilibrium configuration at
    # beta 5.29, which puts kappa 0.1355 at or past its critical value; the
    # forced-accept pure-gauge trajectories bring the plaquette towards
    # equilibrium, where the system is well conditioned as intended
    therm = []
    for _ in range(args.therm):
        therm.append(round(quenched_trajectory(lat, 5.29, 1.0, 50, force_accept=True)[2], 5))
    lat.clover_init(CSW * kappa)
    para = bq.HmcPara(kappa=kappa, csw=CSW)
    print("batch: start plaquettes %s" % therm, file=sys.stderr, flush=True)
    host = np.zeros((lat.volh, 3, 4), np.complex128)
    hbs, hxs = [], []
    for s_ in range(4):                 # point sources at site (0,0,0,0): even, index 0
        for c_ in range(3):
            host[0, c_, s_] = 1.0
            hbs.append(lat.field(host))
            host[0, c_, s_] = 0.0
    for _ in range(4):
        h = lat.field()
        lat.field_gauss(h, 0.5)
        hbs.append(h)
    hxs = [lat.field() for _ in hbs]
    zero = host

    def reset():
        for h in hxs:
            lat.field_set(h, zero)

    # sequential arm: one point source and one Gaussian vector, scaled
    seq = {}
    for name, k in (("point", 0), ("gauss", 12)):
        reset()
        barrier(pg, local)
        t0 = time.perf_counter()
        info = lat.solve_dev(hxs[k], hbs[k], para, precision=bq.PREC_SINGLE, tol=args.tol)
        seq[name] = {"seconds": time.perf_counter() - t0, "iterations": info.niter, "converged": info.converged,
                     "x": lat.field_get(hxs[k])}
        print("batch: sequential %s %.2f s, %d iterations" % (name, seq[name]["seconds"], info.niter),
              file=sys.stderr, flush=True)
    seq_s = allmax(pg, 12 * seq["point"]["seconds"] + 4 * seq["gauss"]["seconds"], local)
    # batched arm (the right-hand sides per launch are autotuned inside the
    # call by timing a few stencil launches, a small part of the solve)
    reset()
    barrier(pg, local)
    t0 = time.perf_counter()
    infos = lat.solve_batch(hxs, hbs, para, precision=bq.PREC_SINGLE, tol=args.tol, block=0)
    batch_s = allmax(pg, time.perf_counter() - t0, local)
    dx = max(float(np.linalg.norm(lat.field_get(hxs[k]) - seq[n]["x"]) / np.linalg.norm(seq[n]["x"]))
             for n, k in (("point", 0), ("gauss", 12)))
    # block CG arm: one Krylov space for the 16 systems (its seven FP32 blocks
    # need the memory of the batched solver's buffers, released first)
    lat.release_scratch(solver=True)
    reset()
    barrier(pg, local)
    t0 = time.perf_counter()
    binfos = lat.solve_block(hxs, hbs, para, tol=args.tol)
    block_s = allmax(pg, time.perf_counter() - t0, local)
    dxb = max(float(np.linalg.norm(lat.field_get(hxs[k]) - seq[n]["x"]) / np.linalg.norm(seq[n]["x"]))
              for n, k in (("point", 0), ("gauss", 12)))
    print("batch: block CG %.2f s, iterations %s" % (block_s, [i.niter for i in binfos]), file=sys.stderr,
          flush=True)
    if rank == 0:
        out = {"metric": "16-RHS batched CG time-to-1e-10 at %s, kappa 0.1355 (FP32 iterations)"
                         % "x".join(map(str, L)),
               "value": round(batch_s, 3), "unit": "s", "n_gpus": world, "steps": 1, "warmup": 0,
               "ms_per_step": round(1e3 * batch_s, 1), "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64 (f32 sloppy iterations)",
               "data": "synthetic: device hot start + %d conf_relax sweep(s) + %d forced-accept pure-gauge "
                       "trajectories at beta 5.29 (plaquettes %s); 12 point sources + 4 Gaussian"
                       % (lat.sweeps, args.therm, therm),
               "config": {"workload": "batched M^+M CG, lattice %s, kappa %.4f, c_sw %.4f, 16 RHS"
                                      % ("x".join(map(str, L)), kappa, CSW), "parallelism": "replicas x%d" % world},
               "sequential_s": round(seq_s, 3), "speedup_vs_sequential": round(seq_s / batch_s, 3),
               "sequential_sample": {n: {k: v for k, v in seq[n].items() if k != "x"} for n in seq},
               "iterations": [i.niter for i in infos], "converged": all(i.converged for i in infos),
               "true_rel_residual_max": max((i.true_rtr / i.b2) ** 0.5 if i.b2 else 0.0 for i in infos),
               "batch_vs_sequential_rel_dx": dx,
               "block_cg": {"seconds": round(block_s, 3), "speedup_vs_sequential": round(seq_s / block_s, 3),
                            "speedup_vs_batched": round(batch_s / block_s, 3),
                            "iterations": [i.niter for i in binfos], "restarts": binfos[0].reliable_updates,
                            "converged": all(i.converged for i in binfos),
                            "true_rel_residual_max": max((i.true_rtr / i.b2) ** 0.5 if i.b2 else 0.0
                                                         for i in binfos),
                            "vs_sequential_rel_dx": dxb}}
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


def run_shifts(args):
    """Optional workload: 8 Gaussian right-hand sides at 64^3x128, each of
    its own hopping parameter kappa_k from 0.134 to 0.136, in one batched
    mixed-precision CG.  c_sw 1.9192: every system has its own clover term,
    A(kappa_k) = 1 + kappa_k T, formed per site from one stored T
    (bqcdg_clover_init_t), and its own hopping coefficient -kappa_k^2.  int16
    links (12 reals), spinors and T, FP64 reliable updates, stop at true
    |r|/|b| < 1e-10 per system; a converged system retires inside the
    kernels while the others go on.  Then each solution is compared with an
    FP64 CG solve of its own system (the per-kappa FP64 operator is checked
    against the oracle's clover_init at each kappa by the test suite), and
    one batched stencil launch is timed for the HBM roofline.  The gauge
    start is the one of the batch workload; only T of the two parities the
    operator reads is kept, and the thermalisation buffers are released
    before the solve, so the 8 systems fit one GPU."""
    import numpy as np
    import bqcdg as bq
    from bqcdg.hmc import quenched_trajectory

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "64,64,64,128")
    kappa, nrhs = 0.136, 8
    kappas = np.linspace(0.134, 0.136, nrhs)

    t_start = time.perf_counter()

    def mem(tag):
        print("shifts: %6.1f s: %s, %.1f GB on the device" % (time.perf_counter() - t_start, tag,
                                                               lat.device_bytes / 1e9), file=sys.stderr, flush=True)

    lat = start_config(bq, L, local, args.cool)
    therm = []
    for _ in range(args.therm):
        therm.append(round(quenched_trajectory(lat, 5.29, 1.0, 50, force_accept=True)[2], 5))
    mem("after thermalisation")
    lat.release_scratch(solver=True, hmc=True)
    lat.clover_init_t(CSW)
    para = bq.HmcPara(kappa=kappa, csw=CSW)
    lat.ranset(0, 1000003 * rank)
    hbs = []
    for _ in range(nrhs):
        h = lat.field()
        lat.field_gauss(h, 0.5)
        hbs.append(h)
    hxs = [lat.field() for _ in range(nrhs)]
    mem("fields ready, plaquettes %s" % therm)
    barrier(pg, local)
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        infos = lat.solve_batch_kappa(hxs, hbs, para, kappas, precision=bq.PREC_HALF, tol=args.tol, block=nrhs)
        wall = time.perf_counter() - t0
    batch_s = allmax(pg, infos[0].seconds, local)
    mem("after the batched solve")
    # one batched first pass over the 8 solutions, and the single-RHS pass
    ms_b = lat.time_pass_batch(hxs, para, bq.PREC_HALF, 20, rhs_per_thread=1)
    ms_1 = lat.time_pass(hxs[0], para, bq.PREC_HALF, 20)
    volh = lat.volh
    alg = volh * (8 * 24 + 148 + nrhs * 2 * 52)      # links and T once, each spinor in and out
    peak, peak_kind = peaks()
    achieved = alg / (ms_b * 1e-3) / 1e9
    # FP64 reference solve of each system, then the batched solution's error
    lat.release_scratch(solver=True)
    zero = np.zeros((volh, 3, 4), np.complex128)
    errs, fp64 = [], []
    for k in range(min(args.ref_rhs, nrhs)):
        xb = lat.field_get(hxs[k])
        lat.field_set(hxs[k], zero)
        info = lat.solve_dev(hxs[k], hbs[k], bq.HmcPara(kappa=float(kappas[k]), csw=CSW), precision=bq.PREC_DOUBLE,
                             tol=args.tol)
        xr = lat.field_get(hxs[k])
        errs.append(float(np.linalg.norm(xb - xr) / np.linalg.norm(xr)))
        fp64.append({"iterations": info.niter, "seconds": round(info.seconds, 3), "converged": info.converged})
        print("shifts: rhs %d fp64 %d iterations %.2f s, rel error %.2e" % (k, info.niter, info.seconds, errs[-1]),
              file=sys.stderr, flush=True)
        del xb, xr
    if rank == 0:
        out = {"metric": "8-RHS batched CG time-to-1e-10 at %s, kappa 0.134-0.136 (int16 iterations)"
                         % "x".join(map(str, L)),
               "value": round(batch_s, 3), "unit": "s", "n_gpus": world, "steps": 1, "warmup": 0,
               "ms_per_step": round(1e3 * batch_s, 1), "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64 (int16 sloppy iterations)",
               "data": "synthetic: device hot start + %d conf_relax sweep(s) + %d forced-accept pure-gauge "
                       "trajectories at beta 5.29 (plaquettes %s); 8 Gaussian right-hand sides"
                       % (lat.sweeps, args.therm, therm),
               "config": {"workload": "batched M^+M CG, lattice %s, c_sw %.4f, 8 RHS each at its own kappa_k "
                                      "%s (its own clover term A(kappa_k) = 1 + kappa_k T and hopping "
                                      "coefficient), one launch of 8"
                                      % ("x".join(map(str, L)), CSW,
                                         ", ".join("%.5f" % x for x in kappas)),
                          "parallelism": "replicas x%d" % world},
               "wall_s": round(wall, 3),
               "kappa": [round(float(k), 6) for k in kappas],
               "iterations": [i.niter for i in infos],
               "reliable_updates": [i.reliable_updates for i in infos],
               "converged": all(i.converged for i in infos),
               "true_rel_residual": [float("%.3e" % ((i.true_rtr / i.b2) ** 0.5)) for i in infos],
               "fp64_rel_error": [float("%.3e" % e) for e in errs],
               "fp64_reference": fp64,
               "fp64_sequential_s": round(sum(f["seconds"] for f in fp64), 3),
               "roofline": {"bound": "hbm", "kernel": "k_pass1<int16, A(kappa)^-1 per site>, 8 right-hand sides "
                                                       "per launch",
                            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                            "frac": round(achieved / peak, 3), "peak_kind": peak_kind,
                            "frac_nominal": round(achieved / NOMINAL_HBM_GBS, 3),
                            "algorithmic_bytes_per_launch": alg, "ms_per_launch": round(ms_b, 4),
                            "single_rhs_ms_per_launch": round(ms_1, 4)},
               "clocks": clk.summary()}
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


# the reference's benchmark jobs (work/input.smp, work/input.mpp): beta 5,
# kappa 0.13, c_sw 1.923076923076923, model A, tau 0.2, cold start, default
# seed, CG capped at 100 iterations (solver_rest 1e-99, no convergence
# ignored), no MRE vectors; the first trajectory is force-accepted
REF_JOBS = {
    "smp": {"L": (24, 24, 24, 48), "ntau": 10, "trajectories": 1, "threads": "40 OpenMP threads, 2012"},
    "mpp": {"L": (48, 48, 48, 96), "ntau": 20, "trajectories": 2, "threads": "6912 MPI processes, 2011"},
}


def run_refjob(args, name):
    """Optional workloads smp / mpp: the reference's own benchmark job run on
    the device through the resident HMC entry points, from the cold start,
    as BQCD runs it.  One step = the whole job; the value is its wall time.
    The job's records (CG statistics, plaquette, exp(-dH), acceptance, final
    seed) are checked against work/out.<job>.reference, whose run time is
    printed beside.  The CPU baseline times the oracle's FP64 CG at the
    job's size on a few iterations, scaled to the job's iteration count."""
    import numpy as np
    import bqcdg as bq
    from bqcdg.hmc import Hmc

    job = REF_JOBS[name]
    with open(os.path.join(ROOT, "tests", "golden", "%s.json" % name)) as f:
        gold = json.load(f)
    want = [dict(gold["fa"], accepted=1)] + gold["mc"]
    world, rank, local, pg = dist_init()
    L = job["L"]
    csw, kappa = 1.923076923076923, 0.13
    times, recs, seed = [], None, None
    for k in range(args.warmup + args.steps):
        lat = bq.Lattice(L, (1, 1, 1, -1), device=local)
        barrier(pg, local)
        t0 = time.perf_counter()
        lat.ranset(0)
        lat.conf_cold()
        hmc = Hmc(lat, beta=5.0, kappa=kappa, csw=csw, rho=0.0, traj_length=0.2, ntau=job["ntau"], m_scale=1,
                  model="A", rest=1e-99, maxiter=100, mre_n_vec=0, cg_log=2)
        recs = [hmc.trajectory(force_accept=(t == 0)) for t in range(job["trajectories"])]
        seed = lat.ranget()
        dt = allmax(pg, time.perf_counter() - t0, local)
        if k >= args.warmup:
            times.append(dt)
        lat.close()
    ok = seed == gold["final_seed"] and len(recs) == len(want)
    for r, w in zip(recs, want):
        ok = ok and [r["cg_calls"], r["cg_it_tot"], r["cg_it_max"]] == [w["cg_calls"], w["cg_it_tot"],
                                                                          w["cg_it_max"]]
        ok = ok and int(r["accepted"]) == w["accepted"] and abs(r["plaq_energy"] - w["plaq_energy"]) <= 2e-9
    cpu = None
    iters = sum(r["cg_it_tot"] for r in recs)
    if rank == 0 and not args.no_cpu_baseline:
        # sampled at the SMP job's size (its host fields take 1.5 GB; the
        # MPP job's would take 24 GB), scaled by volume and iterations
        from oracle import oracle as O
        Ls = REF_JOBS["smp"]["L"]
        g = O.Geom(Ls, (1, 1, 1, -1))
        O.ranset(0)
        u = g.cold()
        clov = g.clover_init(u, kappa * csw)
        b = g.gauss_spinor(0)
        n = 10
        t0 = time.perf_counter()
        g.cg("mtdagmt", np.zeros_like(b), b, g.flip_bc(u.copy()), clov, kappa, kappa * csw, rest=0.0, maxiter=n,
             log=2)
        dt = time.perf_counter() - t0
        scale = (L[0] * L[1] * L[2] * L[3]) / (Ls[0] * Ls[1] * Ls[2] * Ls[3])
        cpu = {"value": round(dt / n * iters * scale, 2), "unit": "s", "cores": O.threads(), "kind": "port",
               "sample": "%d FP64 CG iterations of the oracle at %s = %.2f s, scaled by volume (x%g) to the "
                         "job's %d iterations (the CG part of the job only)"
                         % (n, "x".join(map(str, Ls)), dt, scale, iters)}
    # the CG bin of BQCD's timing report (timing.F90): 7728 flop per even
    # site and iteration, over the device time of the solves
    cg_s = sum(r["cg_seconds"] for r in recs)
    volh = L[0] * L[1] * L[2] * L[3] // 2
    ref_cg = gold.get("timing", {}).get("CG", {})
    cg_line = {"calls": sum(r["cg_calls"] for r in recs), "iterations": iters, "seconds": round(cg_s, 3),
               "gflops_bqcd_model": round(7728.0 * volh * iters / cg_s / 1e9, 1),
               "reference_seconds": ref_cg.get("seconds"), "reference_gflops": ref_cg.get("gflops_total")}
    if rank == 0:
        v = sum(times) / len(times)
        out = {"metric": "BQCD %s benchmark job (work/input.%s) wall time on one GPU" % (name.upper(), name),
               "value": round(v, 3), "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": round(1e3 * v, 1), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64", "data": "the reference's own benchmark input: cold start, default seed",
               "config": {"workload": "work/input.%s: %s, model A, kappa 0.13, c_sw 1.9230769, beta 5, %d "
                                      "trajectory(ies) of %d steps, CG capped at 100 iterations"
                                      % (name, "x".join(map(str, L)), job["trajectories"], job["ntau"]),
                          "parallelism": "replicas x%d" % world},
               "records": [{"plaq_energy": r["plaq_energy"], "exp_dh": r["exp_dh"], "accepted": bool(r["accepted"]),
                            "cg": [r["cg_calls"], r["cg_it_tot"], r["cg_it_max"]]} for r in recs],
               "final_seed": seed, "matches_reference_record": bool(ok),
               "cg": cg_line,
               "reference_published_s": gold["total_s"],
               "reference_published_hardware": "%s (work/out.%s.reference)" % (job["threads"], name),
               "cpu_baseline": cpu}
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def run_slabs(args):
    """Optional workload: the benchmark system (32^3x64, the default line's
    solve) by the mixed-precision CG on the time-slab decomposition
    (bqcdg_dd_solve) with 1, 2 and 4 slabs, all in this process on one GPU,
    against the single-domain solve.  What the decomposition costs: the face
    packing and exchange (device copies here, NCCL messages between GPUs),
    the split interior/boundary launches and the sums over the slabs.  One
    step = one solve from x = 0; device seconds by CUDA events."""
    import numpy as np
    import bqcdg as bq

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "32,32,32,64")
    lat, hb, _ = build_system(bq, L, local, 1000003 * rank, args.cool)
    para = bq.HmcPara(kappa=KAPPA, csw=CSW)
    b = lat.field_get(hb)
    uf = lat.get_gauge(flipped=True)
    a, ai, _ = lat.get_clover()
    zero = np.zeros_like(b)
    bnorm = np.linalg.norm(b)

    def timed(solve):
        for _ in range(args.warmup):
            solve()
        runs = [solve() for _ in range(args.steps)]
        x, info = runs[-1]
        res = np.linalg.norm(b - lat.mtdagmt(x, para)) / bnorm   # FP64 residual on the whole lattice
        return {"seconds": round(sum(r[1].seconds for r in runs) / len(runs), 4), "iterations": info.niter,
                "reliable_updates": info.reliable_updates, "true_rel_residual": float(res),
                "converged": bool(info.converged and res < args.tol)}

    one = timed(lambda: lat.solve(zero, b, para, precision=bq.PREC_HALF, tol=args.tol))
    slabs = {}
    for n in (1, 2, 4):
        if L[3] % n or (L[3] // n) % 2:
            continue
        with bq.SlabDecomposition.local(L, n) as dd:
            dd.load_gauge(uf, flipped=True)
            dd.load_clover(a, ai)
            slabs[n] = timed(lambda: dd.solve(zero, b, para, tol=args.tol))
        print("slabs: %d slab(s) %.4f s, %d iterations" % (n, slabs[n]["seconds"], slabs[n]["iterations"]),
              file=sys.stderr, flush=True)
    if rank == 0:
        nmax = max(slabs)
        out = {"metric": "mixed-precision M^+M CG time-to-1e-10 at %s on %d time slabs of one GPU"
                         % ("x".join(map(str, L)), nmax),
               "value": slabs[nmax]["seconds"], "unit": "s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(1e3 * slabs[nmax]["seconds"], 1),
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64 (int16 sloppy iterations)",
               "data": "synthetic: the default workload's system (plaquette %.4f), Gaussian b" % (1.0 - lat.plaq_energy()),
               "config": {"workload": "bqcdg_dd_solve, lattice %s, kappa %.4f, c_sw %.4f, slabs in one process"
                                      % ("x".join(map(str, L)), KAPPA, CSW), "parallelism": "replicas x%d" % world},
               "single_domain": one,
               "slabs": {str(k): dict(v, overhead_vs_single_domain=round(v["seconds"] / one["seconds"] - 1.0, 4))
                         for k, v in slabs.items()}}
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


def run_confio(args):
    """Optional workload: BQCD's configuration files (conf.F90 conf_write /
    conf_read with the per-slice cksum of cksum.c) for the 32^3x64 links of
    the default workload.  The device reorders, byte-swaps and check-sums
    each time slice in one pass; the files go to a scratch directory.  One
    step = one write and one read of the whole configuration (805 MB of
    slice files), wall-clock time including the file system.  The CPU
    baseline is the oracle's numpy restatement with its C cksum, on a
    bounded number of slices."""
    import shutil
    import tempfile
    import numpy as np
    import bqcdg as bq

    world, rank, local, pg = dist_init()
    L = lattice_of(args, "32,32,32,64")
    lat = start_config(bq, L, local, args.cool)
    d = tempfile.mkdtemp(prefix="bqcd_conf_")
    base = os.path.join(d, "bqcd.001.1.1.00000")
    nbytes = L[0] * L[1] * L[2] * L[3] * 384
    u0 = lat.get_gauge()
    w, r = [], []
    for k in range(args.warmup + args.steps):
        barrier(pg, local)
        t0 = time.perf_counter()
        lat.conf_write(base)
        t1 = time.perf_counter()
        lat.conf_read(base + ".info")
        t2 = time.perf_counter()
        if k >= args.warmup:
            w.append(allmax(pg, t1 - t0, local))
            r.append(allmax(pg, t2 - t1, local))
    dev = float(np.abs(lat.get_gauge() - u0).max())
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import confio
        nsl = min(L[3], 8)
        t0 = time.perf_counter()
        for t in range(nsl):
            confio.cksum(confio.slice_bytes(L, u0, t))
        dt = time.perf_counter() - t0
        cpu = {"value": round(dt / nsl * L[3], 3), "unit": "s", "cores": 1, "kind": "port",
               "sample": "%d of %d slices reordered to the file layout (numpy) and check-summed (C), scaled; "
                         "no file system" % (nsl, L[3])}
    shutil.rmtree(d, ignore_errors=True)
    if rank == 0:
        ws, rs = sum(w) / len(w), sum(r) / len(r)
        out = {"metric": "configuration write + read time at %s (BQCD slice files with cksum)"
                         % "x".join(map(str, L)),
               "value": round(ws + rs, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(1e3 * (ws + rs), 1), "higher_is_better": False,
               "scaling": "weak", "vs_baseline": None, "dtype": "u8 (f64 links)",
               "data": "synthetic: device hot start + %d conf_relax sweep(s)" % lat.sweeps,
               "config": {"workload": "conf_write + conf_read, lattice %s, %d slice files of %d bytes"
                                      % ("x".join(map(str, L)), L[3], nbytes // L[3]),
                          "parallelism": "replicas x%d" % world},
               "write_s": round(ws, 4), "read_s": round(rs, 4),
               "write_gbs": round(nbytes / ws / 1e9, 2), "read_gbs": round(nbytes / rs / 1e9, 2),
               "round_trip_max_abs_diff": dev, "cpu_baseline": cpu}
        print(json.dumps(out))
    lat.close()
    if pg is not None:
        pg.destroy_process_group()


def run_plumbing(args):
    """CPU stand-in for the replica plumbing of the other workloads, for
    testing bench.py --gpus N without a GPU: every rank times the oracle's
    M~^+M~ CG on its own seeded 4^4 system between the same barriers, the
    step time is the max over ranks, and rank 0 prints one line with every
    rank's time beside it.  Not a benchmark."""
    import numpy as np
    from oracle import oracle as O
    world, rank, local, pg = dist_init()
    L = lattice_of(args, "4,4,4,4")
    g = O.Geom(L, (1, 1, 1, -1))
    O.ranset(0, 1000003 * rank)
    u = g.hot()
    clov = g.clover_init(u, CSW * KAPPA)
    g.flip_bc(u)
    b = g.gauss_spinor(0, 0.5)
    for _ in range(args.warmup):
        g.cg("mtdagmt", np.zeros_like(b), b, u, clov, KAPPA, CSW * KAPPA, rest=0.0, maxiter=20, log=2)
    barrier(pg, local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.cg("mtdagmt", np.zeros_like(b), b, u, clov, KAPPA, CSW * KAPPA, rest=0.0, maxiter=20, log=2)
    mine = (time.perf_counter() - t0) / args.steps + 0.01 * rank    # a rank-dependent part, to see the max
    step = allmax(pg, mine, local)
    per_rank = [mine]
    if pg is not None:
        import torch
        t = torch.zeros(world, dtype=torch.float64)
        t[rank] = mine
        pg.all_reduce(t)
        per_rank = t.tolist()
    if rank == 0:
        print(json.dumps({"metric": "replica plumbing (CPU stand-in)", "value": step, "unit": "s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "per_rank_s": per_rank,
                          "scaling": "weak", "config": {"workload": "plumbing", "lattice": list(L),
                                                        "parallelism": "replicas x%d" % world}}))
    if pg is not None:
        pg.destroy_process_group()


def self_launch(args):
    """bench.py --gpus N (N > 1) started without torchrun: start N ranks,
    one per GPU, through torch.distributed.run on 127.0.0.1 with the same
    arguments, and return their exit status.  Rank 0 prints the line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="solve",
                    choices=["solve", "hmc", "batch", "shifts", "confio", "slabs", "smp", "mpp", "plumbing"],
                    help="solve: the M^+M CG time-to-solution (the default line); hmc: full trajectories; "
                         "batch: 16 right-hand sides; shifts: 8 shifted systems at 64^3x128; "
                         "confio: configuration files; slabs: the solve on 1, 2, 4 time slabs of one GPU; "
                         "smp, mpp: the reference's benchmark jobs; "
                         "plumbing: CPU stand-in for testing the multi-process launch")
    ap.add_argument("--therm", type=int, default=10,
                    help="hmc, batch, shifts: forced-accept pure-gauge trajectories on the start configuration")
    ap.add_argument("--therm-dyn", type=int, default=30,
                    help="hmc: forced-accept N_f=2 trajectories after the pure-gauge ones, before the measured ones")
    ap.add_argument("--ref-rhs", type=int, default=8, help="shifts: systems checked against an FP64 solve")
    ap.add_argument("--lattice", default=None,
                    help="x,y,z,t; default 32,32,32,64 (solve), 24,24,24,48 (hmc), 48,48,48,96 (batch), "
                         "64,64,64,128 (shifts)")
    ap.add_argument("--cool", type=int, default=-1,
                    help="conf_relax sweeps; -1: until the plaquette reaches %.2f" % PLAQ_TARGET)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=0, help="timed e2e calls; 0: as many as --steps")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU seconds of the cpu_baseline's CG sample")
    ap.add_argument("--ref-maxiter", type=int, default=20000)
    ap.add_argument("--ref-sample-seconds", type=float, default=1.5,
                    help="reference arm: CPU seconds of each timed step's bounded CG sample (at least 10 iterations)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(self_launch(args))
    if args.workload == "plumbing":
        run_plumbing(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "hmc":
        run_hmc(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "shifts":
        run_shifts(args)
    elif args.workload == "confio":
        run_confio(args)
    elif args.workload == "slabs":
        run_slabs(args)
    elif args.workload in REF_JOBS:
        run_refjob(args, args.workload)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
