"""Headline benchmark: E0 + G(i w_n) solves of the ns=16 half-filled sector.

One step = one impurity solve of the 1 impurity + 15 bath-site Anderson model
(1.66e8 states in the (8,8) sector): mixed-precision Lanczos ground state with
FP64 residual check and one FP64 refinement restart, then the four Green
chains (c_up, c+_up, c_dn, c+_dn) of 300 steps each and the 512-point
Matsubara continued fractions (beta = 50).  Every solve goes through the C-ABI
entry point edk_solve.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: independent replicas (one solve per rank per step, no collective
in the data path); value = total solves / max-over-ranks device time.
The reference arm times the CPU restatement of the reference's FP64 Lanczos
(OpenMP, all host threads) on a bounded sample of Lanczos steps of the same
sector and converts it to the same unit with the step count of an FP64 solve.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="ns16_halffilled_E0_G512", nc=1, nb=15, sector=(8, 8), beta=50.0, nw=512,
                nitergreen=300, nitermax=1000, tolerance=1e-12, tolerance_lowprec=1e-6,
                residual_tol=1e-9, spins=(0, 1), pairs=[(0, 0)], demax0=5.0, fp32_sums=True)
# H*v applications of one plain FP64 solve of this workload (eigen part + Green part),
# measured on B200 with the library's start-vector table; used to convert a
# per-step CPU time into solves/s for the reference arm.
FP64_STEPS_PER_SOLVE = 1418
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "row_tiled_step_ns16_9_8_f32.md")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_launch():
    """dram__bytes_read.sum + dram__bytes_write.sum of one fused step (ncu summary; the
    two-pass step's two kernels together)."""
    try:
        with open(PROFILE_TRAFFIC) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() in ("active", "1"):
                        reasons.add(n)
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons)}


def _dist():
    from ed_solver_b200.replicas import env
    return env()


def _model():
    from ed_solver_b200.model import workload
    return workload("c5").model


def _solve(ctx, model, dtype):
    from ed_solver_b200 import edk
    w = WORKLOAD
    return edk.solve(ctx, model, [w["sector"]], w["beta"], w["nw"], dtype=dtype, neigen=1,
                     nitermax=w["nitermax"], tolerance=w["tolerance"], tolerance_lowprec=w["tolerance_lowprec"],
                     demax0=w["demax0"], nitergreen=w["nitergreen"], spins=w["spins"], pairs=w["pairs"],
                     residual_tol=w["residual_tol"], fp32_sums=w["fp32_sums"] and dtype == "f32")


def _hv_time(ctx, model, peak, reps=10):
    """Plain H*v (FP32 in, FP32 out) of the headline sector: mean CUDA-event time
    of `reps` launches inside the library, algorithmic bytes 2 D 4 B (read x,
    write y; tables below 0.2 %)."""
    import torch
    from ed_solver_b200 import edk
    h = edk.Hamiltonian(ctx, model, *WORKLOAD["sector"])
    x = torch.randn(h.dim, dtype=torch.float32, device=f"cuda:{ctx.device}")
    y = torch.empty_like(x)
    ctx.set_fp32_sums(WORKLOAD["fp32_sums"])
    h.hmult(x, out=y)                                 # launch shape timed here
    h.hmult(x, out=y)
    torch.cuda.synchronize()
    ctx.timing(False)
    ctx.timing(True)
    for _ in range(reps):
        h.hmult(x, out=y)
    torch.cuda.synchronize()
    n, ms, el = ctx.timing_report(4)
    ctx.timing(False)
    ctx.set_fp32_sums(False)
    t = ms / max(n, 1)
    gbs = 2.0 * 4.0 * h.dim / (t * 1e-3) / 1e9
    del x, y
    h.close()
    return {"ms_per_hv": t, "achieved_gbs": gbs, "frac": gbs / peak, "launches": n,
            "fp32_sums": WORKLOAD["fp32_sums"], "algorithmic_bytes": 8.0 * h.dim}


def _cpu_step_time(model, nsteps=2):
    """Seconds per FP64 Lanczos step of the CPU restatement (all host threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    h = O.OracleH(model, *WORKLOAD["sector"])
    v0 = O.start_vector(h.dim)
    O.lanczos_steps(h, 1, v0)                      # warm the pages
    t0 = time.perf_counter()
    O.lanczos_steps(h, nsteps, v0)
    dt = (time.perf_counter() - t0) / nsteps
    return dt, O.num_threads()


def _config(ws):
    """The workload's config, the same on both arms."""
    return {"workload": WORKLOAD["name"], "sector": list(WORKLOAD["sector"]), "dim": 12870 * 12870,
            "nw": WORKLOAD["nw"], "beta": WORKLOAD["beta"], "nitergreen": WORKLOAD["nitergreen"],
            "chains": 4, "parallelism": f"replicas{ws}",
            "l2": "vectors (662 MB FP32) exceed L2 (126 MB); no flush needed"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    model = _model()
    steps_per_solve = FP64_STEPS_PER_SOLVE or 1500
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    h = O.OracleH(model, *WORKLOAD["sector"])
    v0 = O.start_vector(h.dim)
    for _ in range(args.warmup):
        O.lanczos_steps(h, 1, v0)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.lanczos_steps(h, 1, v0)
        ts.append(time.perf_counter() - t0)
    t_step = statistics.median(ts)
    value = 1.0 / (t_step * steps_per_solve)
    # a step of this arm is a bounded sample of the solve: one FP64 Lanczos
    # step of the sector on the host cores; the value converts the median
    # step time to solves/s with the H*v count of one FP64 solve
    line = {
        "impl": "reference", "metric": "impurity solves/s (E0 + G(iw_n), ns=16 sector)", "value": value,
        "unit": "solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "step": "one FP64 Lanczos step of the sector (a bounded sample of the solve)",
        "modelled_solve_s": t_step * steps_per_solve, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(ws),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": O.num_threads(), "kind": "port",
                         "sample": f"{args.steps} FP64 Lanczos steps of the (8,8) sector, median "
                                   f"{t_step:.3f} s/step, x {steps_per_solve} steps per FP64 solve"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.replicas import Replicas
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", timeout_s=600.0, device=local)
    ctx = edk.Context(local)
    model = _model()
    stream = torch.cuda.current_stream(local)
    barrier = rep.barrier

    # ---- warm-up (tables built once and kept on the context) ----
    for _ in range(args.warmup):
        res = _solve(ctx, model, "f32")
    barrier()
    ctx.timing(True)
    launches0 = ctx.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev0.record(stream)
        results = [_solve(ctx, model, "f32") for _ in range(args.steps)]
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launches - launches0
    n6, t6, e6 = ctx.timing_report(6)          # fused Lanczos step, FP32
    n5, t5, e5 = ctx.timing_report(5)          # first Lanczos step, FP32
    ctx.timing(False)
    clocks = clk.summary()
    t_max = rep.max(ms)
    value = ws * args.steps / (t_max * 1e-3)
    res = results[-1]

    out = None
    if rank == 0:
        peak, peak_kind = _peaks()
        step_bytes = 3.0 * 4.0 * e6                      # read v_k, read v_{k-1}, write w per element (FP32)
        achieved = step_bytes / (t6 * 1e-3) / 1e9 if t6 > 0 else None
        traffic = _traffic_per_launch()
        # ---- plain FP64 solves: accuracy reference and speed-up (same clock, up to 5 solves) ----
        torch.cuda.synchronize()
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _solve(ctx, model, "f64")                        # builds FP64 workspace
        n64 = max(1, min(5, args.steps))
        e_a.record(stream)
        r64s = [_solve(ctx, model, "f64") for _ in range(n64)]
        e_b.record(stream)
        torch.cuda.synchronize()
        r64 = r64s[-1]
        t64 = e_a.elapsed_time(e_b) * 1e-3 / n64
        # ---- plain H*v of the (8,8) sector, FP32 (the metric's first half) ----
        hv = _hv_time(ctx, model, peak)
        # ---- the FP32 row-kernel launch shape the timing chose per sector of the solve ----
        chosen = {}
        for sec in [(8, 8), (9, 8), (7, 8), (8, 9), (8, 7)]:
            hs = edk.Hamiltonian(ctx, model, *sec)
            chosen["%d,%d" % sec] = hs.launch_shape_chosen("f32", WORKLOAD["fp32_sums"])
            hs.close()
        steps64 = r64["lanczos_steps"] + r64["green_steps"]
        dG = float(np.abs(res["G"] - r64["G"]).max())
        dE = abs(res["e0"] - r64["e0"]) / abs(r64["e0"])
        # ---- end to end: tables rebuilt and uploaded from host arrays every solve ----
        h2d0, d2h0 = ctx.transfer_bytes()
        t0 = time.perf_counter()
        ne2e = 2
        for _ in range(ne2e):
            ctx.clear_cache()
            _solve(ctx, model, "f32")
        torch.cuda.synchronize()
        t_e2e = (time.perf_counter() - t0) / ne2e
        h2d1, d2h1 = ctx.transfer_bytes()
        # ---- CPU baseline: the CPU restatement on this host ----
        cpu = None
        if ws == 1 and not args.no_cpu:
            t_cpu, cores = _cpu_step_time(model, nsteps=2)
            cpu = {"value": 1.0 / (t_cpu * steps64), "unit": "solves/s", "cores": cores, "kind": "port",
                   "sample": f"2 FP64 Lanczos steps of the (8,8) sector ({t_cpu:.3f} s/step) x {steps64} "
                             f"H*v per FP64 solve"}
        out = {
            "metric": "impurity solves/s (E0 + G(iw_n), ns=16 sector)",
            "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 vectors, f64 alpha/beta/CF (mixed)", "data": "synthetic",
            "config": _config(ws),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "kernel": "fused FP32 Lanczos step (row kernels timed per sector shape: the "
                                   "two-pass tiled step, up_pass_quad_kernel + down_pass_kernel, or "
                                   "row_lean_kernel; one launch = one step)",
                         "launches": n6, "avg_launch_ms": (t6 / n6) if n6 else None,
                         "algorithmic_bytes_per_launch": (step_bytes / n6) if n6 else None},
            "cpu_baseline": cpu,
            "e2e": {"value": 1.0 / t_e2e, "unit": "solves/s",
                    "h2d_bytes_per_step": (h2d1 - h2d0) // ne2e, "d2h_bytes_per_step": (d2h1 - d2h0) // ne2e},
            "gpu_launches": launches,
            "clocks": clocks,
            "fp64": {"solve_s": t64, "solves_per_s": 1.0 / t64, "hv_steps": steps64, "solves_timed": n64},
            "hv": hv,
            "row_kernel_shapes": chosen,
            "speedup_mixed_vs_fp64": t64 / (t_max * 1e-3 / args.steps),
            "accuracy_vs_fp64": {"rel_dE0": dE, "max_abs_dG": dG, "residual": res["residual"],
                                 "docc": float(res["docc"][0]), "docc_fp64": float(r64["docc"][0])},
            "mixed": {"hv_steps": res["lanczos_steps"] + res["green_steps"], "e0": res["e0"]},
        }
    rep.close()
    ctx.close()
    if out is not None:
        print(json.dumps(out), flush=True)


def run_kernel_case(args):
    """Six FP32 Lanczos steps of one ns=16 sector (--kernel-sector, default
    (8,8)) and nothing else: the small case (3.3 GB of vectors) for per-kernel
    ncu captures."""
    import torch
    from ed_solver_b200 import edk
    ctx = edk.Context(0)
    sector = tuple(int(v) for v in args.kernel_sector.split(",")) if args.kernel_sector else WORKLOAD["sector"]
    h = edk.Hamiltonian(ctx, _model(), *sector)
    # one fixed launch shape (--kernel-shape, an index into the sector's list), no timing launches
    ctx.set_fp32_sums(args.fp32_sums)
    shapes = h.launch_shapes("f32")
    ctx.set_kernel_path(16 + args.kernel_shape)
    r = h.lanczos_e0(dtype="f32", nitermax=6, tolerance=0.0, check_every=6)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": f"ns16 {sector} FP32 Lanczos", "dim": h.dim, "niter": r["niter"],
                      "shape": shapes[args.kernel_shape % len(shapes)], "fp32_sums": bool(args.fp32_sums)}),
          flush=True)
    h.close()
    ctx.close()


def run_shape_sweep(args):
    """CUDA-event time of the fused FP32 Lanczos step (FP32 hop sums) at every
    feasible launch shape of the ns=16 sectors given (--shape-sweep, e.g.
    9,8;8,9): each shape pinned in turn, 8 untimed steps, then 40 timed ones;
    one JSON line per shape."""
    import torch
    from ed_solver_b200 import edk
    ctx = edk.Context(0)
    ctx.set_fp32_sums(True)
    ctx.set_graphs(False)
    model = _model()
    for spec in args.shape_sweep.split(";"):
        sector = tuple(int(v) for v in spec.split(","))
        h = edk.Hamiltonian(ctx, model, *sector)
        for i, sh in enumerate(h.launch_shapes("f32")):
            ctx.set_kernel_path(16 + i)
            h.lanczos_e0(dtype="f32", nitermax=8, tolerance=0.0, check_every=8)
            ctx.timing(True)
            h.lanczos_e0(dtype="f32", nitermax=40, tolerance=0.0, check_every=40)
            torch.cuda.synchronize()
            n, ms, _ = ctx.timing_report(6)
            ctx.timing(False)
            step = ms / max(n, 1)
            print(json.dumps({"sector": list(sector), "shape_index": i, "shape": sh, "steps": n,
                              "ms_per_step": step, "algorithmic_gbs": 12.0 * h.dim / step / 1e6}), flush=True)
        h.close()
    ctx.set_kernel_path(0)
    ctx.close()


def run_grad(args):
    """Gradients of E0 + G(i w_n) of the (8,8) ground state with respect to
    the 32 star-model parameters (15 bath levels, 15 hybridisations, impurity
    level, U): one edk_grad_green call (four 300-step chains, 512 frequencies,
    FP64), timed, then central differences (h = 1e-5, FP64 solves) for the
    first args.grad_fd parameters."""
    import numpy as np
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.model import matsubara
    w = WORKLOAD
    ctx = edk.Context(0)
    model = _model()
    params = edk.star_params(model)
    chains = [(0, 0, True), (0, 0, False), (0, 1, True), (0, 1, False)]
    wn = matsubara(w["beta"], w["nw"])
    rng = np.random.default_rng(11)
    gbar = rng.normal(size=(4, w["nw"])) + 1j * rng.normal(size=(4, w["nw"]))
    e0bar = 1.0

    def ground(m):
        h = edk.Hamiltonian(ctx, m, *w["sector"])
        r = h.lanczos_e0("f64", tolerance=1e-14, residual_tol=1e-11, nitermax=w["nitermax"])
        return h, h.lanczos_gs(r["vecp"][0]), float(r["E"][0])

    def loss(m):
        h, psi, e0 = ground(m)
        val = e0bar * e0
        for c, (site, spin, dag) in enumerate(chains):
            phi, ts = h.apply_c(psi, site, spin, dag)
            ht = edk.Hamiltonian(ctx, m, *ts)
            G, _, _, _ = ht.green_chain(phi, w["nitergreen"], e0, 1 if dag else 2, wn, cutoff_dynamic=0.0)
            val += float(np.sum((np.conj(gbar[c]) * G).real))
            ht.close()
            del phi
        h.close()
        return val

    h, psi, e0 = ground(model)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    grad, _, st = h.grad_green(psi, e0, chains, w["nitergreen"], wn, gbar, params, e0bar=e0bar, cg_tol=1e-11)
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    h.close()
    del psi
    ctx.clear_cache()
    nfd = min(args.grad_fd, len(params))
    fd = []
    for p in params[:nfd]:
        fd.append((loss(edk.perturb(model, p, 1e-5)) - loss(edk.perturb(model, p, -1e-5))) / 2e-5)
    fd = np.array(fd)
    err = np.abs(grad[:nfd] - fd)
    out = {"grad": "E0 + G(iw_n) VJP, ns=16 (8,8), 4 chains x 300 steps, 512 frequencies, FP64",
           "n_params": len(params), "grad_s": t_grad, "stats": st,
           "fd_checked": nfd, "fd_h": 1e-5,
           "max_abs_err": float(err.max()) if nfd else None,
           "max_rel_err_vs_largest": float(err.max() / np.abs(fd).max()) if nfd else None,
           "grad": [float(g) for g in grad], "fd": [float(f) for f in fd]}
    print(json.dumps(out), flush=True)
    ctx.close()


def run_configs(args):
    """The smaller configurations as measured records, one JSON line each:
    C1 (ns=8, FP64, ground state to |r| < 1e-12, 1024 Matsubara points,
    200-step chains), C2 (ns=10 Kanamori, all 121 sectors, FP32 Krylov in
    every sector of at least 1000 states beside the FP64 solve: errors in E0,
    double occupancy and G at 512 points, beta = 40) and C3 (ns=14 (7,7):
    H*v and fused-step GB/s in both precisions, mixed against FP64 solve time
    and accuracy, four 300-step chains).  Solve times are wall-clock over one
    solve after a warm-up solve; kernel times are CUDA events."""
    import numpy as np
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.model import workload
    peak, peak_kind = _peaks()
    ctx = edk.Context(0)

    def timed_solve(*a, **k):
        edk.solve(ctx, *a, **k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = edk.solve(ctx, *a, **k)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    # ---- C1 ----
    w = workload("c1")
    r, t = timed_solve(w.model, w.sectors, w.beta, w.nw, dtype="f64", nitergreen=w.nitergreen, spins=(0, 1),
                       pairs=[(0, 0)], tolerance=1e-14, residual_tol=1e-12)
    print(json.dumps({"config": "C1 ns=8 (4,4) FP64", "solve_s": t, "e0": r["e0"], "residual": r["residual"],
                      "nw": w.nw, "nitergreen": w.nitergreen, "lanczos_steps": r["lanczos_steps"],
                      "green_steps": r["green_steps"]}), flush=True)
    # ---- C2 ----
    w = workload("c2")
    kw = dict(neigen=1, nitergreen=w.nitergreen, spins=(0, 1), pairs=[(0, 0), (1, 1)], tolerance=1e-12)
    r64, t64 = timed_solve(w.model, w.sectors, w.beta, w.nw, dtype="f64", **kw)
    r32, t32 = timed_solve(w.model, w.sectors, w.beta, w.nw, dtype="f32", lowprec_min_dim=1000, **kw)
    print(json.dumps({"config": "C2 ns=10 Kanamori, 121 sectors, FP32 Krylov in sectors >= 1000 states",
                      "solve_s_fp64": t64, "solve_s_mixed": t32,
                      "rel_dE0": abs(r32["e0"] - r64["e0"]) / abs(r64["e0"]),
                      "max_abs_ddocc": float(np.abs(r32["docc"] - r64["docc"]).max()),
                      "max_abs_dG": float(np.abs(r32["G"] - r64["G"]).max()), "nw": w.nw, "beta": w.beta,
                      "nstates": r64["nstates"]}), flush=True)
    # ---- C3 ----
    w = workload("c3")
    h = edk.Hamiltonian(ctx, w.model, *w.sectors[0])
    rec = {"config": "C3 ns=14 (7,7)", "dim": h.dim, "peak_hbm_gbs": peak, "peak": peak_kind}
    for dt, eb, s32 in (("f64", 8, False), ("f32", 4, False), ("f32", 4, True)):
        tdt = torch.float64 if dt == "f64" else torch.float32
        ctx.set_fp32_sums(s32, 1)
        x = torch.randn(h.dim, dtype=tdt, device="cuda")
        y = torch.empty_like(x)
        for _ in range(3):
            h.hmult(x, out=y)
        torch.cuda.synchronize()
        ctx.timing(True)
        for _ in range(10):
            h.hmult(x, out=y)
        torch.cuda.synchronize()
        n, ms, _ = ctx.timing_report(0 if dt == "f64" else 4)
        ctx.timing(False)
        ctx.timing(True)
        h.lanczos_e0(dtype=dt, nitermax=40, tolerance=0.0, check_every=40)
        torch.cuda.synchronize()
        ns_, mss, _ = ctx.timing_report(2 if dt == "f64" else 6)
        ctx.timing(False)
        key = dt + ("_fp32sums" if s32 else "")
        t_hv, t_st = ms / max(n, 1), mss / max(ns_, 1)
        rec["hv_" + key] = {"ms": t_hv, "gbs": 2 * eb * h.dim / (t_hv * 1e6), "frac": 2 * eb * h.dim / (t_hv * 1e6) / peak}
        rec["step_" + key] = {"ms": t_st, "gbs": 3 * eb * h.dim / (t_st * 1e6), "frac": 3 * eb * h.dim / (t_st * 1e6) / peak}
        del x, y
    ctx.set_fp32_sums(False)
    h.close()
    kw = dict(neigen=1, nitergreen=w.nitergreen, spins=(0, 1), pairs=[(0, 0)], tolerance=1e-12, residual_tol=1e-9)
    r64, t64 = timed_solve(w.model, w.sectors, w.beta, w.nw, dtype="f64", **kw)
    r32, t32 = timed_solve(w.model, w.sectors, w.beta, w.nw, dtype="f32", fp32_sums=True, **kw)
    rec.update({"solve_s_fp64": t64, "solve_s_mixed": t32, "speedup_mixed_vs_fp64": t64 / t32,
                "rel_dE0": abs(r32["e0"] - r64["e0"]) / abs(r64["e0"]),
                "max_abs_dG": float(np.abs(r32["G"] - r64["G"]).max()),
                "max_abs_ddocc": float(np.abs(r32["docc"] - r64["docc"]).max())})
    print(json.dumps(rec), flush=True)
    ctx.close()


def run_c4(args):
    """The many-small-sectors workload: two-orbital Kanamori model, ns = 12
    (169 sectors, dims up to 924^2), 3 lowest states per sector inside the
    exp(-beta (E - E0)) >= 1e-8 window, 8 Green start vectors per state
    (2 spins x particle/hole x 2 orbitals), 200-step chains, 512 Matsubara
    points, FP64.  Times the solve sector by sector and chain by chain against
    the chains batched into one persistent launch per spin and against the
    ground states of the sectors below a size bound batched into two
    persistent launches; the eigen part alone and the whole solve."""
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.model import workload
    w = workload("c4")
    ctx = edk.Context(0)
    out = {"workload": "c4_ns12_kanamori_all_sectors", "sectors": len(w.sectors)}
    # (green_mode, batch_gs): per sector and per chain / chains batched / ground
    # states of sectors up to 2^12, 2^14, 2^16 states batched; the eigen part
    # alone (no Green chains) and the whole solve, median of 3 runs after one
    # warm-up run of each
    import numpy as np
    modes = {"per_sector": (1, 0), "batched_chains": (0, 0), "batched_gs_4096": (1, 4096),
             "batched_gs_16384": (1, 16384), "batched_gs_65536": (1, 65536)}

    def run(gm, bg, spins):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = edk.solve(ctx, w.model, w.sectors, w.beta, 512, dtype="f64", neigen=3, nitergreen=200,
                      demax0=w.demax0, spins=spins, pairs=[(0, 0), (1, 1)], tolerance=1e-10, green_mode=gm,
                      batch_gs=bg)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    # warm-up: every mode twice (tables, launch shapes, workspaces, the basis pool)
    for _ in range(2):
        for gm, bg in modes.values():
            run(gm, bg, (0, 1))
    te = {k: [] for k in modes}
    ts = {k: [] for k in modes}
    last = {}
    # timed runs interleaved over the modes, so slow phases of the box hit all of them
    for _ in range(5):
        for key, (gm, bg) in modes.items():
            te[key].append(run(gm, bg, ())[1])
    for _ in range(3):
        for key, (gm, bg) in modes.items():
            last[key], t = run(gm, bg, (0, 1))
            ts[key].append(t)
    for key in modes:
        rs = last[key]
        out[key] = {"solve_s": statistics.median(ts[key]), "eigen_s": statistics.median(te[key]),
                    "solve_s_all": ts[key], "eigen_s_all": te[key], "nstates": rs["nstates"], "e0": rs["e0"],
                    "green_steps": rs["green_steps"], "lanczos_steps": rs["lanczos_steps"]}
        out["G_" + key] = rs["G"]
    G0 = out["G_per_sector"]
    for key in modes:
        G = out.pop("G_" + key)
        out[key]["max_abs_dG_vs_per_sector"] = float(np.abs(G - G0).max())
        out[key]["speedup_vs_per_sector"] = out["per_sector"]["solve_s"] / out[key]["solve_s"]
    print(json.dumps(out), flush=True)
    ctx.close()


def run_sz(args):
    """Nambu (Sz) sectors: H*v (on-the-fly term order, HAIMsz_mult_fly_r) and
    fused Lanczos steps of the half-filled sector of the one-orbital
    superconducting star model (seeded synthetic bath, s-wave pairing on every
    bath site) at ns = 14 (40,116,600 states)
    and ns = 16 (601,080,390 states), FP64 and FP32 vectors, timed with CUDA
    events on the context's stream (inputs larger than L2).  Algorithmic bytes
    per state: H*v reads x and writes y (2 elements); a fused step reads s,
    v_k, v_k-1 and writes s', v_k+1 (5 elements).  The CPU oracle's H*v
    (OpenMP, all host threads) is timed once at ns = 14 beside it."""
    import numpy as np
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.model import nambu_workload
    peak, peak_kind = _peaks()
    ctx = edk.Context(0)
    out = {"workload": "nambu_star_halffilled", "peak_hbm_gbs": peak, "peak": peak_kind, "cases": []}
    for ns in (14, 16):
        m = nambu_workload(ns, on_fly=True)
        h = edk.HamiltonianSz(ctx, m, ns)
        for dt, eb in (("f64", 8), ("f32", 4)):
            tdt = torch.float64 if dt == "f64" else torch.float32
            x = torch.randn(h.dim, dtype=tdt, device="cuda")
            y = torch.empty_like(x)
            for _ in range(3):
                h.hmult(x, out=y)
            ctx.timing(True)
            for _ in range(max(args.steps, 5)):
                h.hmult(x, out=y)
            cls = 0 + (4 if dt == "f32" else 0)
            n, ms, el = ctx.timing_report(cls)
            ctx.timing(False)
            hv_ms = ms / max(n, 1)
            del x, y
            torch.cuda.empty_cache()
            ctx.timing(True)
            r = h.lanczos_e0(dt, nitermax=24, tolerance=0.0, check_every=24)
            ns_, ms_s, _ = ctx.timing_report(2 + (4 if dt == "f32" else 0))
            ctx.timing(False)
            st_ms = ms_s / max(ns_, 1)
            case = {"ns": ns, "dim": h.dim, "dtype": dt,
                    "hv_ms": hv_ms, "hv_gbs": 2 * eb * h.dim / hv_ms * 1e-6,
                    "step_ms": st_ms, "step_gbs": 5 * eb * h.dim / st_ms * 1e-6, "step_launches": ns_,
                    "e0_24_steps": float(r["E"][0]) + h.energy_shift}
            case["hv_frac"] = case["hv_gbs"] / peak
            case["step_frac"] = case["step_gbs"] / peak
            out["cases"].append(case)
            print(json.dumps(case), flush=True)
        h.close()
        torch.cuda.empty_cache()
    if not args.no_cpu:
        import oracle as O
        m = nambu_workload(14, on_fly=True)
        ho = O.OracleSz(m, 14)
        xv = np.random.default_rng(0).standard_normal(ho.dim)
        t0 = time.perf_counter()
        ho.hmult(xv)
        t1 = time.perf_counter()
        out["cpu_oracle_hv_ms_ns14"] = (t1 - t0) * 1e3
        out["cpu_threads"] = O.num_threads()
    print(json.dumps(out), flush=True)
    ctx.close()


def run_chiloc(args):
    """The local vertex chi~_loc (DNDN and UPDN) of the ns = 4 star model
    (1 impurity + 3 bath sites, U = 2, seeded bath), sector (2,2) (36 states;
    neighbour sectors of 1 to 36 states), beta = 10, for 4096 frequency
    triples (w1, w2, w3) = (i nu_a, i nu_b, i nu_c) on a grid of fermionic
    Matsubara frequencies, every third one with w2 + w3 = 0.  One step = one
    edk_chiloc call for all triples (inputs uploaded from host arrays, results
    read back).  The reference's own chi_tilde_loc_ (oracle/_ref, serial C++)
    is timed on the first 8 triples of the same batch."""
    import numpy as np
    import torch
    from ed_solver_b200 import edk, vertex
    from ed_solver_b200.model import star_model
    rng = np.random.default_rng(5)
    m = star_model(-1.0, 2.0, rng.uniform(-1.0, 1.0, 3), rng.uniform(0.3, 0.6, 3))
    beta, eps, nup, ndn = 10.0, 1e-5, 2, 2
    ctx = edk.Context(0)
    E, M = vertex.vertex_inputs(ctx, m, nup, ndn)
    Z, gs = vertex.partition(E, beta)
    nu = lambda n: 1j * (2 * n + 1) * np.pi / beta
    w = []
    for a in range(-8, 8):
        for b in range(-8, 8):
            for c in range(-8, 8):
                w.append((nu(a), nu(b), -nu(b) if (a + b + c) % 3 == 0 else nu(c)))
    w = np.array(w)
    nf = len(w)
    # algorithmic work: (j, k, l) evaluations of every active term over all states i and triples
    dims = [0 if e is None else len(e) for e in E]
    for _ in range(2):
        edk.chiloc(ctx, E, M, w, beta, Z, gs, m.ns, nup, ndn, phi_eps=eps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(args.steps, 3)
    e0.record()
    for _ in range(steps):
        pd, pu = edk.chiloc(ctx, E, M, w, beta, Z, gs, m.ns, nup, ndn, phi_eps=eps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"workload": "chiloc_ns4_sector22_4096_triples", "dims": dims, "triples": nf,
           "gpu_ms_per_call": ms, "gpu_triples_per_s": nf / (ms * 1e-3)}
    if not args.no_cpu:
        import oracle as O
        if O.ref_chiloc_lib() is not None:
            ns_cpu = 8
            t0 = time.perf_counter()
            ref = [(O.ref_chiloc(1, t, eps, beta, Z, gs, m.ns, nup, ndn, E, M)[0],
                    O.ref_chiloc(2, t, eps, beta, Z, gs, m.ns, nup, ndn, E, M)[1]) for t in w[:ns_cpu]]
            t1 = time.perf_counter()
            out["cpu_reference"] = {"kind": "reference", "cores": 1, "sample": f"first {ns_cpu} triples",
                                    "triples_per_s": ns_cpu / (t1 - t0)}
            rd = np.array([r[0] for r in ref])
            ru = np.array([r[1] for r in ref])
            out["max_rel_diff_vs_reference"] = float(max(np.abs(pd[:ns_cpu] - rd).max() / np.abs(rd).max(),
                                                         np.abs(pu[:ns_cpu] - ru).max() / np.abs(ru).max()))
            out["speedup_vs_reference"] = out["gpu_triples_per_s"] / out["cpu_reference"]["triples_per_s"]
    print(json.dumps(out), flush=True)
    ctx.close()


def run_chiloc_case(args):
    """One edk_chiloc call on the first 256 triples of the --chiloc batch (the
    small case for per-kernel ncu captures)."""
    import numpy as np
    import torch
    from ed_solver_b200 import edk, vertex
    from ed_solver_b200.model import star_model
    rng = np.random.default_rng(5)
    m = star_model(-1.0, 2.0, rng.uniform(-1.0, 1.0, 3), rng.uniform(0.3, 0.6, 3))
    ctx = edk.Context(0)
    E, M = vertex.vertex_inputs(ctx, m, 2, 2)
    Z, gs = vertex.partition(E, 10.0)
    nu = lambda n: 1j * (2 * n + 1) * np.pi / 10.0
    w = [(nu(a), nu(b), -nu(b) if (a + b + c) % 3 == 0 else nu(c))
         for a in range(-8, 8) for b in range(-8, 8) for c in range(-8, 8)][:256]
    edk.chiloc(ctx, E, M, w, 10.0, Z, gs, m.ns, 2, 2)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": "chiloc ns4 (2,2) 256 triples"}), flush=True)
    ctx.close()


def run_sz_case(args):
    """Three FP64 H*v launches of the ns = 14 half-filled Nambu sector (0.64 GB
    of vectors): the small case for per-kernel ncu captures of the Nambu kernel."""
    import torch
    from ed_solver_b200 import edk
    from ed_solver_b200.model import nambu_workload
    ctx = edk.Context(0)
    h = edk.HamiltonianSz(ctx, nambu_workload(14, on_fly=True), 14)
    x = torch.randn(h.dim, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        h.hmult(x, out=y)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": "ns14 Nambu FP64 H*v", "dim": h.dim}), flush=True)
    h.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--kernel-case", action="store_true",
                    help="run only six FP32 Lanczos steps of the (8,8) sector (profiling case)")
    ap.add_argument("--kernel-shape", type=int, default=0,
                    help="launch shape of the --kernel-case (index into the sector's feasible shapes)")
    ap.add_argument("--kernel-sector", default=None, help="sector of the --kernel-case, e.g. 9,8")
    ap.add_argument("--fp32-sums", action="store_true",
                    help="sum the hop terms of H*v in FP32 in the FP32 passes of large sectors")
    ap.add_argument("--shape-sweep", default=None,
                    help="time the fused FP32 step at every launch shape of these ns=16 sectors, e.g. '9,8;8,9'")
    ap.add_argument("--grad", action="store_true",
                    help="time the 32 parameter gradients of E0 + G and check them by central differences")
    ap.add_argument("--grad-fd", type=int, default=4, help="parameters checked by central differences (--grad)")
    ap.add_argument("--c4", action="store_true", help="time the many-small-sectors solve, batched vs per chain")
    ap.add_argument("--configs", action="store_true", help="measured records of the C1, C2 and C3 configurations")
    ap.add_argument("--sz", action="store_true", help="time H*v and fused steps of Nambu (Sz) sectors")
    ap.add_argument("--sz-case", action="store_true", help="three Nambu H*v launches (profiling case)")
    ap.add_argument("--chiloc", action="store_true", help="time the local vertex against the reference kernel")
    ap.add_argument("--chiloc-case", action="store_true", help="one local-vertex call (profiling case)")
    args = ap.parse_args()
    if args.chiloc_case:
        run_chiloc_case(args)
        return
    if args.chiloc:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        run_chiloc(args)
        return
    if args.sz_case:
        run_sz_case(args)
        return
    if args.sz:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        run_sz(args)
        return
    if args.c4:
        run_c4(args)
        return
    if args.configs:
        run_configs(args)
        return
    if args.grad:
        run_grad(args)
        return
    if args.kernel_case:
        run_kernel_case(args)
        return
    if args.shape_sweep:
        run_shape_sweep(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
