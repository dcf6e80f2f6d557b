#!/usr/bin/env python
"""Benchmark of the B200 hyperbolic-SGN FR right-hand side and BS3(2) stage loop.

Workload: configuration 2 (sgnb.workloads): 2048 x 1024 P=4 elements, 262,144,000 DOF,
reflective walls, elliptic shoal, 8 random-phase sine waves, FP64. A "step" is one
accepted adaptive Bogacki-Shampine 3(2) step (3 right-hand-side evaluations per
attempt, rejected attempts included). Metric: DOF-updates per second per RK stage =
DOF x RHS evaluations / time (the reference's own throughput definition,
README.md:369-377 and apps/sgn_bench.cu:138-141 of the reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fast|exact]
    python bench.py --impl reference ...

Our arm prints one JSON line with value (device-resident, CUDA events over K steps,
max over ranks), e2e (the public API with host buffers: upload from pinned memory,
K steps, download), roofline of the dominant kernel, clocks, the CPU baseline (the
oracle port on rank 0: three right-hand sides of the full state, and under "loop" the
reference's integrateAdaptive on a row strip) and the number of kernel launches. N > 1
runs independent replicas, one per GPU (the path does not exchange data between
instances). At N = 1 the line also carries, each measured after the main run on its own
contexts (--no-extras skips them):
  mixed          configuration 2 in the mixed-precision mode against FP64 in the same run,
                 the eta errors of both step sequences, the exact mode's final-state
                 sha256 with the fast mode's relative difference, and each mode's
                 throughput on the frozen replay of the FP64 run's steps;
  batched        configuration 4's 256-instance sweep, batched against the same instances
                 run one after another;
  batched_mixed  the same sweep in the mixed-precision mode, against the sequential FP64
                 runs of the batched record and the sequential mixed ones;
  slabs          configuration 2 on 4 x slabs of one device (edge copies between the slabs,
                 and the fused exchange) against the whole-mesh loop;
  adjoint        configuration 5's forward and VJP times and a central-difference check;
  reference_gpu  the reference's own single-GPU solver (SGN2DCuda::integrateAdaptive,
                 oracle/_ref/ref_gpu_bench) on configuration 2 with periodic boundaries.

The reference arm times the reference's own CPU solver (oracle/_ref, compiled from the
reference sources; the oracle port when that build is absent) on all host cores as
independent single-core replicas, each evaluating right-hand sides of a row strip of
the same configuration-2 mesh, sized so that the run ends within a few minutes.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sgn-hyperbolic-gpu_b200"))

METRIC = "DOF-updates/s per RK stage"
UNIT = "DOF-updates/s"
# Algorithmic HBM bytes per DOF (8 B doubles) of the fused kernels: U in and dU out (16),
# the nodal depth H (8 / 5 fields = 1.6) and the face depths (2 x 5 per element / 125 DOF
# x 8 = 0.64). The nodal depth gradients dH/dx, dH/dy (3.2 B/DOF more if read) are formed
# from the depth tile in shared memory, so they are not part of the kernels' traffic.
STATIC_B = 1.6 + 0.64
BYTES_PER_DOF = {
    "rhs": 16.0 + STATIC_B,                  # 18.24
    "stage": 8 + 8 + STATIC_B + 8,           # u, k in; k_out out: 26.24
    "fsal": 4 * 8 + STATIC_B + 2 * 8,        # u, k1..k3 in; uNew, k4 out: 50.24
}
# Mixed precision: FP64 state, FP32 stage derivatives (4 B), FP64 statics.
BYTES_PER_DOF_MIXED = {
    "rhs": 16.0 + STATIC_B,                  # FP64 in and out (rhs callers): 18.24
    "stage": 8 + 4 + STATIC_B + 4,           # u (8), k (4) in; k_out (4): 18.24
    "fsal": 8 + 3 * 4 + STATIC_B + 8 + 4,    # u, k1..k3 in; uNew (8), k4 (4) out: 34.24
}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_dof():
    """DRAM bytes per DOF per kernel mode from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic_per_dof.txt")
    out = {}
    try:
        for line in open(p):
            line = line.strip()
            if line and not line.startswith("#") and "=" in line:
                k, v = line.split("=", 1)
                out[k.strip()] = float(v)
    except OSError:
        pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_over_ranks(times, works, dist, device):
    """Replica aggregation: the slowest rank's times (max) and the summed work of all
    ranks. Every rank takes the same two collective steps; dist None = one process."""
    if dist is None:
        return list(times), list(works)
    import torch

    t = torch.tensor(times, dtype=torch.float64, device=device)
    w = torch.tensor(works, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.tolist(), w.tolist()


# --------------------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import torch

    import sgnb
    from sgnb import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)

    Nx, Ny, Lx, Ly = W.CFG2["Nx"], W.CFG2["Ny"], W.CFG2["Lx"], W.CFG2["Ly"]
    if args.mesh:
        Nx, Ny = args.mesh
    kw = W.cfg2_solver_args(Nx, Ny, Lx, Ly)
    if args.bc == "periodic":
        kw.update(bc_x=0, bc_y=0)
    prec = {"fast": sgnb.FP64_FAST, "exact": sgnb.FP64_EXACT, "mixed": sgnb.MIXED}[args.precision]
    dof = 5 * 25 * Nx * Ny
    Ud = W.cfg2_state_torch(Nx, Ny, Lx, Ly, device=f"cuda:{local}")
    U_host = torch.empty(Ud.numel(), dtype=torch.float64, pin_memory=True)
    U_host.copy_(Ud)
    del Ud
    torch.cuda.empty_cache()
    U_np = U_host.numpy()
    out_host = torch.empty_like(U_host, pin_memory=True).numpy()

    solver = sgnb.SGN2DB200(precision=prec, device=local, **kw)
    solver.upload(U_np)
    dt0 = solver.cfl_time_step(0.5)
    _, sptr = solver.state_device_ptr()
    stream = torch.cuda.ExternalStream(sptr, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up (graph capture, clocks)
    solver.integrate_steps(0.0, dt0, max(args.warmup, 1))

    # ---- value: state resident in HBM, CUDA events on the solver's stream ----------
    solver.upload(U_np)
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        st = solver.integrate_steps(0.0, dt0, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    t_dev = e0.elapsed_time(e1) / 1e3
    clocks = clk.summary()

    # ---- roofline of the fused stage kernels, timed alone on the same stream -------
    dt_probe = st.dtLast if st.dtLast > 0 else dt0
    per = {}
    for stage, key in ((2, "stage"), (4, "fsal")):
        solver.launch_stage(stage, dt_probe, 2)
        torch.cuda.synchronize()
        reps = 10
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        solver.launch_stage(stage, dt_probe, reps)
        a1.record(stream)
        torch.cuda.synchronize()
        per[key] = a0.elapsed_time(a1) / 1e3 / reps
    dominant = "fsal" if per["fsal"] >= 2 * per["stage"] else "stage"
    peak, peak_kind = measured_peak_hbm()
    bpd = BYTES_PER_DOF_MIXED if args.precision == "mixed" else BYTES_PER_DOF
    achieved = bpd[dominant] * dof / per[dominant] / 1e9
    tpd = traffic_per_dof()
    traffic = tpd.get(dominant) if args.precision != "mixed" else None
    roofline = {"bound": "hbm", "kernel": f"k_fused_tma ({dominant} mode; k_fused on meshes of partial tiles)",
                "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": (round(traffic * dof) if traffic else None),
                "algorithmic_bytes": round(bpd[dominant] * dof),
                "launch_ms": {k: round(v * 1e3, 4) for k, v in per.items()}}
    # both stage kernels, with their shares of an attempt (two intermediate stages and one
    # end point): the two are close to even, so the dominant one can change between runs
    attempt = 2 * per["stage"] + per["fsal"]
    roofline["kernels"] = {
        k: {"achieved": round(bpd[k] * dof / per[k] / 1e9, 1),
            "frac": round(bpd[k] * dof / per[k] / 1e9 / peak, 4),
            "share_of_attempt": round((2 if k == "stage" else 1) * per[k] / attempt, 4)}
        for k in ("stage", "fsal")}

    # ---- e2e through the public API with host buffers ----------------------------
    torch.cuda.synchronize()
    barrier()
    h0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    solver.upload(U_np)                      # H2D of the step inputs (pinned host)
    st_e = solver.integrate_steps(0.0, dt0, args.steps)
    solver.download(out_host)                # D2H of the result (pinned host)
    e3.record(stream)
    torch.cuda.synchronize()
    t_e2e = max(e2.elapsed_time(e3) / 1e3, 0.0)
    t_e2e_host = time.perf_counter() - h0
    barrier()
    finite = bool(np.isfinite(out_host[:: max(1, out_host.size // 100000)]).all())

    # ---- gather over ranks (max time, summed work) ------------------------------
    (t_dev, t_e2e), (rhs_all, rhs_all_e) = reduce_over_ranks(
        [t_dev, t_e2e], [float(st.rhsEvals), float(st_e.rhsEvals)], dist, f"cuda:{local}")
    value = dof * rhs_all / t_dev
    e2e_value = dof * rhs_all_e / t_e2e
    state_bytes = 8 * 5 * 25 * Nx * Ny

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(U_np, kw, dof)
        cpu["loop"] = cpu_baseline_loop(args)
    solver.close()
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        # measured after the main run, each on its own contexts (the main solver is closed)
        from sgnb import benchmarks as BW

        extras = BW.default_extras(args, ClockSampler, (peak, peak_kind))
        t0 = time.perf_counter()
        try:
            extras["reference_gpu"] = run_reference_gpu(args, summary=True)
        except Exception as e:
            extras["reference_gpu"] = {"error": f"{type(e).__name__}: {e}"}
        extras["reference_gpu"]["wall_s"] = round(time.perf_counter() - t0, 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 state, f32 deviations" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"configuration 2: {Nx}x{Ny} P=4 ({dof:,} DOF), "
                                   f"40x20 basin with {'reflective walls' if args.bc == 'walls' else 'periodic boundaries'}, "
                                   "elliptic shoal, 8 random-phase sines; adaptive BS3(2) steps",
                       "mesh": [Nx, Ny], "dof": dof, "precision": f"fp64-{args.precision}",
                       "accepted": st.accepted, "rejected": st.rejected,
                       "rhs_evals": st.rhsEvals, "l2": "inputs larger than L2 "
                       f"({state_bytes / 1e9:.2f} GB state, 6 state-sized buffers)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps,
                    "host_wall_s": t_e2e_host, "final_state_finite": finite},
            "gpu_launches": int(st.kernel_launches),
            "roofline": roofline,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline_port(U, kw, dof):
    """The oracle port (test infrastructure) on 1 host core: three timed right-hand sides
    of the full configuration-2 state after one untimed one, walls included (about 15 s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    o = O.Oracle(**kw)
    o.rhs(U)
    n = 3
    t0 = time.perf_counter()
    for _ in range(n):
        o.rhs(U)
    t = time.perf_counter() - t0
    return {"value": dof * n / t, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} rhs evaluation(s) of the full configuration-2 state "
                      f"(262,144,000 DOF) after one untimed one, {t:.1f} s"}


def cpu_baseline_loop(args, rows=32, span=0.3):
    """The reference's adaptive loop (integrateAdaptive, src/solver/rk.cpp:67-164, through
    oracle/_ref when it was built, else the oracle port) on 1 host core over
    [0, span x dt_CFL0.5] of a 2048 x `rows` periodic row strip of the configuration-2 mesh
    (same element size; every right-hand side, stage combination and error norm of the loop
    timed). The waves are not periodic across the strip's seam, so the controller settles
    near dt_CFL0.5 / 16: a span of 0.3 is a handful of accepted steps (about 6 s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from sgnb import workloads as W

    use_ref = O.reference_available()
    kw = W.cfg2_solver_args(2048, rows, 40.0, 20.0 * rows / 1024)
    kw.update(bc_x=0, bc_y=0)
    o = O.Oracle(reference=use_ref, **kw)
    U = W.cfg2_state_torch(2048, rows, 40.0, 20.0 * rows / 1024, device="cpu").numpy()
    dt0 = o.cfl_time_step(U, 0.5)
    t0 = time.perf_counter()
    _, st, _ = o.integrate_adaptive(U, 0.0, span * dt0, dt0)
    t = time.perf_counter() - t0
    dof = 5 * o.Nd
    return {"value": dof * st["rhsEvals"] / t, "unit": UNIT, "cores": 1,
            "kind": "reference" if use_ref else "port",
            "sample": f"integrateAdaptive over [0, {span} x dt_CFL0.5] of a 2048x{rows} "
                      f"periodic strip ({dof:,} DOF): {st['accepted']} accepted, "
                      f"{st['rejected']} rejected, {st['rhsEvals']} rhs, {t:.1f} s"}


# --------------------------------------------------------------------------- reference arm
def _ref_worker(args):
    """One single-core replica: right-hand sides of a row strip of the configuration-2
    mesh with the reference's CPU solver (its periodic boundary; per-DOF cost is the
    same), K+W evaluations, the last K timed."""
    rows, K, Wm, use_ref = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "sgn-hyperbolic-gpu_b200"))
    import numpy as np

    import oracle as O
    from sgnb import workloads as W

    kw = W.cfg2_solver_args(2048, rows, 40.0, 20.0 * rows / 1024)
    kw.update(bc_x=0, bc_y=0)
    o = O.Oracle(reference=use_ref, **kw)
    x, y = o.node_coords()
    shoal, (amp, lam, theta, phase) = W.cfg2_params()
    dx, dy = (x - shoal[2]) / shoal[4], (y - shoal[3]) / shoal[5]
    q = np.clip(1.0 - (dx * dx + dy * dy), 0.0, None)
    h = shoal[0] - (shoal[0] - shoal[1]) * q ** 3
    for A, L, T, P in zip(amp, lam, theta, phase):
        h = h + A * np.sin(2 * np.pi / L * (x * np.cos(T) + y * np.sin(T)) + P)
    z = np.zeros_like(h)
    U = o.make_state(h, z, z, z, z)
    for _ in range(Wm):
        o.rhs(U)
    t0 = time.perf_counter()
    for _ in range(K):
        o.rhs(U)
    return time.perf_counter() - t0, 5 * o.Nd


def run_reference_gpu(args, summary=False):
    """The reference's single-GPU solver (SGN2DCuda::integrateAdaptive, compiled from its
    sources by oracle/Makefile) on configuration 2 with periodic boundaries. summary: return
    the measurement (for the default line) instead of printing the reference line."""
    from sgnb import workloads as W

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_bench")
    if not os.path.exists(exe):
        why = ("oracle/_ref/ref_gpu_bench not built (make -C oracle refgpu needs the "
               "reference sources)")
        if summary:
            return {"unavailable": why}
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    Nx, Ny, Lx, Ly = W.CFG2["Nx"], W.CFG2["Ny"], W.CFG2["Lx"], W.CFG2["Ly"]
    if args.mesh:
        Nx, Ny = args.mesh
    shoal, waves = W.cfg2_params()
    argv = [exe, str(Nx), str(Ny), repr(Lx), repr(Ly), str(args.steps), "1"]
    argv += [repr(float(v)) for v in shoal]
    for arr in waves:
        argv += [repr(float(v)) for v in arr]
    with ClockSampler(0) as clk:
        out = subprocess.run(argv, check=True, capture_output=True, text=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    if summary:
        return {"solver": r["solver"], "value": r["value"], "unit": UNIT,
                "ms_per_step": r["time_s"] / max(r["accepted"], 1) * 1e3,
                "accepted": r["accepted"], "rejected": r["rejected"],
                "rhs_evals": r["rhsEvals"], "boundaries": "periodic (the reference's only kind)",
                "mesh": r["mesh"], "clocks": clk.summary()}
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT,
        "n_gpus": 1, "steps": int(r["accepted"]), "warmup": 1,
        "ms_per_step": r["time_s"] / max(r["accepted"], 1) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"configuration 2 mesh ({Nx}x{Ny} P=4), periodic boundaries, "
                               "the reference's single-GPU solver SGN2DCuda::integrateAdaptive "
                               f"over [0, {args.steps} x dt_CFL0.5]", "reference": r},
        "clocks": clk.summary(),
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # under torchrun the other ranks exit without work
    if args.ref_device == "gpu":
        run_reference_gpu(args)
        return
    import multiprocessing as mp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    use_ref = O.reference_available()
    P = os.cpu_count() or 1
    # size each replica's strip so that K + W evaluations take about two minutes
    budget_s = 120.0
    per_eval_s = budget_s / max(args.steps + args.warmup, 1)
    dof_rate = 2.5e7  # per core, order of magnitude of the reference CPU rhs
    rows = int(max(2, min(1024 // P, per_eval_s * dof_rate / (2048 * 125))))
    ctx = mp.get_context("spawn")
    with ctx.Pool(P) as pool:
        res = pool.map(_ref_worker, [(rows, args.steps, args.warmup, use_ref)] * P)
    tmax = max(t for t, _ in res)
    work = sum(d for _, d in res) * args.steps
    value = work / tmax
    sample = (f"{P} single-core replicas, each {args.steps} timed rhs evaluations of a "
              f"2048x{rows} row strip of the configuration-2 mesh "
              f"({res[0][1]:,} DOF), periodic")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tmax / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "configuration 2 mesh (2048x1024 P=4), reference CPU "
                               "right-hand side per RK stage", "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": P,
                         "kind": "reference" if use_ref else "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["sgnb", "reference"], default="sgnb")
    ap.add_argument("--precision", choices=["fast", "exact", "mixed"], default="fast")
    ap.add_argument("--workload", choices=["cfg2", "sweep", "mixed", "adjoint", "slabs"],
                    default="cfg2",
                    help="cfg2: the benchmark (default); sweep: the 256-instance batched "
                         "sweep against sequential single-instance runs; mixed: mixed vs "
                         "FP64 on configuration 2 with the eta error; adjoint: "
                         "configuration 5 forward + VJP; slabs: configuration 2 on x slabs "
                         "of one device against the whole mesh")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the sub-records of the default line (mixed, batched, adjoint, "
                         "reference GPU solver), e.g. for profiler captures")
    ap.add_argument("--bc", choices=["walls", "periodic"], default="walls",
                    help="boundaries of configuration 2 (periodic: the reference solver's "
                         "only kind, for the comparison with --ref-device gpu)")
    ap.add_argument("--ref-device", choices=["cpu", "gpu"], default="cpu",
                    help="reference arm: the reference's CPU solver (default) or its "
                         "single-GPU solver SGN2DCuda (oracle/_ref/ref_gpu_bench) on "
                         "configuration 2 with periodic boundaries")
    ap.add_argument("--mesh", type=int, nargs=2, metavar=("NX", "NY"), default=None,
                    help="smaller mesh of the same workload, for profiler captures only")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("sweep", "mixed", "adjoint", "slabs"):
        from sgnb import benchmarks as BW
        fn = {"sweep": BW.run_sweep, "mixed": BW.run_mixed, "adjoint": BW.run_adjoint,
              "slabs": BW.run_slabs}[args.workload]
        print(json.dumps(fn(args, ClockSampler, measured_peak_hbm())), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
