"""Measurements of the batched sweep, the mixed-precision form and the adjoint, each
returning one JSON line in the format of bench.py (which prints it for --workload
sweep | mixed | adjoint | slabs, and folds summaries of all four into its default line
through default_extras). Every number is taken on the device with CUDA events on the
stream the work runs on, after warm-up, with the state resident in HBM.

sweep    configuration 4: 256 instances (workloads.cfg4_instances) advanced K accepted
         steps each by the batched launches (after the autotuner), against the same
         instances run one after another through the single-instance device loop; FP64
         (fast) or, with --precision mixed, the mixed-precision form on both sides.
mixed    configuration 2 in FP64 (fast) and in the mixed-precision mode, K steps each,
         and the free-surface error of the mixed mode against FP64: every mode replays
         two step sequences from the same state (constant 0.4 x the CFL-0.5 step, and the
         FP64 run's accepted steps), with FP64 fast against FP64 exact as the control;
         eta L2 (RMS over the nodes) and Linf of the differences.
adjoint  configuration 5: the frozen 200-step trajectory with 16 gauges (forward), its
         vector-Jacobian product (checkpoint-and-recompute every 20 steps), and one
         central-difference check of a directional derivative.
"""
from __future__ import annotations

import hashlib
import math
import time

import numpy as np

from . import FP64_FAST, MIXED, SGN2DB200, SGNBatch, SgnbError
from . import workloads as W

METRIC = "DOF-updates/s per RK stage"
UNIT = "DOF-updates/s"
# algorithmic bytes per DOF of one fused BS3(2) attempt (two intermediate stages and the
# end-point stage; nodal depth gradients formed on chip): FP64 and mixed precision
STAGE_LOOP_BYTES = 2 * 26.24 + 50.24
MIXED_LOOP_BYTES = 2 * 18.24 + 34.24


def _rel_per_field(a, b):
    """max over fields of max|a - b| / max|b| (each field's error over its largest value)."""
    a, b = a.view(5, -1), b.view(5, -1)
    out = 0.0
    for v in range(5):
        s = float(b[v].abs().max())
        out = max(out, float((a[v] - b[v]).abs().max()) / (s if s > 0 else 1.0))
    return out


def _events(torch, stream=None):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    return e0, e1


def run_sweep(args, clock_sampler, peak):
    import torch

    inst = W.cfg4_instances()
    n = len(inst)
    mixed = args.precision == "mixed"
    b = SGNBatch(inst, precision=MIXED if mixed else FP64_FAST)
    dofs = np.array([125.0 * k["Nx"] * k["Ny"] for k in inst])
    dt0 = np.zeros(n)

    def reset():
        for i, kw in enumerate(inst):
            b[i].upload_tensor(W.hump_shoal_state_torch(kw))
        torch.cuda.synchronize()

    reset()
    for i in range(n):
        dt0[i] = b[i].cfl_time_step(0.5)
    tune = b.autotune(dt0, reps=3)
    b.integrate_steps(dt0, args.warmup)
    reset()
    stream = torch.cuda.ExternalStream(b.stream)
    e0, e1 = _events(torch, stream)
    torch.cuda.synchronize()
    with clock_sampler(0) as clk:
        e0.record(stream)
        st = b.integrate_steps(dt0, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / 1e3
    rhs = np.array([s.rhsEvals for s in st], dtype=np.float64)
    value = float((dofs * rhs).sum() / t_batch)
    # the same instances and steps, one after another through the single-instance loop
    reset()
    for i in range(n):  # warm each context's graph
        b[i].integrate_steps(0.0, dt0[i], 1)
    reset()
    t_seq = 0.0
    rhs_seq = 0.0
    for i in range(n):
        _, sp = b[i].state_device_ptr()
        s_i = torch.cuda.ExternalStream(sp)
        a0, a1 = _events(torch, s_i)
        a0.record(s_i)
        si = b[i].integrate_steps(0.0, dt0[i], args.steps)
        a1.record(s_i)
        torch.cuda.synchronize()
        t_seq += a0.elapsed_time(a1) / 1e3
        rhs_seq += dofs[i] * si.rhsEvals
    seq_value = rhs_seq / t_seq
    shape, blocks = b.config
    best_ms = float(tune[tune > 0].min())  # -1 marks shapes a mixed batch does not use
    achieved = (MIXED_LOOP_BYTES if mixed else STAGE_LOOP_BYTES) * dofs.sum() / (best_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_batch / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 state, f32 deviations" if mixed else "f64", "data": "synthetic",
        "config": {"workload": "configuration 4: 256 instances (Nx U{64..512}, Ny U{32..256}, "
                               "alpha U[1.5,6], shoal crest U[0.3,0.9], Gaussian hump), "
                               "walls, per-instance adaptive BS3(2), K accepted steps each",
                   "instances": n, "dof_total": int(dofs.sum()),
                   "tile_shape": ["8x4", "16x2", "4x8"][shape],
                   "grid": "one CTA per tile" if blocks == 0 else f"{blocks} persistent CTAs",
                   "rejected": int(sum(s.rejected for s in st)),
                   "l2": f"inputs larger than L2 ({8 * dofs.sum() / 1e9:.1f} GB per state)"},
        "sequential_single_instance": {"value": seq_value, "unit": UNIT, "time_s": t_seq},
        "speedup_vs_sequential": value / seq_value,
        "autotune_ms_per_attempt": {"shapes": ["8x4", "16x2", "4x8 (-1: not used)"],
                                    "grids": ["per tile", "1/SM", "2/SM", "3/SM", "4/SM"],
                                    "ms": np.round(tune, 3).tolist()},
        "roofline": {"bound": "hbm", "kernel": "batched stage kernels, one attempt",
                     "achieved": round(achieved, 1), "peak": peak[0], "peak_kind": peak[1],
                     "unit": "GB/s", "frac": round(achieved / peak[0], 4), "traffic": None},
        "clocks": clk.summary(),
        "gpu_launches": int(st[0].kernel_launches),
    }
    b.close()
    return line


def run_mixed(args, clock_sampler, peak):
    import torch

    from . import FP64_EXACT

    Nx, Ny = W.CFG2["Nx"], W.CFG2["Ny"]
    if args.mesh:
        Nx, Ny = args.mesh
    kw = W.cfg2_solver_args(Nx, Ny)
    dof = 125.0 * Nx * Ny
    Ud = W.cfg2_state_torch(Nx, Ny)
    res = {}
    seqs = {}
    finals = {"adaptive": {}, "stable": {}}
    full = {}
    replay = {}
    clocks = None
    for name, prec in (("fp64", FP64_FAST), ("mixed", MIXED), ("exact", FP64_EXACT)):
        with SGN2DB200(precision=prec, **kw) as d:
            d.upload_tensor(Ud)
            dt0 = d.cfl_time_step(0.5)
            if name != "exact":
                d.integrate_steps(0.0, dt0, args.warmup)
                d.upload_tensor(Ud)
                _, sp = d.state_device_ptr()
                stream = torch.cuda.ExternalStream(sp)
                e0, e1 = _events(torch, stream)
                torch.cuda.synchronize()
                with clock_sampler(0) as clk:
                    e0.record(stream)
                    st = d.integrate_steps(0.0, dt0, args.steps)
                    e1.record(stream)
                    torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / 1e3
                res[name] = dict(value=dof * st.rhsEvals / t, time_s=t, accepted=st.accepted,
                                 rejected=st.rejected, launches=st.kernel_launches)
                if name == "mixed":
                    clocks = clk.summary()
            if name == "fp64":
                log = d.attempt_log()
                seqs["adaptive"] = log[log[:, 3] == 1][:, 1].copy()
                seqs["stable"] = np.full(len(seqs["adaptive"]), 0.4 * dt0)
            # free surface after each step sequence, from the same state (the adaptive
            # sequence's replay timed, after the stable one has warmed the kernels up: the
            # exact mode's throughput beside the fast one's)
            for key in ("stable", "adaptive"):
                dts = seqs[key]
                d.upload_tensor(Ud)
                try:
                    _, sp = d.state_device_ptr()
                    stream = torch.cuda.ExternalStream(sp)
                    e0, e1 = _events(torch, stream)
                    torch.cuda.synchronize()
                    e0.record(stream)
                    d.bs3_steps(0.0, dts)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    if key == "adaptive":
                        replay[name] = dof * 3 * len(dts) / (e0.elapsed_time(e1) / 1e3)
                    finals[key][name] = d.state_tensor()[: d.Nd].clone()  # h
                    if key == "adaptive" and name in ("fp64", "exact"):
                        full[name] = d.state_tensor().clone()
                except SgnbError:  # the replay left the stable range (non-finite state)
                    finals[key][name] = None

    def err(key, a, b):
        if finals[key][a] is None or finals[key][b] is None:
            return {"diverged": [n for n in (a, b) if finals[key][n] is None]}
        diff = (finals[key][a] - finals[key][b]).double()  # eta differences = h differences
        return {"l2_rms": float(torch.sqrt(torch.mean(diff * diff))),
                "linf": float(diff.abs().max())}

    errors = {
        "stable_steps": {"mixed_vs_fp64": err("stable", "mixed", "fp64"),
                         "fp64_fast_vs_exact": err("stable", "fp64", "exact"),
                         "steps": "constant 0.4 x the CFL-0.5 step"},
        "adaptive_steps": {"mixed_vs_fp64": err("adaptive", "mixed", "fp64"),
                           "fp64_fast_vs_exact": err("adaptive", "fp64", "exact"),
                           "steps": "the FP64 run's accepted step sizes (near the stability "
                                    "limit: round-off of any kind is amplified)"},
        "how": "each mode replays the step sequence from the same state (bs3 steps)",
    }
    # fingerprint of the exact mode's final state (bit-identical to the reference's CPU
    # solver on the same steps) and the fast mode's largest relative difference per field
    if "exact" in full:
        ex = full["exact"].cpu().numpy()
        errors["exact_state"] = {
            "sha256": hashlib.sha256(ex.tobytes()).hexdigest(),
            "steps": int(len(seqs["adaptive"])),
            "fast_rel_diff_per_field": (
                _rel_per_field(full["fp64"], full["exact"]) if "fp64" in full else None)}
    ratio = res["mixed"]["value"] / res["fp64"]["value"]
    achieved = MIXED_LOOP_BYTES * res["mixed"]["value"] / 3.0 / 1e9  # bytes per attempt
    line = {
        "metric": METRIC, "value": res["mixed"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["mixed"]["time_s"] / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 state, f32 deviations",
        "data": "synthetic",
        "config": {"workload": f"configuration 2 ({Nx}x{Ny}, {int(dof):,} DOF), mixed "
                               "precision against FP64 (fast)", "mesh": [Nx, Ny]},
        "fp64": res["fp64"], "mixed": res["mixed"], "speedup_vs_fp64": ratio,
        "replay_value": {"how": "the FP64 run's accepted step sizes replayed as frozen BS3 "
                                "steps (3 right-hand sides each), CUDA events", **replay},
        "eta_error": errors,
        "roofline": {"bound": "hbm", "kernel": "mixed stage loop (average over an attempt)",
                     "achieved": round(achieved, 1), "peak": peak[0], "peak_kind": peak[1],
                     "unit": "GB/s", "frac": round(achieved / peak[0], 4), "traffic": None},
        "clocks": clocks,
        "gpu_launches": int(res["mixed"]["launches"]),
    }
    return line


def run_adjoint(args, clock_sampler, peak):
    import torch

    from . import adjoint as ADJ

    cfg = W.CFG5
    P = W.cfg5_problem()
    kw = P["kw"]
    d = SGN2DB200(precision=FP64_FAST, **kw)
    x, y = W.node_coords_np(cfg["Nx"], cfg["Ny"], cfg["Lx"], cfg["Ly"])
    # initial state on the cell-mean bathymetry, then the frozen accepted steps
    from . import setup_bathymetry
    H = setup_bathymetry(**{k: kw[k] for k in ("P", "Nx", "Ny", "Lx", "Ly", "bc_x", "bc_y",
                                              "bathy_kind", "bathy_par")})["Hnod"]
    z = np.zeros_like(H)
    d.upload(SGN2DB200.make_state(H + P["eta0"], z, z, z, z))
    dt0 = d.cfl_time_step(0.5)
    d.integrate_steps(0.0, dt0, cfg["steps"])
    log = d.attempt_log()
    dts = log[log[:, 3] == 1][:, 1].copy()
    A = ADJ.SGNAdjoint(d, dts, P["gauges"], cfg["checkpoint"])
    target = A.forward(P["target_means"], P["target_eta0"])
    for _ in range(max(args.warmup, 1)):
        eta = A.forward(P["means"], P["eta0"])
        A.vjp(2 * (eta - target))
    torch.cuda.synchronize()
    reps = max(1, min(args.steps, 20))
    with clock_sampler(0) as clk:
        t0 = time.perf_counter()
        for _ in range(reps):
            eta = A.forward(P["means"], P["eta0"])
        t_fwd = (time.perf_counter() - t0) / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            gm, ge = A.vjp(2 * (eta - target))
        t_vjp = (time.perf_counter() - t0) / reps
    # one directional derivative against central differences (smooth eta0 direction)
    rng = np.random.default_rng(7)
    de = np.zeros_like(x)
    for _ in range(12):
        kx, ky = rng.integers(0, 5, 2) * 2 * np.pi / np.array([cfg["Lx"], cfg["Ly"]])
        de += rng.standard_normal() * np.cos(kx * x + ky * y + rng.uniform(0, 2 * np.pi))
    de *= 0.01 / math.sqrt(12)
    adj = float(ge @ de)
    eps = 1e-5
    Lp = float(((A.forward(P["means"], P["eta0"] + eps * de) - target) ** 2).sum())
    Lm = float(((A.forward(P["means"], P["eta0"] - eps * de) - target) ** 2).sum())
    fd = (Lp - Lm) / (2 * eps)
    dof = 125.0 * cfg["Nx"] * cfg["Ny"]
    N = len(dts)
    line = {
        "metric": METRIC, "value": dof * 4 * N / t_fwd, "unit": UNIT, "n_gpus": 1,
        "steps": N, "warmup": args.warmup, "ms_per_step": t_fwd / N * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "configuration 5: 256x128, 200 frozen BS3(2) steps from an "
                               "adaptive run, 16 gauges, checkpoints every 20 steps; value "
                               "counts the forward's 4 right-hand sides per step",
                   "gradient_sizes": {"means": int(gm.size), "eta0": int(ge.size)}},
        "forward_s": t_fwd, "vjp_s": t_vjp, "vjp_over_forward": t_vjp / t_fwd,
        "fd_check": {"direction": "smooth random eta0 field", "eps": eps, "fd": fd,
                     "adjoint": adj, "rel_err": abs(fd - adj) / max(abs(fd), abs(adj))},
        "clocks": clk.summary(), "roofline": None, "gpu_launches": None,
        "timing": "host wall clock around synchronous C-ABI calls (forward and vjp each "
                  "synchronise at the end)",
    }
    A.close()
    d.close()
    return line


def run_slabs(args, clock_sampler, peak, counts=(1, 2, 4),
              fused_runs=((2, "per-slab"), (2, "shared"), (4, "per-slab"), (4, "shared"))):
    """Configuration 2 on x slabs of one device (1, 2 and 4 slabs: the edge exchange and
    the partial gather between slabs are device copies on the solver's stream, every
    stage launched from the host), against the whole-mesh device loop: K accepted steps
    each from the same state, throughput and the largest relative difference per field
    of the final states."""
    import torch

    from .slabs import PeerSlabSolver, SlabSolver

    Nx, Ny = W.CFG2["Nx"], W.CFG2["Ny"]
    if args.mesh:
        Nx, Ny = args.mesh
    kw = dict(W.cfg2_solver_args(Nx, Ny), precision=FP64_FAST)
    dof = 125.0 * Nx * Ny
    Ud = W.cfg2_state_torch(Nx, Ny)

    def rel(a, b):
        a, b = a.view(5, -1), b.view(5, -1)
        out = 0.0
        for v in range(5):
            s = float(b[v].abs().max())
            out = max(out, float((a[v] - b[v]).abs().max()) / (s if s > 0 else 1.0))
        return out

    with SGN2DB200(**kw) as d:
        d.upload_tensor(Ud)
        dt0 = d.cfl_time_step(0.5)
        d.integrate_steps(0.0, dt0, args.warmup)
        d.upload_tensor(Ud)
        _, sp = d.state_device_ptr()
        stream = torch.cuda.ExternalStream(sp)
        e0, e1 = _events(torch, stream)
        torch.cuda.synchronize()
        e0.record(stream)
        st = d.integrate_steps(0.0, dt0, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        whole = dict(value=dof * st.rhsEvals / t, ms_per_step=t / args.steps * 1e3,
                     accepted=st.accepted, rejected=st.rejected)
        ref = d.state_tensor().clone()
    slabs = {}
    clocks = None
    for n in counts:
        with SlabSolver(kw, nslabs=n) as s:
            s.upload_tensor(Ud)
            s.integrate_steps(0.0, dt0, args.warmup)
            s.upload_tensor(Ud)
            e0, e1 = _events(torch, s.stream)
            torch.cuda.synchronize()
            with clock_sampler(0) as clk:
                e0.record(s.stream)
                st = s.integrate_steps(0.0, dt0, args.steps)
                e1.record(s.stream)
                torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            slabs[str(n)] = dict(value=dof * st.rhsEvals / t, ms_per_step=t / args.steps * 1e3,
                                 accepted=st.accepted, rejected=st.rejected,
                                 rel_diff_vs_whole=rel(s.download_tensor(), ref))
            clocks = clk.summary()
    # the fused edge exchange: stage kernels store the neighbours' ghosts, controllers read
    # every slab's partials in place; one stream per slab (ordered by events) or one shared
    fused = {}
    for n, mode in fused_runs:
        with PeerSlabSolver(kw, nslabs=n, streams=mode) as s:
            s.upload_tensor(Ud)
            s.integrate_steps(0.0, dt0, args.warmup)
            s.upload_tensor(Ud)
            e0, e1 = _events(torch, s.stream)
            torch.cuda.synchronize()
            e0.record(s.stream)
            st = s.integrate_steps(0.0, dt0, args.steps)
            e1.record(s.stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            fused[f"{n} {mode}"] = dict(value=dof * st.rhsEvals / t,
                                       ms_per_step=t / args.steps * 1e3,
                                       accepted=st.accepted, rejected=st.rejected,
                                       rel_diff_vs_whole=rel(s.download_tensor(), ref))
    nmax = max(counts)
    top = slabs[str(nmax)]
    edge_bytes = 5 * Ny * 5 * 8
    line = {
        "metric": METRIC, "value": top["value"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": top["ms_per_step"],
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"configuration 2 ({Nx}x{Ny}, walls, adaptive BS3(2)) on "
                               f"{nmax} x slabs of one device; the whole-mesh loop and "
                               f"{', '.join(str(n) for n in counts if n != nmax) or 'no other'} "
                               "slab counts beside it",
                   "edge_bytes": edge_bytes,
                   "exchange_bytes_per_attempt_per_slab": 3 * 2 * edge_bytes,
                   "l2": f"inputs larger than L2 ({8 * 5 * dof / 1e9:.1f} GB per state)"},
        "whole_mesh": whole, "slabs": slabs, "fused_exchange": fused,
        "slab_over_whole": {k: v["value"] / whole["value"] for k, v in slabs.items()},
        "clocks": clocks, "roofline": None, "gpu_launches": None,
        "timing": "CUDA events on the solver's stream around the K steps (the host launches "
                  "every stage and reads the controller every 4 attempts)",
    }
    return line


def default_extras(args, clock_sampler, peak):
    """Summaries of the mixed-precision, batched and adjoint measurements for the default
    benchmark line, each with the same K and W as the main measurement (the adjoint's
    timing repeats at most 3 times). A measurement that fails records its error instead."""
    import copy
    import gc

    import torch

    out = {}
    a = copy.copy(args)
    a.mesh, a.precision = None, "fast"

    def timed(name, fn, summary):
        t0 = time.perf_counter()
        try:
            r = summary(fn(a, clock_sampler, peak))
        except Exception as e:  # recorded, the main measurement stands
            r = {"error": f"{type(e).__name__}: {e}"}
        r["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = r
        gc.collect()
        torch.cuda.empty_cache()

    timed("mixed", run_mixed, lambda m: {
        "value": m["value"], "fp64_value_same_run": m["fp64"]["value"],
        "ratio_vs_fp64": m["speedup_vs_fp64"], "steps": m["steps"],
        "replay_value": m["replay_value"],
        "eta_error": m["eta_error"], "roofline": m["roofline"], "clocks": m["clocks"]})
    timed("batched", run_sweep, lambda s: {
        "value": s["value"], "sequential_value": s["sequential_single_instance"]["value"],
        "ratio_vs_sequential": s["speedup_vs_sequential"], "steps": s["steps"],
        "instances": s["config"]["instances"], "dof_total": s["config"]["dof_total"],
        "tile_shape": s["config"]["tile_shape"], "grid": s["config"]["grid"],
        "roofline": s["roofline"], "clocks": s["clocks"]})
    # the same sweep in mixed precision, against the same instances run one after another
    # in plain FP64 (the batched record's sequential runs) and in mixed precision
    a_mix = copy.copy(a)
    a_mix.precision = "mixed"
    seq64 = out["batched"].get("sequential_value")
    timed("batched_mixed", lambda _a, c, p: run_sweep(a_mix, c, p), lambda s: {
        "value": s["value"], "sequential_fp64_value": seq64,
        "ratio_vs_sequential_fp64": s["value"] / seq64 if seq64 else None,
        "sequential_mixed_value": s["sequential_single_instance"]["value"],
        "ratio_vs_sequential_mixed": s["speedup_vs_sequential"], "steps": s["steps"],
        "tile_shape": s["config"]["tile_shape"], "grid": s["config"]["grid"],
        "roofline": s["roofline"], "clocks": s["clocks"]})
    # x slabs of one device: 4 slabs with copies between them and with the fused exchange
    timed("slabs", lambda _a, c, p: run_slabs(_a, c, p, counts=(4,), fused_runs=((4, "per-slab"),)),
          lambda s: {"whole_mesh": s["whole_mesh"], "slabs": s["slabs"],
                     "fused_exchange": s["fused_exchange"],
                     "slab_over_whole": s["slab_over_whole"], "clocks": s["clocks"],
                     "timing": s["timing"]})
    a_adj = copy.copy(a)
    a_adj.steps = min(a.steps, 3)
    a_adj.warmup = 1
    timed("adjoint", lambda _a, c, p: run_adjoint(a_adj, c, p), lambda j: {
        "forward_ms": j["forward_s"] * 1e3, "vjp_ms": j["vjp_s"] * 1e3,
        "vjp_over_forward": j["vjp_over_forward"], "fd_check": j["fd_check"],
        "steps": j["steps"], "timing": j["timing"]})
    return out
