"""Profiling entry: repeated launches of one fused stage kernel on the benchmark workload.

    python sgn-hyperbolic-gpu_b200/sgnb/profile_stage.py --mesh 512 512 --stage 4 --count 3

sets up configuration 2 (elliptic shoal, 8 random-phase sines, walls) on the given mesh,
and launches the chosen kernel `count` times at the CFL-0.5 step size: stage 0 is the
right-hand side alone (R(u) -> dU), 2 and 3 the intermediate BS3(2) stages, 4 the
end-point stage (candidate, k4, error partials). Every launch does its full work (the
controller never runs, so no launch exits early), which is what a profiler capture of one
launch needs. Prints the CUDA-event time per launch.

    python sgn-hyperbolic-gpu_b200/sgnb/profile_stage.py --batch 8 --count 1

runs the batched stage kernels instead: the first N instances of configuration 4's sweep
(one autotune pass, `count` attempts per tile shape and grid form, each attempt the three
stage launches, all launched directly rather than inside the device-side loop's graph).
The first end-point launch is the 8x4-tile, one-CTA-per-tile form. Prints the
autotuner's time per attempt for each form.
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import torch  # noqa: E402

import sgnb  # noqa: E402
from sgnb import workloads as W  # noqa: E402


def profile_batch(a, prec):
    import numpy as np

    inst = W.cfg4_instances()[: a.batch]
    with sgnb.SGNBatch(inst, precision=prec) as b:
        for i, kw in enumerate(inst):
            b[i].upload_tensor(W.hump_shoal_state_torch(kw))
        dt0 = np.array([b[i].cfl_time_step(0.5) for i in range(len(inst))])
        tune = b.autotune(dt0, reps=a.count)
        dof = sum(125 * kw["Nx"] * kw["Ny"] for kw in inst)
        print(f"batch of {len(inst)} instances ({dof:,} DOF), {a.precision}: ms per attempt "
              f"[8x4, 16x2, 4x8] x [per tile, 1..4 per SM] = {np.round(tune, 4).tolist()}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, nargs=2, default=(512, 512))
    ap.add_argument("--stage", type=int, choices=(0, 2, 3, 4), default=4)
    ap.add_argument("--count", type=int, default=3)
    ap.add_argument("--precision", choices=("fast", "exact", "mixed"), default="fast")
    ap.add_argument("--batch", type=int, default=0,
                    help="profile the batched kernels on the sweep's first N instances")
    a = ap.parse_args()
    prec = {"fast": sgnb.FP64_FAST, "exact": sgnb.FP64_EXACT, "mixed": sgnb.MIXED}[a.precision]
    if a.batch > 0:
        profile_batch(a, prec)
        return
    Nx, Ny = a.mesh
    kw = W.cfg2_solver_args(Nx, Ny)
    with sgnb.SGN2DB200(precision=prec, **kw) as d:
        d.upload_tensor(W.cfg2_state_torch(Nx, Ny))
        dt = d.cfl_time_step(0.5)
        _, sp = d.state_device_ptr()
        stream = torch.cuda.ExternalStream(sp)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if a.stage == 0:
            u, _ = d.state_device_ptr()
            out = torch.empty(d.n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(a.count):
                d.rhs_device(u, out.data_ptr())
            e1.record(stream)
        else:
            torch.cuda.synchronize()
            e0.record(stream)
            d.launch_stage(a.stage, dt, a.count)
            e1.record(stream)
        torch.cuda.synchronize()
        print(f"mesh {Nx}x{Ny} stage {a.stage} {a.precision}: "
              f"{e0.elapsed_time(e1) / a.count:.4f} ms per launch")


if __name__ == "__main__":
    main()
