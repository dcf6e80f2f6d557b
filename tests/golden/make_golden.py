"""Generate the golden fixtures of tests/golden/ by running the reference's own CPU solver.

Test infrastructure. Needs oracle/_ref/libsgnref.so, built from the reference sources by
``make -C oracle ref`` (that tree exists only on the machine that builds the fixtures);
the fixtures are committed so the tests never need the reference at run time.

    python tests/golden/make_golden.py

Fixtures (golden.npz):
  bump_*        the GPU-parity case of the reference's test/test_cuda_sgn2d.cu:38-64
                (8x6 elements on 10x8, Gaussian bump H = 1 - 0.4 exp(-r^2/6), smooth
                state): the state, its rhs, and bathymetry arrays
  wall_*        the same state on reflective walls (reference on the mirror-doubled domain)
  cfg1_*        configuration 1 (128x64 on 20x10, flat H = 1, Gaussian hump): sha256 of the
                rhs bytes, 64 sampled entries, the adaptive run to 100 accepted steps
                (stats, the accepted step sizes, sha256 + samples of the final state)
  run_*         a short adaptive run of the bump case (tEnd 0.05, atol 1e-10, rtol 1e-8)
  gauss_*       Gauss-Legendre points (tests/cases.py gauss_case, flat bottom H = 0): the
                FR tables, the state and its rhs, periodic; the same short adaptive run
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from cases import bump_case, cfg1_case, gauss_case, CFG1_STEPS  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main() -> None:
    if not O.reference_available():
        raise SystemExit("oracle/_ref/libsgnref.so is missing: run `make -C oracle ref` first")
    out = {}
    # --- bump case, periodic and walls -------------------------------------------
    for tag, bc in (("bump", O.BC_PERIODIC), ("wall", O.BC_WALL)):
        kw, U = bump_case(bc)
        ref = O.Oracle(reference=True, **kw)
        R = ref.rhs(U)
        out[f"{tag}_U"] = U
        out[f"{tag}_R"] = R
        b = ref.bathymetry()
        for k in ("Hnod", "Hx", "Hy", "HfaceX", "HfaceY"):
            out[f"{tag}_{k}"] = b[k]
        if bc == O.BC_WALL:
            out[f"{tag}_HfaceXEnd"] = b["HfaceXEnd"]
            out[f"{tag}_HfaceYEnd"] = b["HfaceYEnd"]
    # --- short adaptive run of the bump case ----------------------------------------
    kw, U = bump_case(O.BC_PERIODIC)
    ref = O.Oracle(reference=True, **kw)
    dt0 = ref.cfl_time_step(U, 0.5)
    u, st, _ = ref.integrate_adaptive(U, 0.0, 0.05, dt0, atol=1e-10, rtol=1e-8)
    out["run_dt0"] = np.array([dt0])
    out["run_stats"] = np.array([st["accepted"], st["rejected"], st["rhsEvals"]], dtype=np.int64)
    out["run_U"] = u
    # --- Gauss-Legendre points ------------------------------------------------------------
    kw, U = gauss_case()
    ref = O.Oracle(reference=True, **kw)
    for k, a in ref.tables().items():
        out[f"gauss_{k}"] = a
    out["gauss_U"] = U
    out["gauss_R"] = ref.rhs(U)
    dt0 = ref.cfl_time_step(U, 0.5)
    u, st, _ = ref.integrate_adaptive(U, 0.0, 0.05, dt0, atol=1e-10, rtol=1e-8)
    out["gauss_run_stats"] = np.array([st["accepted"], st["rejected"], st["rhsEvals"]],
                                      dtype=np.int64)
    out["gauss_run_U"] = u
    # --- configuration 1 -----------------------------------------------------------------
    kw, U = cfg1_case()
    ref = O.Oracle(reference=True, **kw)
    R = ref.rhs(U)
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(R.size, 64, replace=False))
    out["cfg1_rhs_sha"] = np.array([sha(R)])
    out["cfg1_idx"] = idx
    out["cfg1_rhs_samples"] = R[idx]
    dt0 = ref.cfl_time_step(U, 0.5)
    # the restatement's attempt log gives the time of the 100th accepted step; the
    # reference then integrates to exactly that time
    mine = O.Oracle(**kw)
    _, _, log = mine.integrate_adaptive(U, 0.0, 1e9 * dt0, dt0, max_log=4 * CFG1_STEPS,
                                        stop_after=CFG1_STEPS)
    acc = log[log[:, 3] == 1]
    tEnd = float(acc[CFG1_STEPS - 1, 0] + acc[CFG1_STEPS - 1, 1])
    u, st, _ = ref.integrate_adaptive(U, 0.0, tEnd, dt0)
    assert st["accepted"] == CFG1_STEPS, st
    out["cfg1_dts"] = acc[:CFG1_STEPS, 1].copy()  # the accepted step sizes, in order
    out["cfg1_dt0"] = np.array([dt0])
    out["cfg1_tEnd"] = np.array([tEnd])
    out["cfg1_stats"] = np.array([st["accepted"], st["rejected"], st["rhsEvals"]], dtype=np.int64)
    out["cfg1_final_sha"] = np.array([sha(u)])
    out["cfg1_final_samples"] = u[idx]
    out["cfg1_mass"] = np.array([ref.mass(U), ref.mass(u)])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), "tEnd", tEnd, "stats", st)


if __name__ == "__main__":
    main()
