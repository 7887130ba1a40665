"""Time the reference's own source against the oracle port on the CPU, on the
1M-triangle RK3 microbenchmark (or a smaller sample of it).

The GPU box has no copy of the reference, so the benchmark's CPU baseline
and reference arm run the oracle (the NumPy restatement under ``oracle/``).
This script, run where the CFD-demo source tree is available, times the
reference's own ``ssp_rk3_step`` (under the NumPy stand-in for ``jax`` that
make_golden.py uses; JAX itself is not installed) and the oracle's step on
the same mesh and state, one process each, so that the port's numbers can be
read as the reference's:

    python tests/golden/time_reference.py --reference PATH [--nx 724] [--steps 3]

Prints one JSON line: seconds per RK3 step of each, DOF-steps/s, and the
largest relative difference between the two final states.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the CFD-demo source tree")
    ap.add_argument("--nx", type=int, default=724)
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()

    from make_golden import load_reference

    ref = load_reference(args.reference)
    import oracle
    from cfd_demo_b200.workloads import GAMMA, MEAN_STATE, conserved_fields, microbenchmark_mesh
    from oracle.physics import FixedState as OFixed

    mesh = microbenchmark_mesh(args.nx)
    v, e = np.array(mesh.vertices), np.array(mesh.elements)
    edges = {k: np.array(x) for k, x in mesh.boundary_edges.items()}

    t0 = time.perf_counter()
    rmesh = ref["mesh"].TriangleMesh(vertices=v, elements=e, boundary_edges=edges)
    rmean = ref["boundary"].FixedState.from_primitive(*MEAN_STATE, GAMMA)
    rcfg = ref["solver"].SolverConfig(flux="roe", limiter="unlimited", gamma=GAMMA)
    rsolver = ref["solver"].EulerSolver(rmesh, {t: rmean for t in ("left", "right", "bottom", "top")}, rcfg)
    ref_setup = time.perf_counter() - t0

    t0 = time.perf_counter()
    omesh = oracle.mesh.TriangleMesh(v, e, edges)
    omean = OFixed.from_primitive(*MEAN_STATE, GAMMA)
    osolver = oracle.OracleSolver(omesh, {t: omean for t in ("left", "right", "bottom", "top")}, flux="roe",
                                  limiter="unlimited", gamma=GAMMA)
    port_setup = time.perf_counter() - t0

    x, y = osolver.node_coordinates()
    q0 = conserved_fields(x, y, np)
    k = osolver.mesh.num_elements

    def march(step_fn, dt_fn):
        q = q0
        t = time.perf_counter()
        for _ in range(args.steps):
            q, _ = step_fn(q, float(dt_fn(q)))
        return (time.perf_counter() - t) / args.steps, np.asarray(q)

    ref_s, ref_q = march(rsolver.step, rsolver.time_step)
    port_s, port_q = march(osolver.step, osolver.time_step)
    scale = np.maximum(np.abs(ref_q).reshape(-1, 4).max(axis=0), 1e-300)
    print(json.dumps({
        "workload": f"{args.nx}x{args.nx} quads x 2 (K={k}), jitter 0.2h, 8-mode Fourier fields, roe/unlimited",
        "steps": args.steps, "threads": "one process (NumPy; BLAS threads as configured)",
        "reference_s_per_step": ref_s, "port_s_per_step": port_s,
        "reference_dof_steps_per_s": k * 15 / ref_s, "port_dof_steps_per_s": k * 15 / port_s,
        "port_over_reference_speed": ref_s / port_s,
        "setup_s": {"reference": ref_setup, "port": port_setup},
        "max_rel_state_difference": float((np.abs(ref_q - port_q) / scale).max()),
    }), flush=True)


if __name__ == "__main__":
    main()
