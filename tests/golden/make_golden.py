"""Generate the golden fixtures of the CFD-demo hot path from the reference's
own source.

Run in a container that has the CFD-demo source tree (its path is the
required ``--reference`` argument) but no JAX: ``numpy_jax.install()`` puts a NumPy stand-in
for ``jax`` in ``sys.modules`` and the reference's modules are imported and
called unchanged. The outputs are small ``.npz`` files beside this script;
the tests read them on machines without the reference.

    python tests/golden/make_golden.py --reference PATH [--only NAME ...]

Fixtures (all float64 unless noted):
  element.npz      reference-triangle tables
  pointwise.npz    interface fluxes and phi(r) on seeded and edge-case inputs
  rhs.npz          dg_rhs (rhs, boundary flux) for 4 mesh/BC/state cases x 3 fluxes
  limit.npz        apply_limiters for 4 cases x 5 limiters (+ troubled flags)
  step.npz         one SSP-RK3 step for every flux x limiter pair
  sod_short.npz    run() of the 20x2 Sod-like case to t = 0.01
  sod_100x10.npz  run() of the 100x10 Sod tube to t = 0.2 (rusanov/minmod),
                   with per-step dt, report and per-stage troubled counts and
                   the troubled flags of the first 25 steps
  sod_100x10_flags.npz  the same run's troubled flags at every stage of every
                   step (bit-packed, each stage XOR the previous one) and its
                   borderline detection decisions: every element whose
                   largest excess / threshold ratio lies within 1e-3 of one
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy_jax  # noqa: E402

FLUXES = ("rusanov", "roe", "hllc")
LIMITERS = ("minmod", "mc", "van_leer", "superbee", "unlimited")
GAMMA = 1.4
FREE_STREAM = (1.2, 0.4, -0.3, 0.9)


def load_reference(path: str):
    numpy_jax.install()
    sys.path.insert(0, os.path.join(path, "src"))
    import cfd_demo  # noqa: F401
    from cfd_demo import boundary, cases, dg, euler, fluxes, limiters, limiting, mesh, reference_element, solver

    return dict(boundary=boundary, cases=cases, dg=dg, euler=euler, fluxes=fluxes, limiters=limiters,
                limiting=limiting, mesh=mesh, reference_element=reference_element, solver=solver)


def perturbed(ref, nx, ny, amplitude=0.25, seed=0):
    """Same construction as the reference tests' perturbed_mesh helper."""
    m = ref["mesh"].rectangle_mesh(nx, ny)
    v = np.array(m.vertices)
    inside = np.all((v > 1e-12) & (v < 1.0 - 1e-12), axis=1)
    rng = np.random.default_rng(seed)
    d = rng.uniform(-1.0, 1.0, size=v.shape)
    v[inside] += amplitude * d[inside] / np.array([nx, ny])
    return ref["mesh"].TriangleMesh(vertices=v, elements=m.elements, boundary_edges=m.boundary_edges)


def mesh_arrays(prefix, m):
    out = {f"{prefix}/vertices": np.asarray(m.vertices), f"{prefix}/elements": np.asarray(m.elements)}
    for tag, pairs in m.boundary_edges.items():
        out[f"{prefix}/edges/{tag}"] = np.asarray(pairs)
    return out


def bc_arrays(prefix, conditions):
    out = {}
    for tag, c in conditions.items():
        out[f"{prefix}/bc/{tag}"] = np.array([c.kind, *(c.state if c.kind == 2 else (0, 0, 0, 0))], dtype=np.float64)
    return out


def fixed_all(ref, primitive):
    c = ref["boundary"].FixedState.from_primitive(*primitive, GAMMA)
    return {t: c for t in ("left", "right", "bottom", "top")}


def walls_all(ref):
    return {t: ref["boundary"].SlipWall() for t in ("left", "right", "bottom", "top")}


def sod_bcs(ref):
    fs = ref["boundary"].FixedState
    return {"left": fs.from_primitive(1.0, 0.0, 0.0, 1.0, GAMMA), "right": fs.from_primitive(0.125, 0.0, 0.0, 0.1, GAMMA),
            "bottom": ref["boundary"].SlipWall(), "top": ref["boundary"].SlipWall()}


def make_solver(ref, m, bcs, flux="rusanov", limiter="minmod", cfl=0.5):
    cfg = ref["solver"].SolverConfig(flux=flux, limiter=limiter, gamma=GAMMA, cfl=cfl)
    return ref["solver"].EulerSolver(m, bcs, cfg)


def random_state(ref, solver, seed, lo=(0.5, -0.4, -0.4, 0.5), hi=(1.5, 0.4, 0.4, 1.5)):
    rng = np.random.default_rng(seed)
    prim = rng.uniform(lo, hi, size=solver.state_shape[:2] + (4,))
    return np.asarray(ref["euler"].primitive_to_conserved(*(prim[..., k] for k in range(4)), GAMMA))


def sod_state(ref, solver):
    left = np.asarray(ref["euler"].primitive_to_conserved(1.0, 0.0, 0.0, 1.0, GAMMA))
    right = np.asarray(ref["euler"].primitive_to_conserved(0.125, 0.0, 0.0, 0.1, GAMMA))
    on_left = solver.geometry.centroid[:, 0] < 0.5
    s = np.empty(solver.state_shape)
    s[:, on_left] = left
    s[:, ~on_left] = right
    return s


def gen_element(ref):
    R = ref["reference_element"].build_reference_triangle(4)
    return {k: np.asarray(getattr(R, k)) for k in ("r", "s", "dr", "ds", "lift", "face_nodes", "cell_weights",
                                                   "face_weights", "face_midpoint_nodes", "p1_midpoint",
                                                   "linear_midpoint_basis", "mass", "vandermonde")}


def gen_pointwise(ref):
    eu, fl, li = ref["euler"], ref["fluxes"], ref["limiters"]
    rng = np.random.default_rng(2024)
    n = 256
    pm = rng.uniform([0.1, -2.0, -2.0, 0.05], [2.0, 2.0, 2.0, 2.0], size=(n, 4))
    pp = rng.uniform([0.1, -2.0, -2.0, 0.05], [2.0, 2.0, 2.0, 2.0], size=(n, 4))
    ang = rng.uniform(0, 2 * np.pi, n)
    # edge cases: identical states, stationary contact, supersonic both ways, double rarefaction
    extra_m = [(1.0, 0.0, 0.0, 1.0), (1.0, 0.0, 0.0, 1.0), (1.0, 5.0, 0.0, 1.0), (0.8, 5.0, 0.0, 1.2),
               (1.0, -2.0, 0.0, 0.4), (1.3, 0.7, -0.4, 2.1), (0.125, 0.0, 0.0, 0.1)]
    extra_p = [(1.0, 0.0, 0.0, 1.0), (0.125, 0.0, 0.0, 1.0), (0.8, 5.0, 0.0, 1.2), (1.0, 5.0, 0.0, 1.0),
               (1.0, 2.0, 0.0, 0.4), (1.3, 0.7, -0.4, 2.1), (1.0, 0.0, 0.0, 1.0)]
    extra_a = [0.0, 0.0, 0.0, np.pi, 0.0, 2.214297435588181, np.pi]
    pm = np.concatenate([pm, np.array(extra_m)])
    pp = np.concatenate([pp, np.array(extra_p)])
    ang = np.concatenate([ang, np.array(extra_a)])
    nx, ny = np.cos(ang), np.sin(ang)
    qm = np.asarray(eu.primitive_to_conserved(*pm.T, GAMMA))
    qp = np.asarray(eu.primitive_to_conserved(*pp.T, GAMMA))
    out = {"q_minus": qm, "q_plus": qp, "nx": nx, "ny": ny}
    for name in FLUXES:
        out[f"flux/{name}"] = np.asarray(fl.get_interface_flux(name)(qm, qp, nx, ny, GAMMA))
    fx, fy = eu.cartesian_fluxes(qm, GAMMA)
    out["cartesian/f"], out["cartesian/g"] = np.asarray(fx), np.asarray(fy)
    out["normal_flux"] = np.asarray(eu.normal_flux(qm, nx, ny, GAMMA))
    r = np.concatenate([np.linspace(-5, 5, 41), [-1.0, 0.0, 0.25, 0.5, 1.0, 2.0, 4.0, 1e-300, 1e300, -1e300]])
    out["phi/r"] = r
    for name in LIMITERS:
        out[f"phi/{name}"] = np.asarray(li.get_limiter_function(name)(r))
    return out


def rhs_cases(ref):
    """(name, mesh, bcs, state) for the rhs and limit fixtures."""
    cases = []
    m = perturbed(ref, 6, 5)
    bc = fixed_all(ref, FREE_STREAM)
    s = make_solver(ref, m, bc)
    cases.append(("freestream", m, bc, np.broadcast_to(np.asarray(ref["euler"].primitive_to_conserved(*FREE_STREAM, GAMMA)), s.state_shape).copy()))
    m = perturbed(ref, 5, 4, seed=3)
    s = make_solver(ref, m, bc)
    cases.append(("random_fixed", m, bc, random_state(ref, s, 11)))
    m = perturbed(ref, 5, 4, seed=4)
    w = walls_all(ref)
    s = make_solver(ref, m, w)
    cases.append(("random_walls", m, w, random_state(ref, s, 12)))
    m = perturbed(ref, 10, 3, amplitude=0.2, seed=9)
    sb = sod_bcs(ref)
    s = make_solver(ref, m, sb)
    x, y = s.node_coordinates()
    prim = (1.0 + 0.3 * np.sin(6 * x) * np.cos(9 * y), 0.3 * np.cos(5 * x), -0.2 * np.sin(7 * y), 1.0 + 0.2 * np.cos(4 * x + 3 * y))
    cases.append(("smooth_mixed", m, sb, np.asarray(ref["euler"].primitive_to_conserved(*prim, GAMMA))))
    return cases


def gen_rhs(ref):
    out = {}
    for name, m, bcs, q in rhs_cases(ref):
        out.update(mesh_arrays(name, m))
        out.update(bc_arrays(name, bcs))
        out[f"{name}/q"] = q
        for flux in FLUXES:
            s = make_solver(ref, m, bcs, flux=flux)
            rhs, bflux = s.rhs(q)
            out[f"{name}/rhs/{flux}"] = rhs
            out[f"{name}/bflux/{flux}"] = bflux
    return out


def limit_cases(ref):
    cases = []
    bc = fixed_all(ref, FREE_STREAM)
    # noisy linear state on a perturbed mesh (test_limiting_and_time.py:34-42)
    m = perturbed(ref, 6, 5, seed=5)
    s = make_solver(ref, m, bc)
    x, y = s.node_coordinates()
    base = np.asarray(ref["euler"].primitive_to_conserved(*FREE_STREAM, GAMMA))
    q = base + np.array([0.05, 0.03, -0.02, 0.07]) * (0.3 * x + 0.2 * y)[..., None]
    q = q * (1.0 + 0.3 * np.random.default_rng(1).standard_normal(q.shape))
    cases.append(("noisy_linear", m, bc, q))
    # one oscillating cell (test_limiting_and_time.py:55-74)
    m = ref["mesh"].rectangle_mesh(8, 8)
    s = make_solver(ref, m, bc)
    q = np.broadcast_to(base, s.state_shape).copy()
    R = s.reference
    osc = 0.2 * np.cos(4.0 * np.pi * R.r) * np.cos(3.0 * np.pi * R.s)
    osc -= R.cell_weights @ osc / R.cell_weights.sum()
    q[:, 2 * (4 * 8 + 4), 0] += osc
    cases.append(("oscillation", m, bc, q))
    # negative density / pressure nodes (test_limiting_and_time.py:91-109)
    m = ref["mesh"].rectangle_mesh(4, 4)
    s = make_solver(ref, m, bc)
    q = np.broadcast_to(np.asarray(ref["euler"].primitive_to_conserved(1.0, 0.0, 0.0, 1.0, GAMMA)), s.state_shape).copy()
    dev = np.linspace(-1.5, 1.5, 15)
    dev -= R.cell_weights @ dev / R.cell_weights.sum()
    q[:, 5, 0] += dev
    q[:, 5, 3] += 1.2 * dev
    q[:, 9, 3] -= 2.0 * np.abs(dev)  # pressure-only violation in a second cell
    cases.append(("positivity", m, bc, q))
    # a rough Sod state with mixed boundaries (walls and fixed states)
    m = perturbed(ref, 12, 3, amplitude=0.15, seed=21)
    sb = sod_bcs(ref)
    s = make_solver(ref, m, sb)
    q = sod_state(ref, s) * (1.0 + 0.05 * np.random.default_rng(5).standard_normal(s.state_shape))
    cases.append(("rough_sod", m, sb, q))
    return cases


def gen_limit(ref):
    lim = ref["limiting"]
    out = {}
    for name, m, bcs, q in limit_cases(ref):
        out.update(mesh_arrays(name, m))
        out.update(bc_arrays(name, bcs))
        out[f"{name}/q"] = q
        for limiter in LIMITERS:
            s = make_solver(ref, m, bcs, limiter=limiter)
            limited, avg, count = s._limit(s._as_state(q), s.limiter_operators)
            out[f"{name}/limited/{limiter}"] = np.asarray(limited)
            out[f"{name}/count/{limiter}"] = np.asarray(int(count))
            if limiter != "unlimited":
                _, flags = lim.troubled_cell_limit(q, np.asarray(avg), s.limiter_operators, ref["limiters"].get_limiter_function(limiter))
                out[f"{name}/troubled/{limiter}"] = np.asarray(flags)
        out[f"{name}/averages"] = np.asarray(s.cell_averages(q))
        out[f"{name}/integral"] = np.asarray(s.integrate(q))
    return out


def gen_step(ref):
    out = {}
    m = perturbed(ref, 6, 3, amplitude=0.15, seed=33)
    sb = sod_bcs(ref)
    out.update(mesh_arrays("mesh", m))
    out.update(bc_arrays("mesh", sb))
    s0 = make_solver(ref, m, sb)
    q = sod_state(ref, s0) * (1.0 + 0.03 * np.random.default_rng(8).standard_normal(s0.state_shape))
    out["q"] = q
    for flux in FLUXES:
        for limiter in LIMITERS:
            s = make_solver(ref, m, sb, flux=flux, limiter=limiter)
            dt = s.time_step(q)
            qn, rep = s.step(q, dt)
            key = f"{flux}/{limiter}"
            out[f"{key}/dt"] = np.asarray(dt)
            out[f"{key}/q_new"] = qn
            out[f"{key}/boundary_flux"] = np.asarray(rep.boundary_flux)
            out[f"{key}/admissible"] = np.asarray(bool(rep.admissible))
            out[f"{key}/min_density"] = np.asarray(float(rep.min_density))
            out[f"{key}/min_pressure"] = np.asarray(float(rep.min_pressure))
            out[f"{key}/troubled_cells"] = np.asarray(int(rep.troubled_cells))
    return out


def instrumented_run(ref, solver, q0, final_time, flag_steps=0):
    """The loop of solver.py:167-216, recording per-step dt, report fields and
    per-stage troubled counts (and flags of the first ``flag_steps`` steps)."""
    lim = ref["limiting"]
    original = lim.troubled_cell_limit
    stage_flags = []

    def recording(*args, **kwargs):
        q, flags = original(*args, **kwargs)
        stage_flags.append(np.asarray(flags).copy())
        return q, flags

    lim.troubled_cell_limit = recording
    dts, counts, flags, bflux, mins = [], [], [], [], []
    orig_step = solver._step
    attempts = []

    def step_capture(*args):
        stage_flags.clear()
        out = orig_step(*args)
        attempts.append((float(args[1]), out[1], [f.copy() for f in stage_flags]))
        return out

    solver._step = step_capture
    try:
        t0 = time.perf_counter()
        result = solver.run(q0, final_time)
        for dt, rep, fl in attempts:
            if not bool(rep.admissible):
                continue
            dts.append(dt)
            counts.append([int(f.sum()) for f in fl] if fl else [0, 0, 0])
            if len(flags) < flag_steps:
                flags.append(np.stack(fl) if fl else np.zeros((3, q0.shape[1]), bool))
            bflux.append(np.asarray(rep.boundary_flux))
            mins.append([float(rep.min_density), float(rep.min_pressure)])
        print(f"  run: {result.steps} steps in {time.perf_counter() - t0:.1f} s")
    finally:
        lim.troubled_cell_limit = original
        solver._step = orig_step
    out = {
        "state": np.asarray(result.state), "time": np.asarray(result.time), "steps": np.asarray(result.steps),
        "rejected_steps": np.asarray(result.rejected_steps), "boundary_flux_integral": np.asarray(result.boundary_flux_integral),
        "min_density": np.asarray(result.min_density), "min_pressure": np.asarray(result.min_pressure),
        "max_troubled_cells": np.asarray(result.max_troubled_cells), "dt": np.asarray(dts),
        "stage_troubled": np.asarray(counts, dtype=np.int32), "step_boundary_flux": np.asarray(bflux),
        "step_minima": np.asarray(mins), "initial_state": np.asarray(q0),
    }
    if flags:
        out["troubled_flags_packed"] = np.packbits(np.stack(flags).astype(np.uint8), axis=-1)
        out["troubled_flags_shape"] = np.asarray(np.stack(flags).shape)
    return out


def gen_sod_short(ref):
    s = make_solver(ref, ref["mesh"].rectangle_mesh(20, 2), sod_bcs(ref))
    return instrumented_run(ref, s, sod_state(ref, s), 0.01, flag_steps=10**6)


def gen_sod_100x10(ref):
    case = ref["cases"].sod_shock_tube(100, 10, flux="rusanov", limiter="minmod")
    return instrumented_run(ref, case.solver, case.initial_state, case.final_time, flag_steps=25)


def gen_sod_100x10_flags(ref):
    """Every stage's troubled flags of the config-0 run, plus the decisions
    that round-off can flip: the detection of limiting.py:141-151 evaluated
    with the reference's own helpers on the stage's arguments, giving each
    element's largest excess / threshold ratio (flag = ratio > 1)."""
    lim = ref["limiting"]
    original = lim.troubled_cell_limit
    stage_rows = []

    def recording(q, averages, operators, phi):
        out_q, flags = original(q, averages, operators, phi)
        differences = lim.neighbor_averages(averages, operators) - averages[None]
        paired = np.take_along_axis(differences, np.asarray(operators.partner_face)[..., None], axis=0)
        scaled = lim.NEIGHBOR_FACTOR * (np.asarray(operators.alpha)[..., None] * differences
                                        + np.asarray(operators.beta)[..., None] * paired)
        trace = q[np.asarray(operators.midpoint_nodes)] - averages[None]
        comps = np.asarray(lim.DETECTION_COMPONENTS)
        excess = np.abs(lim._minmod(trace, scaled) - trace)[..., comps]
        threshold = lim.DETECTION_TOLERANCE * np.abs(averages[:, comps])
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(threshold[None] > 0, excess / threshold[None], np.where(excess > 0, np.inf, 0.0))
        worst = ratio.max(axis=(0, 2))
        assert np.array_equal(worst > 1.0, np.asarray(flags)), "ratio test disagrees with the reference's flags"
        stage_rows.append((np.asarray(flags).copy(), worst))
        return out_q, flags

    case = ref["cases"].sod_shock_tube(100, 10, flux="rusanov", limiter="minmod")
    solver = case.solver
    orig_step = solver._step
    attempts = []

    def step_capture(*args):
        stage_rows.clear()
        out = orig_step(*args)
        attempts.append((bool(out[1].admissible), list(stage_rows)))
        return out

    lim.troubled_cell_limit = recording
    solver._step = step_capture
    try:
        solver.run(case.initial_state, case.final_time)
    finally:
        lim.troubled_cell_limit = original
        solver._step = orig_step
    flags, border = [], []
    for ok, rows in attempts:
        if not ok:
            continue
        n = len(flags)
        flags.append(np.stack([r[0] for r in rows]))
        for k, (_, worst) in enumerate(rows):
            for e in np.nonzero(np.abs(worst - 1.0) <= 1e-3)[0]:
                border.append((n, k, int(e), float(worst[e])))
    flags = np.stack(flags).astype(np.uint8)  # (steps, 3, K)
    seq = flags.reshape(-1, flags.shape[-1])
    delta = seq.copy()
    delta[1:] ^= seq[:-1]
    border = np.asarray(border, dtype=np.float64).reshape(-1, 4)
    print(f"  {flags.shape[0]} steps, {int(flags.sum())} troubled decisions, {len(border)} borderline")
    return {"flags_delta_packed": np.packbits(delta, axis=-1), "flags_shape": np.asarray(flags.shape),
            "border": border}


GENERATORS = {
    "element": gen_element, "pointwise": gen_pointwise, "rhs": gen_rhs, "limit": gen_limit, "step": gen_step,
    "sod_short": gen_sod_short, "sod_100x10": gen_sod_100x10, "sod_100x10_flags": gen_sod_100x10_flags,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the CFD-demo source tree")
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    ref = load_reference(args.reference)
    for name, gen in GENERATORS.items():
        if args.only and name not in args.only:
            continue
        t0 = time.perf_counter()
        data = gen(ref)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{name}: {len(data)} arrays, {os.path.getsize(path) / 1024:.0f} KiB, {time.perf_counter() - t0:.1f} s")


if __name__ == "__main__":
    main()
