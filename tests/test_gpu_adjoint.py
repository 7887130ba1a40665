"""Discrete adjoint of the fixed-schedule RK3 run against finite differences
of the same run, on the GPU.

The reference differentiates with jax.grad, which is not installed here. The
adjoint's semantics are those of a gradient through the reference's step:
dt is a constant of each step, the limiter branches are the ones taken, and
|x| has derivative sign(x) with sign(0) = 0. The positivity limiter's
bisection theta gets its implicit derivative, which is what a difference
quotient of the forward step sees. A difference quotient of the forward map
with the same step sizes checks the products directly.

The check is the central difference with eps = 1e-6, formed from the
nodewise difference of the two final states (J is linear in the final
state). Its round-off noise is measured, not assumed: the spread of the central quotients at eps = 5e-7,
1e-6 and 2e-6 (a truncation error would grow as eps^2 instead). Where the
derivative is a tiny tail effect (dJ/drho_L at t << the shock's arrival at
x = 0.7) that noise is about 1e-3 relative; the small cases therefore also
use a target at x = 0.5, where the derivative is of order one. A
fourth-order stencil with h = 1e-4 is reported beside it: along dJ/drho_L
its large steps cross limiter switches and lose accuracy, along smooth
density perturbations inside the bump it is the quieter of the two
estimates and the random-direction checks use it.

Directions are chosen where the forward map is differentiable: rescaling
features that are already present (the left density, the density bump) or,
with the limiter off, any smooth perturbation. A random perturbation of a
flat region switches the troubled-cell detector (threshold 1e-10 |average|)
and has no derivative.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

EPS = 1e-6
H4 = 1e-4


def _quotients(run, objective, spread=False):
    """Difference quotients of objective(run(s)) at s = 0 for a LINEAR
    objective, formed from nodewise differences of the final states (exact
    subtractions; a difference of two sums near |J| would lose digits to the
    rounding of J itself): the central quotient with eps = 1e-6, the
    fourth-order stencil with h = 1e-4 and, with spread=True, the spread of
    the central quotients at eps = 5e-7, 1e-6, 2e-6 (round-off noise)."""
    def central_at(e):
        return float(objective(run(e) - run(-e))) / (2 * e)

    central = central_at(EPS)
    fourth = float(objective(run(-2 * H4) - 8 * run(-H4) + 8 * run(H4) - run(2 * H4))) / (12 * H4)
    if not spread:
        return central, fourth
    return central, fourth, max(abs(central_at(e) - central) for e in (0.5 * EPS, 2 * EPS))


def _rho_left(case, runner, spread=False):
    """dJ/drho_L by the adjoint (autograd through differentiable_run) and by
    difference quotients of the forward run."""
    from cfd_demo_b200.adjoint import differentiable_run

    dev = case.solver.operators.device
    base_bc = case.solver.operators.bc_states.clone()
    rho = torch.tensor(case.rho_left, dtype=torch.float64, device=dev, requires_grad=True)
    j = case.objective(differentiable_run(runner, case.initial_state(rho), case.boundary_states(rho)))
    j.backward()

    def run(s):
        with torch.no_grad():
            r = torch.tensor(case.rho_left + s, dtype=torch.float64, device=dev)
            return differentiable_run(runner, case.initial_state(r), case.boundary_states(r))

    quotients = _quotients(run, case.objective, spread)
    case.solver.operators.bc_states.copy_(base_bc)
    return (float(rho.grad), *quotients, float(j.detach()))


def _direction(case, runner, direction, spread=False):
    """<dJ/dq0, direction> by the adjoint and by difference quotients."""
    from cfd_demo_b200.adjoint import differentiable_run

    dev = case.solver.operators.device
    rho = torch.tensor(case.rho_left, dtype=torch.float64, device=dev)
    q0 = case.initial_state(rho).detach().clone().requires_grad_(True)
    bc = case.boundary_states(rho)
    j = case.objective(differentiable_run(runner, q0, bc))
    j.backward()

    def run(s):
        with torch.no_grad():
            return differentiable_run(runner, q0 + s * direction, bc)

    quotients = _quotients(run, case.objective, spread)
    return (float((q0.grad * direction).sum()), *quotients, q0.grad)


def _sod_case(nx, ny, steps, checkpoint_every, **kw):
    from cfd_demo_b200.adjoint import AdjointRun, SodSensitivity, cfl_schedule

    case = SodSensitivity(nx, ny, **kw)
    rho = torch.tensor(case.rho_left, dtype=torch.float64, device=case.solver.operators.device)
    dts = cfl_schedule(case.solver, case.initial_state(rho).cpu().numpy(), steps=steps)
    return case, AdjointRun(case.solver, dts, checkpoint_every=checkpoint_every)


def _bump_direction(case):
    d = torch.zeros(case.solver.state_shape, dtype=torch.float64, device=case.solver.operators.device)
    d[..., 0] = case.bump / case.amplitude
    return d


def _rel(a, b):
    return abs(a - b) / abs(b)


@pytest.mark.parametrize("limiter", ["minmod", "mc", "van_leer", "superbee", "unlimited"])
def test_rho_left_gradient_matches_central_difference(limiter, report):
    case, runner = _sod_case(40, 4, 30, 7, limiter=limiter, seed=1, target=0.5)
    adjoint, central, fourth, spread, _ = _rho_left(case, runner, spread=True)
    report(f"adjoint Sod 40x4 rusanov/{limiter} 30 steps, target x = 0.5: dJ/drho_L {adjoint:.10e}; "
           f"rel to central(1e-6) {_rel(adjoint, central):.1e} (noise {spread / abs(central):.0e}), "
           f"to 4th-order(1e-4) {_rel(adjoint, fourth):.1e}")
    assert abs(adjoint - central) < 3 * spread + 1e-6 * abs(central)


def test_rho_left_gradient_tail_effect_within_noise(report):
    """dJ/drho_L with the target at x = 0.7: the left state reaches it only
    through the scheme's numerical stencil, a derivative 1e-6 of the size of
    J's own terms; the central quotient agrees within its measured noise."""
    case, runner = _sod_case(40, 4, 30, 7, seed=1)
    adjoint, central, _, spread, _ = _rho_left(case, runner, spread=True)
    report(f"adjoint Sod 40x4 rusanov/minmod 30 steps, target x = 0.7: dJ/drho_L {adjoint:.10e}; "
           f"rel to central(1e-6) {_rel(adjoint, central):.1e} (noise {spread / abs(central):.0e})")
    assert abs(adjoint - central) < 3 * spread + 1e-6 * abs(central)


@pytest.mark.parametrize("flux", ["rusanov", "roe", "hllc"])
def test_bump_gradient_matches_difference_quotients(flux, report):
    case, runner = _sod_case(40, 4, 30, 10, flux=flux, limiter="minmod", bump_center=0.65)
    adjoint, central, fourth, _ = _direction(case, runner, _bump_direction(case))
    report(f"adjoint Sod 40x4 {flux}/minmod 30 steps: dJ/d(bump amplitude) {adjoint:.10e}; "
           f"rel to central(1e-6) {_rel(adjoint, central):.1e}, to 4th-order(1e-4) {_rel(adjoint, fourth):.1e}")
    assert _rel(adjoint, central) < 1e-8


def _smooth_case(flux, seed=0):
    """Jittered mesh, smooth random state, fixed exterior states on every
    side, limiter off: the forward map is smooth, any direction will do."""
    from cfd_demo_b200 import EulerSolver, FixedState, SolverConfig, jittered_rectangle_mesh

    mesh = jittered_rectangle_mesh(12, 10, amplitude=0.2, seed=seed)
    mean = FixedState.from_primitive(1.0, 0.1, -0.05, 1.0, 1.4)
    bcs = {t: mean for t in ("left", "right", "bottom", "top")}
    solver = EulerSolver(mesh, bcs, SolverConfig(flux=flux, limiter="unlimited", gamma=1.4))
    x, y = solver.node_coordinates()
    rng = np.random.default_rng(seed)
    prim = []
    for lo, hi in ((0.7, 1.3), (-0.3, 0.3), (-0.3, 0.3), (0.7, 1.3)):
        f = np.zeros_like(x)
        for _ in range(4):
            kx, ky = rng.integers(1, 4, size=2)
            f += rng.uniform(-1, 1) * np.sin(np.pi * (kx * x + ky * y) + rng.uniform(0, 2 * np.pi))
        f = (f - f.min()) / (f.max() - f.min())
        prim.append(lo + (hi - lo) * f)
    rho, u, v, p = prim
    q = np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=-1)
    return solver, q, x, y


@pytest.mark.parametrize("flux", ["rusanov", "roe", "hllc"])
def test_smooth_state_random_direction_unlimited(flux, report):
    from cfd_demo_b200.adjoint import AdjointRun, cfl_schedule, differentiable_run

    solver, q, x, y = _smooth_case(flux)
    dts = cfl_schedule(solver, q, steps=12)
    runner = AdjointRun(solver, dts, checkpoint_every=5)
    dev = solver.operators.device
    weight = torch.from_numpy(np.exp(-((x - 0.6) ** 2 + (y - 0.4) ** 2) / 0.05)).to(dev)
    rng = np.random.default_rng(7)
    direction = torch.from_numpy(rng.normal(size=q.shape)).to(dev)
    cotangent = torch.from_numpy(rng.normal(size=4)).to(dev)

    def objective(qf):
        return ((qf * cotangent).sum(-1) * weight).sum()

    q0 = torch.from_numpy(q).to(dev).requires_grad_(True)
    bc = solver.operators.bc_states.clone().requires_grad_(True)
    j = objective(differentiable_run(runner, q0, bc))
    j.backward()
    adjoint = float((q0.grad * direction).sum())
    with torch.no_grad():
        central, _ = _quotients(lambda s: differentiable_run(runner, q0 + s * direction, bc), objective)
    dbc = torch.from_numpy(rng.normal(size=bc.shape)).to(dev)
    ad_bc = float((bc.grad * dbc).sum())
    with torch.no_grad():
        central_bc, _ = _quotients(lambda s: differentiable_run(runner, q0, bc + s * dbc), objective)
    report(f"adjoint smooth 12x10 {flux}/unlimited 12 steps: state rel {_rel(adjoint, central):.1e}, "
           f"exterior state rel {_rel(ad_bc, central_bc):.1e}")
    assert _rel(adjoint, central) < 1e-6
    assert _rel(ad_bc, central_bc) < 1e-6


@pytest.mark.parametrize("flux", ["rusanov", "hllc"])
def test_exact_state_boundaries_random_direction_unlimited(flux, report):
    """Exact-state faces (one exterior row per face node) on two sides of the
    smooth case: the gradient in the initial state and in the per-node
    exterior rows against central differences."""
    from cfd_demo_b200 import EulerSolver, ExactState, FixedState, SolverConfig
    from cfd_demo_b200.adjoint import AdjointRun, cfl_schedule, differentiable_run

    base, q, x, y = _smooth_case(flux, seed=2)

    def far(xx, yy):
        rho = 1.0 + 0.2 * np.sin(2.0 * xx + 1.0) * np.cos(3.0 * yy)
        u, v, p = 0.1 + 0.05 * np.cos(xx), -0.05 + 0.03 * np.sin(yy), 1.0 + 0.1 * np.sin(xx + yy)
        return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=-1)

    mean = FixedState.from_primitive(1.0, 0.1, -0.05, 1.0, 1.4)
    bcs = {"left": mean, "bottom": mean, "top": ExactState(far), "right": ExactState(far)}
    solver = EulerSolver(base.mesh, bcs, SolverConfig(flux=flux, limiter="unlimited", gamma=1.4))
    dts = cfl_schedule(solver, q, steps=12)
    runner = AdjointRun(solver, dts, checkpoint_every=5)
    dev = solver.operators.device
    weight = torch.from_numpy(np.exp(-((x - 0.8) ** 2 + (y - 0.8) ** 2) / 0.05)).to(dev)
    rng = np.random.default_rng(11)
    direction = torch.from_numpy(rng.normal(size=q.shape)).to(dev)
    cotangent = torch.from_numpy(rng.normal(size=4)).to(dev)

    def objective(qf):
        return ((qf * cotangent).sum(-1) * weight).sum()

    q0 = torch.from_numpy(q).to(dev).requires_grad_(True)
    bc = solver.operators.bc_states.clone().requires_grad_(True)
    assert bc.shape[0] == 1 + 6 * (12 + 10)  # one fixed row, six rows per exact-state face
    j = objective(differentiable_run(runner, q0, bc))
    j.backward()
    adjoint = float((q0.grad * direction).sum())
    with torch.no_grad():
        central, _ = _quotients(lambda s: differentiable_run(runner, q0 + s * direction, bc), objective)
    dbc = torch.from_numpy(rng.normal(size=bc.shape)).to(dev)
    ad_bc = float((bc.grad * dbc).sum())
    with torch.no_grad():
        central_bc, _ = _quotients(lambda s: differentiable_run(runner, q0, bc + s * dbc), objective)
    report(f"adjoint smooth 12x10 {flux}/unlimited 12 steps, exact-state top and right: state rel "
           f"{_rel(adjoint, central):.1e}, exterior rows rel {_rel(ad_bc, central_bc):.1e}")
    assert _rel(adjoint, central) < 1e-6
    assert _rel(ad_bc, central_bc) < 1e-6


def test_checkpoint_interval_does_not_change_the_gradient():
    from cfd_demo_b200.adjoint import AdjointRun

    case, runner = _sod_case(40, 4, 25, 25, seed=3)
    direction = torch.ones(case.solver.state_shape, dtype=torch.float64, device=case.solver.operators.device)
    grads = []
    for every in (1, 6, 25):
        r = AdjointRun(case.solver, runner.dts.cpu().numpy()[:, 0], checkpoint_every=every)
        grads.append(_direction(case, r, direction)[3].cpu().numpy())
    assert np.array_equal(grads[0], grads[1])
    assert np.array_equal(grads[0], grads[2])


def test_hold_theta_changes_the_gradient_only_where_positivity_scaled():
    """With the pressure-scaling theta held constant (jax.grad's derivative of
    the bisection loop) the gradient is the implicit one wherever the
    positivity limiter never scaled, and differs where it did."""
    from cfd_demo_b200.adjoint import AdjointRun, cfl_schedule, differentiable_run

    def grads(solver, q, steps):
        dts = cfl_schedule(solver, q, steps=steps)
        out = []
        for hold in (False, True):
            runner = AdjointRun(solver, dts, checkpoint_every=steps, hold_theta=hold)
            q0 = torch.from_numpy(q).to(solver.operators.device).requires_grad_(True)
            differentiable_run(runner, q0)[..., 0].sum().backward()
            out.append(q0.grad)
        return out

    solver, q, _, _ = _smooth_case("rusanov")
    implicit, held = grads(solver, q, 4)
    assert torch.equal(implicit, held)  # no element needed the positivity limiter

    case, _ = _sod_case(40, 4, 1, 1, limiter="unlimited", seed=4)
    rho = torch.tensor(case.rho_left, dtype=torch.float64, device=case.solver.operators.device)
    implicit, held = grads(case.solver, case.initial_state(rho).cpu().numpy(), 30)
    assert torch.isfinite(implicit).all() and torch.isfinite(held).all()
    assert not torch.equal(implicit, held)  # the Sod jump drives nodes to the pressure floor


def test_sod_400x40_200_steps_sensitivity(report):
    """The sensitivity study at full size: Sod 400x40 (K = 32,000),
    rusanov/minmod, 200 CFL steps, checkpoints every 20 steps, the bump at its
    seeded position."""
    case, runner = _sod_case(400, 40, 200, 20, seed=0)
    adjoint, central, fourth, spread, j = _rho_left(case, runner, spread=True)
    ad_b, central_b, fourth_b, _ = _direction(case, runner, _bump_direction(case))
    report(f"adjoint Sod 400x40 rusanov/minmod 200 steps (bump at x = {case.bump_center:.4f}): J {j:.10e}; "
           f"dJ/drho_L {adjoint:.10e} rel to central(1e-6) {_rel(adjoint, central):.1e} "
           f"(noise {spread / abs(central):.0e}), to 4th-order(1e-4) {_rel(adjoint, fourth):.1e}; "
           f"dJ/d(bump amplitude) {ad_b:.10e} rel to central {_rel(ad_b, central_b):.1e}, "
           f"to 4th-order {_rel(ad_b, fourth_b):.1e}")
    assert _rel(ad_b, central_b) < 1e-4
    # dJ/drho_L is a tail effect here (about 1e-8 of J's term scale): the
    # central quotient's measured round-off spread bounds the comparison
    assert abs(adjoint - central) < 3 * spread + 1e-4 * abs(central)


def _smooth_bump_direction(case, seed):
    """A random smooth density perturbation inside the bump: the bump's
    Gaussian envelope times a random smooth modulation along the tube
    (random amplitude, wavelength and phase). The initial velocity is zero
    and the pressure is untouched, so the perturbation is a density (entropy)
    profile in the region where the solution already varies smoothly, and it
    vanishes where the solution is flat: the forward map is differentiable
    along it (a perturbation of a flat region would switch the troubled-cell
    detector, whose threshold is 1e-10 |average|)."""
    x = torch.as_tensor(case.solver.node_coordinates()[0], device=case.solver.operators.device)
    gen = np.random.default_rng(seed)
    b, wavelength, phase = gen.uniform(-0.8, 0.8), gen.uniform(0.1, 0.3), gen.uniform(0, 2 * np.pi)
    d = torch.zeros(case.solver.state_shape, dtype=torch.float64, device=x.device)
    d[..., 0] = case.bump / case.amplitude * (1.0 + b * torch.sin(2 * np.pi * (x - case.bump_center) / wavelength + phase))
    return d


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_sod_400x40_random_smooth_direction(seed, report):
    """The sensitivity study (Sod 400x40, 200 steps, checkpoints every 20): <dJ/dq0, d>
    for random smooth density directions d in the bump region. The adjoint
    must agree with the fourth-order difference quotient (h = 1e-4) to 1e-4
    relative, and with the central quotient (eps = 1e-6) within that
    quotient's measured spread over eps = 5e-7 .. 2e-6 (plus 1e-4 relative).
    Along these directions the two quotients differ from each other by up to
    7e-4 while the fourth-order one agrees with the adjoint to a few 1e-6:
    the small-eps quotient is the noisier estimate here, and its noise is
    measured rather than assumed."""
    case, runner = _sod_case(400, 40, 200, 20, seed=0)
    d = _smooth_bump_direction(case, seed)
    ad, central, fourth, spread, _ = _direction(case, runner, d, spread=True)
    report(f"adjoint Sod 400x40 200 steps, random smooth density direction (seed {seed}): {ad:.10e}, "
           f"rel to 4th-order(1e-4) {_rel(ad, fourth):.1e}, to central(1e-6) {_rel(ad, central):.1e} "
           f"(spread of the central quotient {spread / abs(central):.1e})")
    assert _rel(ad, fourth) < 1e-4
    assert abs(ad - central) < 3 * spread + 1e-4 * abs(central)


def test_fp32_mixed_gradient_tracks_fp64(report):
    """FP32-mixed adjoint against the FP64 adjoint on the same schedule: the
    gradient field dJ/dq0 (L1 norm; the FP32-mixed form detects troubled
    cells at 1e-5 |average| instead of 1e-10, so a few elements take other
    limiter branches) and dJ/drho_L (a sum with heavy cancellation)."""
    from cfd_demo_b200.adjoint import AdjointRun

    case64, run64 = _sod_case(400, 40, 200, 20, seed=0)
    case32, _ = _sod_case(400, 40, 1, 1, seed=0, precision="fp32_mixed")
    run32 = AdjointRun(case32.solver, run64.dts.cpu().numpy()[:, 0], checkpoint_every=20)
    direction = _bump_direction(case64)
    _, _, _, g64 = _direction(case64, run64, direction)
    _, _, _, g32 = _direction(case32, run32, direction)
    field = float((g32 - g64).abs().sum() / g64.abs().sum())  # L1 relative
    field_max = float((g32 - g64).abs().max() / g64.abs().max())
    a64 = _rho_left(case64, run64)[0]
    a32 = _rho_left(case32, run32)[0]
    scale = float(g64[..., 0].abs().sum())  # size of the terms that cancel in dJ/drho_L
    report(f"adjoint Sod 400x40 200 steps FP32-mixed vs FP64: gradient field L1 rel {field:.1e} "
           f"(max-norm rel {field_max:.1e}: elements where the FP32 detection threshold takes another branch); "
           f"dJ/drho_L {a32:.8e} vs {a64:.8e} (difference {abs(a32 - a64):.1e} against term scale {scale:.1e})")
    assert field < 1e-3
    assert abs(a32 - a64) < 1e-5 * scale
