"""CPU checks of the verification diagnostics (cfd_demo_b200.verification):
the exact Riemann solver and the split quadrature."""

from __future__ import annotations

import numpy as np
import pytest

from cfd_demo_b200.mesh import jittered_rectangle_mesh, rectangle_mesh
from cfd_demo_b200.verification import ExactRiemann, collapsed_gauss, lagrange_at, quadrature

GAMMA = 1.4


def test_sod_star_state():
    ex = ExactRiemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), GAMMA, 0.5)
    assert ex.p_star == pytest.approx(0.30313, abs=5e-6)
    assert ex.u_star == pytest.approx(0.92745, abs=5e-6)
    waves = ex.wave_positions(0.2)
    assert list(waves) == ["head", "tail", "contact", "shock"]
    assert waves["shock"] == pytest.approx(0.5 + 0.2 * 1.75216, abs=1e-5)


@pytest.mark.parametrize("left,right", [((1.0, 0.0, 1.0), (0.125, 0.0, 0.1)),
                                        ((1.0, 0.75, 1.0), (0.125, 0.0, 0.1)),
                                        ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4)),
                                        ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.095))])
def test_exact_solution_satisfies_the_jump_conditions(left, right):
    """Rankine-Hugoniot across shocks, the isentrope and constant Riemann
    invariant across rarefactions, continuity of u and p at the contact."""
    ex = ExactRiemann(left, right, GAMMA, 0.0)
    t, g = 1.0, GAMMA
    waves = ex.wave_positions(t)
    rho, u, p = ex.sample(np.array(sorted(waves.values())) + np.array([[-1e-9], [1e-9]]), t)
    for name, x in waves.items():
        i = sorted(waves.values()).index(x)
        (r1, r2), (u1, u2), (p1, p2) = rho[:, i], u[:, i], p[:, i]
        if "shock" in name:
            s = x / t
            m1, m2 = r1 * (u1 - s), r2 * (u2 - s)
            assert m1 == pytest.approx(m2, rel=1e-9)
            assert m1 * u1 + p1 == pytest.approx(m2 * u2 + p2, rel=1e-9)
        elif name == "contact":
            assert u1 == pytest.approx(u2, rel=1e-9) and p1 == pytest.approx(p2, rel=1e-9)
    # across each rarefaction fan: entropy p / rho^g and the outgoing invariant are constant
    xs = np.linspace(-3, 3, 2001)
    r, uu, pp = ex.sample(xs, t)
    for side, sign in (("left", -1.0), ("right", 1.0)):
        st = ex.left if side == "left" else ex.right
        if ex.p_star <= st.p:
            c_s = np.sqrt(g * st.p / st.rho)
            head = st.u + sign * c_s
            tail = ex.u_star + sign * np.sqrt(g * ex.p_star / (st.rho * (ex.p_star / st.p) ** (1 / g)))
            fan = (xs > min(head, tail)) & (xs < max(head, tail))
            assert fan.any()
            assert np.allclose(pp[fan] / r[fan] ** g, st.p / st.rho ** g, rtol=1e-9)
            c = np.sqrt(g * pp[fan] / r[fan])
            assert np.allclose(uu[fan] - sign * 2 * c / (g - 1), st.u - sign * 2 * c_s / (g - 1), rtol=1e-9, atol=1e-12)


def test_collapsed_rule_is_exact_for_degree_eight_on_a_triangle():
    bary, w = collapsed_gauss(5)
    assert w.sum() == pytest.approx(1.0, abs=1e-15)
    # the integral of l1^a l2^b l0^c over the unit-area triangle is 2 a! b! c! / (a+b+c+2)!
    from math import factorial
    for a, b, c in [(2, 3, 1), (4, 4, 0), (0, 0, 8), (1, 5, 2)]:
        exact = 2 * factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 2)
        assert np.sum(w * bary[:, 1] ** a * bary[:, 2] ** b * bary[:, 0] ** c) == pytest.approx(exact, rel=1e-13)


@pytest.mark.parametrize("mesh", [rectangle_mesh(5, 3, (0.0, 1.0), (0.0, 0.3)),
                                  jittered_rectangle_mesh(6, 4, amplitude=0.2, seed=3)])
def test_split_quadrature_integrates_polynomials_and_keeps_pieces_on_one_side(mesh):
    breaks = [0.123, 0.5, 0.777]
    q = quadrature(mesh, breaks, 6)
    lo, hi = mesh.vertices.min(0), mesh.vertices.max(0)
    assert q.area == pytest.approx((hi - lo).prod(), rel=1e-13)
    f = lambda x, y: x ** 3 * y + 2 * x * y ** 2  # noqa: E731
    # exact over the rectangle [lo, hi]
    X = lambda n: (hi[0] ** n - lo[0] ** n) / n  # noqa: E731
    Y = lambda n: (hi[1] ** n - lo[1] ** n) / n  # noqa: E731
    assert np.sum(q.weight * f(q.x, q.y)) == pytest.approx(X(4) * Y(2) + 2 * X(2) * Y(3), rel=1e-12)
    # points of the reference coordinates map back to the same physical points
    c = mesh.vertices[mesh.elements][q.parent]
    lam = np.stack([-(q.r + q.s) / 2, (1 + q.r) / 2, (1 + q.s) / 2], -1)
    assert np.allclose(np.einsum("mv,mvd->md", lam, c), np.stack([q.x, q.y], -1), atol=1e-13)


def test_lagrange_basis_is_nodal():
    from cfd_demo_b200.reference_element import build_reference_triangle

    ref = build_reference_triangle(4)
    L = lagrange_at(ref.r, ref.s, ref)
    assert np.allclose(L, np.eye(15), atol=1e-12)
