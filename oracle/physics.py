"""Oracle: Euler relations, interface fluxes, limiter functions and boundary
conditions (test infrastructure only).

Restates ``src/cfd_demo/euler.py``, ``fluxes.py``, ``limiters.py`` and
``boundary.py`` of CFD-demo in NumPy float64. Conserved variables are
(rho, rho u, rho v, E) along the last axis. NumPy's minimum/maximum propagate
NaN exactly as jax.numpy's do.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SLIP_WALL = 1  # boundary.py:13
FIXED_STATE = 2  # boundary.py:14
EXACT_STATE = 3  # proposed, docs/adr/0012-sheared-rectangle-mesh-and-far-field-boundaries.md:32-46
ROE_ENTROPY_FIX = 0.1  # fluxes.py:21


@dataclass(frozen=True)
class SlipWall:
    """boundary.py:17-24."""

    kind: int = SLIP_WALL


@dataclass(frozen=True)
class FixedState:
    """boundary.py:27-43."""

    state: tuple
    kind: int = FIXED_STATE

    def __post_init__(self):
        object.__setattr__(self, "state", tuple(float(v) for v in self.state))

    @classmethod
    def from_primitive(cls, rho, u, v, p, gamma):
        return cls((rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)))


@dataclass(frozen=True, eq=False)
class ExactState:
    """The proposed far-field condition of ADR 0012 (docs/adr/0012-...:32-46),
    not implemented in the reference: `function(x, y)` gives conserved
    states x.shape + (4,), evaluated at the face nodes of the tagged faces;
    the ghost average across a face is the function's cell average over the
    boundary element reflected across that face (`cell_average(corners)`
    when given)."""

    function: object
    cell_average: object = None
    kind: int = EXACT_STATE


def primitive_to_conserved(rho, u, v, p, gamma):
    """euler.py:14-18."""
    rho, u, v, p = (np.asarray(a, dtype=np.float64) for a in (rho, u, v, p))
    e = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack(np.broadcast_arrays(rho, rho * u, rho * v, e), axis=-1)


def conserved_to_primitive(q, gamma):
    """euler.py:21-27."""
    rho = q[..., 0]
    u = q[..., 1] / rho
    v = q[..., 2] / rho
    p = (gamma - 1.0) * (q[..., 3] - 0.5 * (q[..., 1] * u + q[..., 2] * v))
    return rho, u, v, p


def pressure(q, gamma):
    """euler.py:30-32."""
    return conserved_to_primitive(q, gamma)[3]


def sound_speed(rho, p, gamma):
    """euler.py:35-37."""
    return np.sqrt(gamma * p / rho)


def cartesian_fluxes(q, gamma):
    """euler.py:40-46."""
    rho, u, v, p = conserved_to_primitive(q, gamma)
    mx, my, e = q[..., 1], q[..., 2], q[..., 3]
    f = np.stack([mx, mx * u + p, my * u, (e + p) * u], axis=-1)
    g = np.stack([my, mx * v, my * v + p, (e + p) * v], axis=-1)
    return f, g


def normal_flux(q, nx, ny, gamma):
    """euler.py:49-61."""
    rho, u, v, p = conserved_to_primitive(q, gamma)
    un = u * nx + v * ny
    return np.stack([rho * un, q[..., 1] * un + p * nx, q[..., 2] * un + p * ny, (q[..., 3] + p) * un], axis=-1)


def _nonzero(x):
    """fluxes.py:24-25: replace exact zeros by the smallest normal double."""
    return np.where(x == 0.0, np.finfo(np.float64).tiny, x)


def rusanov(qm, qp, nx, ny, gamma):
    """fluxes.py:28-37."""
    rm, um, vm, pm = conserved_to_primitive(qm, gamma)
    rp, up, vp, pp = conserved_to_primitive(qp, gamma)
    sm = np.abs(um * nx + vm * ny) + sound_speed(rm, pm, gamma)
    sp = np.abs(up * nx + vp * ny) + sound_speed(rp, pp, gamma)
    a = np.maximum(sm, sp)[..., None]
    return 0.5 * (normal_flux(qm, nx, ny, gamma) + normal_flux(qp, nx, ny, gamma)) - 0.5 * a * (qp - qm)


def _roe_mean(qm, qp, gamma):
    """fluxes.py:40-51."""
    rm, um, vm, pm = conserved_to_primitive(qm, gamma)
    rp, up, vp, pp = conserved_to_primitive(qp, gamma)
    hm = (qm[..., 3] + pm) / rm
    hp = (qp[..., 3] + pp) / rp
    wm, wp = np.sqrt(rm), np.sqrt(rp)
    u = (wm * um + wp * up) / (wm + wp)
    v = (wm * vm + wp * vp) / (wm + wp)
    h = (wm * hm + wp * hp) / (wm + wp)
    c = np.sqrt((gamma - 1.0) * (h - 0.5 * (u * u + v * v)))
    return wm * wp, u, v, h, c


def roe(qm, qp, nx, ny, gamma):
    """Roe flux with Harten's entropy fix (fluxes.py:54-98)."""
    rm, um, vm, pm = conserved_to_primitive(qm, gamma)
    rp, up, vp, pp = conserved_to_primitive(qp, gamma)
    rho, u, v, h, c = _roe_mean(qm, qp, gamma)
    un = u * nx + v * ny
    ut = -u * ny + v * nx
    drho = rp - rm
    dp = pp - pm
    dun = (up * nx + vp * ny) - (um * nx + vm * ny)
    dut = (-up * ny + vp * nx) - (-um * ny + vm * nx)
    c2 = c * c
    a_m = (dp - rho * c * dun) / (2.0 * c2)
    a_e = drho - dp / c2
    a_s = rho * dut
    a_p = (dp + rho * c * dun) / (2.0 * c2)
    delta = ROE_ENTROPY_FIX * (np.abs(un) + c)

    def fixed(lam):
        mag = np.abs(lam)
        return np.where(mag < delta, (lam**2 + delta**2) / (2.0 * delta), mag)

    l_m, l_p, l_0 = fixed(un - c), fixed(un + c), np.abs(un)
    one, zero = np.ones_like(un), np.zeros_like(un)
    r_m = np.stack([one, u - c * nx, v - c * ny, h - c * un], axis=-1)
    r_e = np.stack([one, u, v, 0.5 * (u * u + v * v)], axis=-1)
    r_s = np.stack([zero, -ny * one, nx * one, ut], axis=-1)
    r_p = np.stack([one, u + c * nx, v + c * ny, h + c * un], axis=-1)
    diss = ((l_m * a_m)[..., None] * r_m + (l_0 * a_e)[..., None] * r_e
            + (l_0 * a_s)[..., None] * r_s + (l_p * a_p)[..., None] * r_p)
    return 0.5 * (normal_flux(qm, nx, ny, gamma) + normal_flux(qp, nx, ny, gamma)) - 0.5 * diss


def hllc(qm, qp, nx, ny, gamma):
    """Toro's HLLC with Einfeldt speeds (fluxes.py:101-143)."""
    rm, um, vm, pm = conserved_to_primitive(qm, gamma)
    rp, up, vp, pp = conserved_to_primitive(qp, gamma)
    unm, unp = um * nx + vm * ny, up * nx + vp * ny
    cm, cp = sound_speed(rm, pm, gamma), sound_speed(rp, pp, gamma)
    _, u, v, _, c = _roe_mean(qm, qp, gamma)
    un = u * nx + v * ny
    s_m = np.minimum(unm - cm, un - c)
    s_p = np.maximum(unp + cp, un + c)
    mm = rm * (s_m - unm)
    mp = rp * (s_p - unp)
    s_star = (pp - pm + mm * unm - mp * unp) / _nonzero(mm - mp)

    def star(q, r, uk, vk, p, unk, sk, mk):
        fac = mk / _nonzero(sk - s_star)
        sh = s_star - unk
        return fac[..., None] * np.stack(
            [np.ones_like(r), uk + sh * nx, vk + sh * ny, q[..., 3] / r + sh * (s_star + p / _nonzero(mk))], axis=-1)

    fm, fp = normal_flux(qm, nx, ny, gamma), normal_flux(qp, nx, ny, gamma)
    fsm = fm + s_m[..., None] * (star(qm, rm, um, vm, pm, unm, s_m, mm) - qm)
    fsp = fp + s_p[..., None] * (star(qp, rp, up, vp, pp, unp, s_p, mp) - qp)
    s_m, s_p, s_star = s_m[..., None], s_p[..., None], s_star[..., None]
    return np.where(s_m >= 0.0, fm, np.where(s_star >= 0.0, fsm, np.where(s_p > 0.0, fsp, fp)))


INTERFACE_FLUXES = {"rusanov": rusanov, "roe": roe, "hllc": hllc}


def get_interface_flux(name):
    """fluxes.py:153-159."""
    try:
        return INTERFACE_FLUXES[name]
    except KeyError:
        raise ValueError(f"Unknown interface flux {name!r}; choose one of: {', '.join(sorted(INTERFACE_FLUXES))}.") from None


def minmod(r):
    """limiters.py:16-18."""
    return np.maximum(0.0, np.minimum(1.0, r))


def mc(r):
    """limiters.py:21-23."""
    return np.maximum(0.0, np.minimum(np.minimum(2.0 * r, 0.5 * (1.0 + r)), 2.0))


def van_leer(r):
    """limiters.py:26-28."""
    return (r + np.abs(r)) / (1.0 + np.abs(r))


def superbee(r):
    """limiters.py:31-33."""
    return np.maximum(0.0, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)))


def unlimited(r):
    """limiters.py:36-39."""
    return np.ones_like(np.asarray(r, dtype=np.float64))


LIMITER_FUNCTIONS = {"minmod": minmod, "mc": mc, "van_leer": van_leer, "superbee": superbee, "unlimited": unlimited}


def get_limiter_function(name):
    """limiters.py:51-57."""
    try:
        return LIMITER_FUNCTIONS[name]
    except KeyError:
        raise ValueError(f"Unknown limiter {name!r}; choose one of: {', '.join(sorted(LIMITER_FUNCTIONS))}.") from None
