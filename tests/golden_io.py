"""Read the golden fixtures of ``tests/golden`` (written by make_golden.py)."""

from __future__ import annotations

import os
from functools import lru_cache

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FLUXES = ("rusanov", "roe", "hllc")
LIMITERS = ("minmod", "mc", "van_leer", "superbee", "unlimited")
GAMMA = 1.4


@lru_cache(maxsize=None)
def load(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as data:
        return {k: data[k] for k in data.files}


def case_prefixes(data: dict) -> list[str]:
    return sorted({k.split("/")[0] for k in data if k.endswith("/vertices")})


def mesh_parts(data: dict, prefix: str):
    """(vertices, elements, boundary_edges dict) stored under ``prefix``."""
    edges = {k.split("/")[-1]: data[k] for k in data if k.startswith(f"{prefix}/edges/")}
    return data[f"{prefix}/vertices"], data[f"{prefix}/elements"], edges


def boundary_specs(data: dict, prefix: str) -> dict:
    """tag -> (kind, state tuple) with kind 1 = slip wall, 2 = fixed state."""
    out = {}
    for k in data:
        if k.startswith(f"{prefix}/bc/"):
            row = data[k]
            out[k.split("/")[-1]] = (int(row[0]), tuple(float(v) for v in row[1:]))
    return out


def unpack_flags(data: dict) -> np.ndarray:
    shape = tuple(int(v) for v in data["troubled_flags_shape"])
    return np.unpackbits(data["troubled_flags_packed"], axis=-1, count=shape[-1]).astype(bool).reshape(shape)


def flag_history() -> np.ndarray:
    """(steps, 3, K) bool: the reference's troubled flags at every stage of
    the config-0 Sod run (sod_100x10_flags.npz stores each stage XOR the
    previous one, bit-packed)."""
    data = load("sod_100x10_flags")
    shape = tuple(int(v) for v in data["flags_shape"])
    delta = np.unpackbits(data["flags_delta_packed"], axis=-1, count=shape[-1]).astype(bool)
    return np.logical_xor.accumulate(delta, axis=0).reshape(shape)


def borderline_decisions() -> dict:
    """(step, stage, element) -> the reference's largest excess / threshold
    ratio there, for every decision of the config-0 run within 1e-3 of one."""
    rows = load("sod_100x10_flags")["border"]
    return {(int(n), int(k), int(e)): float(r) for n, k, e, r in rows}
