"""Selectable interface fluxes (names of CFD-demo src/cfd_demo/fluxes.py:146-159).

Each callable ``flux(q_minus, q_plus, nx, ny, gamma)`` evaluates, on the GPU,
the same ``__device__`` flux function that the fused DG kernels use
(csrc/physics.cuh), for arrays of states (..., 4) and broadcastable normals.
"""

from __future__ import annotations

from collections.abc import Callable

import numpy as np

FLUX_IDS = {"rusanov": 0, "roe": 1, "hllc": 2}


def _device_flux(flux_id: int) -> Callable:
    def flux(q_minus, q_plus, nx, ny, gamma: float):
        import torch

        from . import _native

        qm = np.asarray(q_minus, dtype=np.float64)
        qp = np.asarray(q_plus, dtype=np.float64)
        shape = np.broadcast_shapes(qm.shape[:-1], qp.shape[:-1], np.shape(nx), np.shape(ny))
        arrs = [np.broadcast_to(qm, shape + (4,)), np.broadcast_to(qp, shape + (4,)),
                np.broadcast_to(np.asarray(nx, np.float64), shape), np.broadcast_to(np.asarray(ny, np.float64), shape)]
        # copies: broadcast views are read-only, which torch does not accept as tensor storage
        dev = [torch.from_numpy(np.array(a, dtype=np.float64)).reshape(-1).cuda() for a in arrs]
        n = int(np.prod(shape)) if shape else 1
        out = torch.empty(4 * n, dtype=torch.float64, device="cuda")
        lib = _native.load()
        _native.check(lib.cfd_interface_flux(flux_id, n, *(d.data_ptr() for d in dev), float(gamma), out.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream))
        return out.cpu().numpy().reshape(shape + (4,))

    return flux


rusanov = _device_flux(0)
roe = _device_flux(1)
hllc = _device_flux(2)
rusanov.__doc__ = "Rusanov (local Lax-Friedrichs) flux (fluxes.py:28-37), on the GPU."
roe.__doc__ = "Roe flux with Harten's entropy fix (fluxes.py:54-98), on the GPU."
hllc.__doc__ = "HLLC with Einfeldt wave speeds (fluxes.py:101-143), on the GPU."

INTERFACE_FLUXES: dict[str, Callable] = {"rusanov": rusanov, "roe": roe, "hllc": hllc}


def get_interface_flux(name: str) -> Callable:
    """Return the interface flux with the given stable name."""
    try:
        return INTERFACE_FLUXES[name]
    except KeyError:
        options = ", ".join(sorted(INTERFACE_FLUXES))
        raise ValueError(f"Unknown interface flux {name!r}; choose one of: {options}.") from None
