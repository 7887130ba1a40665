"""Selectable TVD limiter functions phi(r) (names of CFD-demo
src/cfd_demo/limiters.py:42-57).

Each callable evaluates, on the GPU, the ``__device__`` phi of the limiter
kernel (csrc/physics.cuh) elementwise.
"""

from __future__ import annotations

from collections.abc import Callable

import numpy as np

LIMITER_IDS = {"minmod": 0, "mc": 1, "van_leer": 2, "superbee": 3, "unlimited": 4}


def _device_phi(limiter_id: int) -> Callable:
    def phi(r):
        import torch

        from . import _native

        ra = np.asarray(r, dtype=np.float64)
        d = torch.from_numpy(np.array(ra, dtype=np.float64)).reshape(-1).cuda()  # a copy: r may be read-only
        out = torch.empty_like(d)
        _native.check(_native.load().cfd_limiter_phi(limiter_id, d.numel(), d.data_ptr(), out.data_ptr(),
                                                     torch.cuda.current_stream().cuda_stream))
        return out.cpu().numpy().reshape(ra.shape)

    return phi


minmod = _device_phi(0)
mc = _device_phi(1)
van_leer = _device_phi(2)
superbee = _device_phi(3)
unlimited = _device_phi(4)

LIMITER_FUNCTIONS: dict[str, Callable] = {
    "minmod": minmod, "mc": mc, "van_leer": van_leer, "superbee": superbee, "unlimited": unlimited,
}


def get_limiter_function(name: str) -> Callable:
    """Return the limiter function with the given stable name."""
    try:
        return LIMITER_FUNCTIONS[name]
    except KeyError:
        options = ", ".join(sorted(LIMITER_FUNCTIONS))
        raise ValueError(f"Unknown limiter {name!r}; choose one of: {options}.") from None
