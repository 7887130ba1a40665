"""The allocation-free RK3 step, cfd_rk3_step_noalloc, through the C ABI.

That entry point serves callers that cannot allocate device memory (a
foreign-language binding holding only the buffers it was handed, or an
application whose memory pool forbids outside allocations): all its scratch
is a static array inside libcfd_b200.so. Here it is checked against the
regular entry point (cfd_rk3_attempt with caller-allocated scratch, which
EulerSolver.step uses) on two calls in a row, in both precisions, and a mesh
larger than the static scratch must be refused. The file name makes pytest
collect it last.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_step(solver, q_host, dt):
    import torch

    from cfd_demo_b200 import _native

    lib = _native.load()
    x_in = solver.upload(q_host)
    x_in_before = x_in.clone()
    x_out = torch.zeros_like(x_in)
    rep = torch.zeros(_native.SIZES["CfdStepReport"], dtype=torch.uint8, device=x_in.device)
    st = solver.native
    rc = lib.cfd_rk3_step_noalloc(C.byref(st.mesh), st.flux, st.limiter, st.precision, st.gamma, st.cfl,
                                  x_in.data_ptr(), x_out.data_ptr(), float(dt), rep.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    _native.check(rc)
    torch.cuda.synchronize()
    # the entry point takes q_in as const: the step must leave it as it was
    assert torch.equal(x_in, x_in_before)
    report = _native.CfdStepReport.from_buffer_copy(rep.cpu().numpy().tobytes())
    return solver.download(x_out), report


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
@pytest.mark.parametrize("flux,limiter", [("rusanov", "minmod"), ("hllc", "unlimited"), ("roe", "superbee")])
def test_noalloc_step_matches_the_regular_entry_point(precision, flux, limiter):
    from cfd_demo_b200 import sod_shock_tube

    case = sod_shock_tube(60, 6, flux=flux, limiter=limiter, precision=precision)
    s = case.solver
    q = case.initial_state
    for _ in range(3):  # a state with some structure
        q, _ = s.step(q, s.time_step(q))
    dt = s.time_step(q)
    ref_q, ref_rep = s.step(q, dt)
    scale = np.maximum(np.abs(ref_q).reshape(-1, 4).max(axis=0), 1e-300)
    tol = 1e-12 if precision == "fp64" else 1e-6
    for _ in range(2):  # two calls in a row share the static scratch
        out_q, rep = _noalloc_step(s, q, dt)
        assert float((np.abs(out_q - ref_q) / scale).max()) <= tol
        assert bool(rep.admissible) == ref_rep.admissible
        assert rep.troubled_cells == ref_rep.troubled_cells
        np.testing.assert_allclose(rep.boundary_flux[:], ref_rep.boundary_flux, rtol=tol, atol=1e-15)
        assert rep.min_density == pytest.approx(ref_rep.min_density, rel=tol)


def test_noalloc_step_refuses_meshes_beyond_its_scratch():
    import torch

    from cfd_demo_b200 import _native, sod_shock_tube

    case = sod_shock_tube(100, 90, flux="rusanov", limiter="minmod")  # K = 18000 > 16384
    s = case.solver
    assert s.operators.ld > _native.NOALLOC_MAX_ELEMENTS
    lib = _native.load()
    x = s.upload(case.initial_state)
    rep = torch.zeros(_native.SIZES["CfdStepReport"], dtype=torch.uint8, device=x.device)
    st = s.native
    rc = lib.cfd_rk3_step_noalloc(C.byref(st.mesh), st.flux, st.limiter, st.precision, st.gamma, st.cfl,
                                  x.data_ptr(), torch.zeros_like(x).data_ptr(), 1e-4, rep.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"static scratch limit" in lib.cfd_last_error()
