// control.cuh — the per-instance scalar steps of an attempt: zeroing the
// reduction slots, the StepReport (time_integration.py:69-83 of CFD-demo) and
// one pass of the run-loop body (solver.py:180-204), as device functions used
// by the small kernels of kernels.cu and by the persistent batch kernel.
// Included by common.cuh inside namespace cfd.
#pragma once

__device__ __forceinline__ void reset_acc_one(CfdStageAcc* acc, int i) {
  CfdStageAcc z;
  z.boundary_flux[0] = z.boundary_flux[1] = z.boundary_flux[2] = z.boundary_flux[3] = 0.0;
  z.min_rho_key = z.min_p_key = z.dt_key = KEY_EMPTY;
  z.troubled = 0;
  z.flags = 0;
  acc[i] = z;
}

__device__ __forceinline__ double key_min_value(unsigned long long k) {
  return k == KEY_EMPTY ? INFINITY : dkey_decode(k);
}

// StepReport of instance i's attempt (time_integration.py:69-83).
__device__ __forceinline__ void report_one(const CfdStageAcc* acc, const CfdControl* ctl, CfdStepReport* rep, int i,
                                           double cfl) {
  if (ctl[i].status != CFD_RUN_ACTIVE) return;
  const CfdStageAcc* a = acc + 3 * i;
  const double dt = ctl[i].dt;
  CfdStepReport r;
  for (int c = 0; c < 4; ++c)
    r.boundary_flux[c] = dt * (a[0].boundary_flux[c] / 6.0 + a[1].boundary_flux[c] / 6.0 + 2.0 * a[2].boundary_flux[c] / 3.0);
  const int fl = a[0].flags | a[1].flags | a[2].flags;
  r.admissible = (fl & FLAG_ADMISSIBILITY) == 0;
  double rmin = INFINITY, pmin = INFINITY;
  int tr = 0;
  for (int s = 0; s < 3; ++s) {
    rmin = fmin(rmin, key_min_value(a[s].min_rho_key));
    pmin = fmin(pmin, key_min_value(a[s].min_p_key));
    tr = max(tr, a[s].troubled);
  }
  if (fl & FLAG_NONFINITE) {
    rmin = NAN;
    pmin = NAN;
  }
  r.min_density = rmin;
  r.min_pressure = pmin;
  r.troubled_cells = tr;
  r.dt = dt;
  r.dt_next = (a[2].flags & FLAG_NAN_DT) ? (double)NAN : cfl * dkey_decode(a[2].dt_key);
  r.reserved[0] = r.reserved[1] = 0;
  rep[i] = r;
}

// One pass of the body of solver.py:180-204 for instance i after an attempt.
__device__ __forceinline__ void control_one(CfdControl* ctl, const CfdStepReport* rep, int i, int max_rejections) {
  CfdControl c = ctl[i];
  if (c.status != CFD_RUN_ACTIVE) return;
  const CfdStepReport r = rep[i];
  if (r.admissible) {
    c.parity ^= 1;
    c.time = c.reaches_end ? c.final_time : c.time + c.dt;
    c.steps += 1;
    for (int k = 0; k < 4; ++k) c.flux_integral[k] += r.boundary_flux[k];
    if (r.min_density < c.min_density) c.min_density = r.min_density;
    if (r.min_pressure < c.min_pressure) c.min_pressure = r.min_pressure;
    c.max_troubled = max(c.max_troubled, r.troubled_cells);
    c.attempts = 0;
    if (!(c.time < c.final_time)) {
      c.status = CFD_RUN_DONE;
    } else {
      const double dt = r.dt_next;
      if (!isfinite(dt) || dt <= 0.0) {
        c.status = CFD_RUN_BAD_DT;
        c.dt = dt;
      } else {
        const double remaining = c.final_time - c.time;
        c.reaches_end = dt >= remaining;
        c.dt = c.reaches_end ? remaining : dt;
      }
    }
  } else {
    c.rejected += 1;
    c.attempts += 1;
    if (c.attempts >= max_rejections + 1) {
      c.status = CFD_RUN_REJECTED;
    } else {
      c.reaches_end = 0;
      c.dt *= 0.5;
    }
  }
  ctl[i] = c;
}
