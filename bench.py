"""Benchmark of the DG Euler RK3 step on B200 (one JSON line on rank 0).

Workload (the 1M-triangle microbenchmark): [0,1]^2 meshed as 724x724 quads,
each split into 2 triangles (K = 1,048,352, P = 4, Np = 15), interior
vertices jittered by seeded uniform +-0.2h; per-node fields are sums of 8
seeded random Fourier modes mapped affinely to rho in [0.5,1.5], u,v in
[-0.5,0.5], p in [0.5,1.5]; every boundary tag is a fixed state at the mean
state; flux=roe, limiter=unlimited (positivity still runs). A step is one full
SSP-RK3 step: 3 fused stages, positivity, device CFL dt and the device
run-loop control. DOF = K * Np solution nodes (4 conserved scalars each).

Headline `value`: DOF-steps/s of the FP32-mixed form with the state resident
in HBM; `fp64` holds the plain FP64 form on the same workload; `l1_rho_vs_fp64`
is the domain-averaged L1 density difference after the timed steps; `e2e`
runs EulerSolver.run() from a pinned host state to a host result; `adjoint`
times the discrete adjoint of 200 RK3 steps of the Sod sensitivity study
(400x40 quads x 2, rusanov/minmod, FP64, checkpoints every 20 steps) against
its forward pass and against the production run loop over the same steps
(also alone: --workload adjoint). `--workload precision` runs the precision
study (Sod 2000x200, hllc/van_leer, t = 0.2, FP32-mixed against FP64) and
`--workload batch` the batched Riemann instances.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (torchrun, one rank per GPU) every rank advances its own
replica of the workload (weak scaling; the path needs no data exchange
between replicas) and the timing is the maximum over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-steps/s FP32-mixed vs FP64 plain at L1(rho)<=1e-5; adjoint/forward time"
from cfd_demo_b200.workloads import JITTER, NX  # noqa: E402

NP_NODES = 15
PRECISION_STEPS = 25  # steps of the FP32-mixed vs FP64 comparison
FALLBACK_HBM_GBS = 6650.0
# Algorithmic bytes per element per RK3 step of the three stage launches:
# state read + write per stage, the stage base state in stages 2-3, and the
# per-element geometry (4 metric + 9 face values + face_info + 3 neighbour ids,
# + dt_geo in stage 3). Neighbour-trace gathers are counted once (in the
# neighbour's own read).
# DRAM bytes per element of each stage launch (dram__bytes_read.sum +
# dram__bytes_write.sum) measured by ncu on the autotuned stage kernels (FP32
# shape 9, FP64 shape 5) at 512x512 quads (K = 524,288; the 724x724 workload
# is too large for a full capture),
# scaled to a launch of the benchmark by its element count (traffic grows in
# proportion to K). Writes still in L2 when a launch ends are not counted
# there, so the stage result's 240 / 480 B appear partly.
NCU_BYTES_PER_ELEMENT = {"fp32_mixed": (480.2, 739.5, 750.5), "fp64": (1007.3, 1522.3, 1528.0)}
# Warp instructions issued per element of each stage launch (ncu
# smsp__inst_executed.sum / K, same captures). With 148 SMs issuing at most
# 4 warp instructions per cycle each, they bound a launch from below at
# instructions / (148 * 4 * SM clock): the instruction-issue roofline.
NCU_WARP_INSTRUCTIONS_PER_ELEMENT = {"fp32_mixed": (267.0, 289.2, 304.9), "fp64": (512.1, 527.1, 581.3)}
SMS, ISSUE_PER_SM_CYCLE = 148, 4


def stage_bytes(real_bytes: int) -> list[int]:
    state = 60 * real_bytes
    geo = 13 * real_bytes + 4 + 12
    return [2 * state + geo, 3 * state + geo, 3 * state + geo + 8]


# ---------------------------------------------------------------- workload ---
def make_workload(nx: int = NX, precision: str = "fp32_mixed", device="cuda"):
    """(solver, initial state as a device (Np, K, 4) float64 tensor)."""
    from cfd_demo_b200.workloads import microbenchmark

    return microbenchmark(nx, precision, device)


# ----------------------------------------------------------- CPU baseline ---
def _oracle_sample_worker(args):
    """Time RK3 steps of the oracle on an nx x nx sample of the workload: one
    untimed warm-up step, then as many timed steps as fit in `budget_s`
    (at least one, at most `steps`); returns (elements, steps, seconds)."""
    nx, steps, budget_s = args
    sys.path.insert(0, ROOT)
    import oracle
    from cfd_demo_b200.workloads import GAMMA, MEAN_STATE, conserved_fields, microbenchmark_mesh
    from oracle.physics import FixedState

    m = microbenchmark_mesh(nx)
    om = oracle.mesh.TriangleMesh(np.array(m.vertices), np.array(m.elements),
                                  {k: np.array(v) for k, v in m.boundary_edges.items()})
    mean = FixedState.from_primitive(*MEAN_STATE, GAMMA)
    s = oracle.OracleSolver(om, {t: mean for t in ("left", "right", "bottom", "top")}, flux="roe",
                            limiter="unlimited", gamma=GAMMA)
    x, y = s.node_coordinates()
    q = conserved_fields(x, y, np)
    w0 = time.perf_counter()
    dt = s.time_step(q)
    q, _ = s.step(q, dt)
    per_step = time.perf_counter() - w0
    n = max(1, min(steps, int(budget_s / max(per_step, 1e-9))))
    t0 = time.perf_counter()
    for _ in range(n):
        dt = s.time_step(q)
        q, _ = s.step(q, dt)
    return s.mesh.num_elements, n, time.perf_counter() - t0


def cpu_baseline(nx: int, steps: int, processes: int, budget_s: float = 90.0) -> dict:
    """The CPU oracle (NumPy restatement of the reference) on `processes`
    spawned workers, each timing RK3 steps of an nx x nx sample of the
    workload (at most `steps`, within `budget_s` of CPU time per worker). With
    nx = 724 / sqrt(processes) the workers together hold about the
    benchmark's K elements."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes) as pool:
        results = pool.map(_oracle_sample_worker, [(nx, steps, budget_s)] * processes)
    k = results[0][0]
    # whole-job rate: every worker's DOF-steps over the slowest worker's time
    slowest = max(r[2] for r in results)
    value = sum(r[0] * NP_NODES * r[1] for r in results) / slowest
    n = min(r[1] for r in results)
    return {"value": value, "unit": "DOF-steps/s", "cores": processes, "kind": "port",
            "sample": f"{processes} process(es), each {n}+ RK3 steps of a {nx}x{nx}-quad sample of the workload "
                      f"(K={k} per process, {processes * k} in all; roe/unlimited, jitter 0.2h, Fourier fields), "
                      f"NumPy float64 oracle after one warm-up step; slowest worker {slowest:.1f} s",
            "elements_total": processes * k}


def sample_nx(processes: int) -> int:
    """Quads per side of each worker's sample: together the workers cover
    about the benchmark's 724 x 724 quads."""
    return max(8, int(round(NX / math.sqrt(max(processes, 1)))))


# ----------------------------------------------------------------- clocks ---
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str):
        self.bus_id = bus_id.lower()
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # the timed region starts only once nvidia-smi is sampling
        deadline = time.time() + 10.0
        while self.proc is not None and time.time() < deadline and self.proc.poll() is None:
            self.file.flush()
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)
        self.start_offset = os.path.getsize(self.file.name)
        self.end_offset = None
        return self

    def mark_start(self) -> None:
        """Samples from here on belong to the timed region."""
        self.file.flush()
        self.start_offset = os.path.getsize(self.file.name)

    def mark_end(self) -> None:
        """End of the timed region; waits for one more sample so that the
        region's last interval is covered."""
        size = os.path.getsize(self.file.name)
        deadline = time.time() + 1.0
        while time.time() < deadline and os.path.getsize(self.file.name) == size:
            time.sleep(0.01)
        self.end_offset = os.path.getsize(self.file.name)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            f.seek(getattr(self, "start_offset", 0))
            text = f.read() if self.end_offset is None else f.read(self.end_offset - self.start_offset)
            for line in text.splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                bus = parts[1].lower()
                if self.bus_id and not bus.startswith(self.bus_id):
                    continue
                rows.append(parts)
        if not rows:
            with open(self.file.name) as f:
                head = f.read(300).strip().splitlines()
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"],
                    "bus_id": self.bus_id, "first_line": head[0] if head else None}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[6:10]) if v.strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][3]),
                "reasons": reasons, "samples": len(rows), "power_w_max": max(float(r[4]) for r in rows)}


# -------------------------------------------------------------- GPU timing ---
def max_over_ranks(values, world: int, device) -> list:
    """Element-wise maximum of per-rank timings (the replicas' whole-job time
    is that of the slowest rank); identity on one rank."""
    if world <= 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def _barrier(world: int) -> None:
    import torch

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()


def timed_steps(solver, steps: int, warmup: int, world: int = 1, stage_events: bool = True, sampler=None,
                min_seconds: float = 1.0, max_repeats: int = 200, repeats: int | None = None) -> dict:
    """Advance the resident state `warmup` + `steps` RK3 steps (device CFL dt,
    device run-loop control); time the `steps` with CUDA events on the
    launching stream, and each stage launch separately. The block of exactly
    `steps` steps is timed back to back `repeats` times (the same count on
    every rank), enough blocks for the clock samples to span `min_seconds`;
    each block is bracketed by a barrier and a device synchronisation."""
    import ctypes as C

    import torch

    from cfd_demo_b200 import _native

    lib, st = solver._lib, solver.native
    ws = solver._ws
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    ptr = C.byref(st)
    x0, x1, sg = ws.x0.data_ptr(), ws.x1.data_ptr(), ws.stage.data_ptr()

    def one_step(ev=None):
        _native.check(lib.cfd_rk3_begin(ptr, sp))
        for k in (1, 2, 3):
            if ev is not None:
                ev[k - 1][0].record(stream)
            _native.check(lib.cfd_rk3_stage(ptr, x0, x1, sg, k, sp))
            if ev is not None:
                ev[k - 1][1].record(stream)
        _native.check(lib.cfd_rk3_finish(ptr, sp))
        _native.check(lib.cfd_run_control(ptr, sp))

    def block():
        evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(3)] for _ in range(steps)]
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _barrier(world)
        start.record(stream)
        for i in range(steps):
            one_step(evs[i] if stage_events else None)
        stop.record(stream)
        _barrier(world)
        return start.elapsed_time(stop), [sum(evs[i][k][0].elapsed_time(evs[i][k][1]) for i in range(steps))
                                          for k in range(3)]

    for _ in range(warmup):
        one_step()
    if sampler is not None:
        sampler.mark_start()
    totals, stages = [], []
    t, sm = block()
    totals.append(t)
    stages.append(sm)
    if repeats is None:
        repeats = min(max_repeats, max(1, math.ceil(min_seconds * 1e3 / max(t, 1e-3))))
        repeats = int(max_over_ranks([repeats], world, torch.device("cuda", torch.cuda.current_device()))[0])
    for _ in range(repeats - 1):
        t, sm = block()
        totals.append(t)
        stages.append(sm)
    if sampler is not None:
        sampler.mark_end()
    c = solver._read(ws.control, _native.CfdControl)
    if c.status != _native.RUN_ACTIVE:
        raise RuntimeError(f"run-loop status {c.status} during the benchmark")
    med = int(np.argsort(totals)[len(totals) // 2])
    return {"total_ms": totals[med], "stage_ms": stages[med], "block_ms": totals, "repeats": repeats,
            "launches_per_step": 6, "time": c.time, "steps_done": c.steps,
            "flux_integral": np.array(c.flux_integral[:])}


def l1_density(solver, qa, qb) -> float:
    """Domain-averaged L1 of rho_a - rho_b by the nodal quadrature."""
    w = solver.reference.cell_weights
    jac = np.asarray(solver.geometry.jacobian)
    diff = np.abs(qa[..., 0] - qb[..., 0])
    return float(np.einsum("i,ik,k->", w, diff, jac) / np.einsum("i,k->", w, jac))


def measured_peak_hbm() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def run_ours(args, rank: int, world: int) -> dict | None:
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nx = args.nx
    steps, warmup = args.steps, args.warmup

    t_setup = time.perf_counter()
    fp32, q0 = make_workload(nx, "fp32_mixed", dev)
    fp64 = fp32.with_precision("fp64")
    setup_s = time.perf_counter() - t_setup
    from cfd_demo_b200.autotune import autotune

    tuned = {}
    for name, solver in (("fp32_mixed", fp32), ("fp64", fp64)):
        variant = args.variant_fp64 if name == "fp64" and args.variant_fp64 is not None else args.variant
        if variant is None:
            tuned[name] = autotune(solver, q0)
        else:
            solver.set_variant(variant)
            tuned[name] = {"choice": (variant, 0), "ms": {}}
    k = fp32.mesh.num_elements
    dof = k * NP_NODES

    results = {}
    # FP32-mixed first: its block count is reused for FP64, so that both forms
    # take the same number of steps and their end states can be compared
    forms = (("fp32_mixed", fp32), ("fp64", fp64))
    if args.profile_form:  # one form's timed steps only: the command line of the profiler captures
        forms = tuple(f for f in forms if f[0] == args.profile_form)
    props = torch.cuda.get_device_properties(dev)
    # nvidia-smi prints the PCI address as dddddddd:bb:dd.f
    bus = "%08x:%02x:%02x" % (int(getattr(props, "pci_domain_id", 0) or 0),
                              int(getattr(props, "pci_bus_id", 0) or 0),
                              int(getattr(props, "pci_device_id", 0) or 0))
    for name, solver in forms:
        solver.begin_run(q0, math.inf)
        sampler = ClockSampler(bus)
        with sampler:
            if name == "fp32_mixed":
                r = timed_steps(solver, steps, warmup, world, sampler=sampler, min_seconds=args.min_seconds)
            else:
                r = timed_steps(solver, steps, warmup, world, sampler=sampler, min_seconds=args.min_seconds,
                                repeats=results["fp32_mixed"]["repeats"] if "fp32_mixed" in results else None)
        r["clocks"] = sampler.summary()
        results[name] = r

    if args.profile_form:
        r = results[args.profile_form]
        if rank == 0:
            print(json.dumps({"profile_form": args.profile_form, "elements": fp32.mesh.num_elements,
                              "ms_per_step": r["total_ms"] / steps, "stage_ms": [v / steps for v in r["stage_ms"]],
                              "stage_kernel": list(tuned[args.profile_form]["choice"])}), flush=True)
        return None

    # max over ranks of the timed region
    m32, m64 = max_over_ranks([results["fp32_mixed"]["total_ms"], results["fp64"]["total_ms"]], world, dev)
    tot = {"fp32_mixed": m32, "fp64": m64}

    # end to end through the public API: pinned host state in, host result out
    host_q0 = q0.cpu().pin_memory()
    t_k = results["fp32_mixed"]["time"]
    fp32.run(host_q0, t_k)  # warm (captures the chunk graphs)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    res = fp32.run(host_q0, t_k)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - w0
    e2e_steps = res.steps
    e2e_s = max_over_ranks([e2e_s], world, dev)[0]

    if rank != 0:
        return None

    peak, peak_kind = measured_peak_hbm()
    out = {}
    for name, real in (("fp32_mixed", 4), ("fp64", 8)):
        r = results[name]
        sb = stage_bytes(real)
        stage_s = [ms / 1e3 / steps for ms in r["stage_ms"]]
        achieved = sum(sb) * k / sum(stage_s) / 1e9
        out[name] = {
            "value": world * dof * steps / (tot[name] / 1e3),
            "ms_per_step": tot[name] / steps,
            "stage_ms": [round(1e3 * s, 4) for s in stage_s],
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": round(sum(NCU_BYTES_PER_ELEMENT[name]) * k / 3),
                         "traffic_note": "bytes per stage launch (mean of the 3 launches of a step), ncu at "
                                         "K=524,288 scaled to this K; algorithmic bytes per launch "
                                         f"{round(sum(sb) * k / 3)}",
                         "peak_source": peak_kind, "algorithmic_bytes_per_element_step": sum(sb)},
        }
        mhz = r["clocks"].get("sm_mhz") if r.get("clocks") else None
        if mhz:
            inst = NCU_WARP_INSTRUCTIONS_PER_ELEMENT[name]
            bound_s = [n * k / (SMS * ISSUE_PER_SM_CYCLE * mhz * 1e6) for n in inst]
            out[name]["issue_roofline"] = {
                "warp_instructions_per_element": list(inst), "sm_mhz": mhz,
                "bound_ms": [round(1e3 * b, 4) for b in bound_s],
                "frac": round(sum(bound_s) / sum(stage_s), 4),
                "note": "instruction-issue bound of the three stage launches (148 SMs x 4 warp instructions per "
                        "cycle at the median SM clock of the timed region; instruction counts from ncu at "
                        "K=524,288, per element) over their CUDA-event time"}
    # precision: both forms advance the same state by PRECISION_STEPS steps of
    # the run loop (each with its own device CFL steps), untimed
    states, conservation = {}, {}
    for name, solver in (("fp32_mixed", fp32), ("fp64", fp64)):
        solver.begin_run(q0, math.inf)
        c = solver.advance(PRECISION_STEPS)
        states[name] = solver.download(solver.state_tensor())
        defect = solver.integrate(states[name]) - solver.integrate(q0) + np.array(c.flux_integral[:])
        conservation[name] = {"mass_defect": float(defect[0]), "energy_defect": float(defect[3]),
                              "time": float(c.time), "steps": int(c.steps)}
    l1 = l1_density(fp32, states["fp32_mixed"], states["fp64"])
    linf = float(np.abs(states["fp32_mixed"][..., 0] - states["fp64"][..., 0]).max())
    state_bytes = q0.numel() * 8
    line = {
        "metric": METRIC,
        "value": out["fp32_mixed"]["value"],
        "unit": "DOF-steps/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": out["fp32_mixed"]["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"1M-triangle RK3 microbenchmark: {nx}x{nx} quads x 2 triangles, jitter +-{JITTER}h, "
                        "8-mode Fourier fields, roe/unlimited, fixed-state boundaries",
            "elements_per_gpu": k, "np": NP_NODES, "dof_per_gpu": dof, "flux": "roe", "limiter": "unlimited",
            "precision": "fp32_mixed (f32 state/arithmetic; f64 averages, positivity, reductions)",
            "dof_definition": "K*Np solution nodes, each with 4 conserved scalars",
            "step": "one SSP-RK3 step: 3 fused stage kernels + device CFL dt + device run-loop control",
            "l2": "inputs larger than L2 (state 252 MB f32 / 503 MB f64 per buffer > 126 MB)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "setup_s": round(setup_s, 2),
            "stage_kernel": {n: {"choice": list(t["choice"]), "attempt_ms": {k: round(v, 4) for k, v in t["ms"].items()}}
                             for n, t in tuned.items()},
        },
        "roofline": out["fp32_mixed"]["roofline"],
        "issue_roofline": out["fp32_mixed"].get("issue_roofline"),
        "stage_ms": out["fp32_mixed"]["stage_ms"],
        "fp64": {"value": out["fp64"]["value"], "ms_per_step": out["fp64"]["ms_per_step"],
                 "stage_ms": out["fp64"]["stage_ms"], "roofline": out["fp64"]["roofline"],
                 "issue_roofline": out["fp64"].get("issue_roofline"), "dtype": "f64",
                 "clocks": results["fp64"].get("clocks")},
        "fp32_over_fp64": out["fp32_mixed"]["value"] / out["fp64"]["value"],
        "l1_rho_vs_fp64": l1,
        "linf_rho_vs_fp64": linf,
        "conservation": conservation,
        "precision_note": f"FP32-mixed and FP64 states after {PRECISION_STEPS} steps of the run loop from the "
                          "workload's state, each with its own device CFL steps (end times in `conservation`); "
                          "defects = final - initial integral + time-integrated boundary flux",
        "timing": {"repeats": results["fp32_mixed"]["repeats"], "block_steps": steps,
                   "block_ms_fp32_mixed": [round(v, 4) for v in results["fp32_mixed"]["block_ms"]],
                   "note": "each block times exactly `steps` RK3 steps (barrier + synchronise on both sides); "
                           "value and ms_per_step from the median block; blocks repeat until the clock samples "
                           "span >= 1 s"},
        "e2e": {"value": world * dof * e2e_steps / e2e_s, "unit": "DOF-steps/s",
                "h2d_bytes_per_step": state_bytes / e2e_steps, "d2h_bytes_per_step": (state_bytes + 104 * e2e_steps) / e2e_steps,
                "api": "EulerSolver.run(pinned host (Np,K,4) float64 state, t_K) -> RunResult with host state",
                "steps": e2e_steps, "seconds": e2e_s},
        "gpu_launches": 6 * steps,
        "clocks": results["fp32_mixed"]["clocks"],
    }
    if line["clocks"].get("sm_mhz"):
        # time x clock: comparable across runs at different SM clocks
        line["clocks"]["kcycles_per_step"] = round(line["ms_per_step"] * line["clocks"]["sm_mhz"], 1)
    return line


def run_batch(args, sequential_stride: int = 1, count: int | None = None) -> dict:
    """The batching form: seeded Riemann instances of uneven size (hllc/superbee,
    FP32-mixed) advanced together from t = 0 to t = 0.15, each with its own
    CFL steps, against the same instances advanced one at a time
    (EulerSolver.run, graph-replayed run loop). The batch's execution form
    (one persistent launch per chunk, or graph chunks of the separate
    launches) and tile shape are picked by the autotuner. The sequential arm
    times every `sequential_stride`-th instance; the ratio is of DOF-steps/s
    (sum over instances of K_i Np x steps_i per second of wall time)."""
    import torch

    from cfd_demo_b200 import EulerSolver, SolverConfig
    from cfd_demo_b200.autotune import autotune_batch
    from cfd_demo_b200.batch import BatchedEulerSolver, riemann_batch

    torch.cuda.set_device(0)
    cases = riemann_batch(count or args.batch_count, seed=0)
    cfg = SolverConfig(flux="hllc", limiter="superbee", gamma=1.4, precision="fp32_mixed")
    t_end = args.batch_final_time
    states = [c.initial_state for c in cases]
    batch = BatchedEulerSolver(cases, cfg, graph_chunk=args.batch_chunk)
    tuned = autotune_batch(batch, states, t_end)
    cap = args.batch_max_attempts
    batch.run_to(states, t_end, max_attempts=256)  # warm-up: captures every chunk size's graph
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctl = batch.run_to(states, t_end, max_attempts=cap)
    torch.cuda.synchronize()
    batched_s = time.perf_counter() - t0
    done = np.array([c.steps for c in ctl])
    sizes = np.array([c.mesh.num_elements for c in cases])
    status = np.array([c.status for c in ctl])
    dof_steps = float((done * sizes * NP_NODES).sum())
    picked = list(range(0, len(cases), sequential_stride))
    seq_s, seq_dof, mismatched = 0.0, 0.0, []
    for i in picked:
        c = cases[i]
        single = EulerSolver(c.mesh, c.boundary_conditions, cfg, graph_chunk=args.batch_chunk)
        single.set_variant(9)
        single.begin_run(c.initial_state, t_end)  # warm-up: captures the chunk graphs
        for n in (1, 2, 4, 8, 16, 32, 64):
            if n <= args.batch_chunk:
                single.advance(n)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        single.begin_run(c.initial_state, t_end)
        chunk, attempts = 1, 0
        while True:
            cs = single.advance(chunk)
            attempts += chunk
            if cs.status != 0 or attempts >= cap:
                break
            chunk = min(2 * chunk, args.batch_chunk)
        torch.cuda.synchronize()
        seq_s += time.perf_counter() - t1
        seq_dof += cs.steps * c.mesh.num_elements * NP_NODES
        if cs.steps != done[i] or cs.status != status[i]:
            mismatched.append(i)
    seq_value = seq_dof / seq_s if seq_s else None
    names = {1: "done", -1: "bad CFL step", -2: "too many rejections", 0: f"still active after {cap} attempts"}
    return {
        "metric": "batched vs sequential DOF-steps/s (seeded Riemann instances to t = 0.15)",
        "value": dof_steps / batched_s, "unit": "DOF-steps/s", "n_gpus": 1, "higher_is_better": True,
        "data": "synthetic", "dtype": "f32",
        "config": {"workload": f"{len(cases)} seeded Riemann instances on [0,1]x[0,0.1] (left/right rho, p uniform in "
                               f"[0.1,1], u = v = 0), nx in 50..400, ny = floor(nx/10), hllc/superbee, FP32-mixed, "
                               f"t = 0 -> {t_end}",
                   "elements_total": int(sizes.sum()), "instances": len(cases),
                   "execution": {"choice": list(tuned["choice"]), "attempt_chunk_ms": tuned["ms"]}},
        "batched_seconds": batched_s, "batched_instance_steps": int(done.sum()), "max_steps": int(done.max()),
        "instances_by_status": {names.get(int(k), str(k)): int((status == k).sum()) for k in np.unique(status)},
        "stopped_early": [{"instance": int(i), "status": names.get(int(status[i])), "steps": int(done[i]),
                           "time": float(ctl[i].time), "dt": float(ctl[i].dt),
                           "nx": int(len(np.unique(cases[i].mesh.vertices[:, 0])) - 1)}
                          for i in np.nonzero(status != 1)[0]],
        "sequential": {"instances_timed": len(picked), "stride": sequential_stride, "seconds": seq_s,
                       "value": seq_value, "step_count_mismatches": mismatched},
        "speedup_vs_sequential": (dof_steps / batched_s) / seq_value if seq_value else None,
    }


def run_adjoint(args) -> dict:
    """The differentiation form: the sensitivity study on the Sod tube 400x40
    (K = 32,000, rusanov/minmod, FP64), 200 CFL steps, checkpoints every 20
    steps. Times, with CUDA events, the forward pass of the fixed-schedule run
    (keeping checkpoints), the backward pass (segment recompute with the tape
    + adjoint steps), and the production run loop (EulerSolver.advance,
    graph-replayed) over the same 200 steps."""
    import torch

    from cfd_demo_b200.adjoint import AdjointRun, SodSensitivity, cfl_schedule

    torch.cuda.set_device(0)
    steps, every = args.adjoint_steps, 20
    case = SodSensitivity(400, 40, flux="rusanov", limiter="minmod", seed=0)
    dev = case.solver.operators.device
    q0 = case.initial_state(torch.tensor(case.rho_left, dtype=torch.float64, device=dev))
    dts = cfl_schedule(case.solver, q0.cpu().numpy(), steps=steps)
    runner = AdjointRun(case.solver, dts, checkpoint_every=every)
    x0 = runner.pack(q0)
    g = runner.pack(torch.stack([case.weight] + [torch.zeros_like(case.weight)] * 3, dim=-1))

    def timed(fn, repeats=3):
        fn()  # warm-up
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(repeats):
            out = fn()
        stop.record()
        stop.synchronize()
        return start.elapsed_time(stop) / repeats, out

    fwd_ms, (xT, checkpoints) = timed(lambda: runner.forward(x0))
    bwd_ms, _ = timed(lambda: runner.backward(g, checkpoints))
    solver = case.solver
    solver.begin_run(q0.cpu().numpy(), math.inf)

    def production():
        solver.begin_run(q0.cpu().numpy(), math.inf)
        return solver.advance(steps)

    run_ms, _ = timed(production, repeats=2)
    return {
        "workload": f"Sod 400x40 quads x 2 (K={solver.mesh.num_elements}), rusanov/minmod, FP64, {steps} CFL steps, "
                    f"checkpoints every {every}",
        "forward_ms": fwd_ms, "backward_ms": bwd_ms, "run_loop_ms": run_ms,
        "adjoint_over_forward": bwd_ms / fwd_ms,
        "adjoint_over_run_loop": bwd_ms / run_ms,
        "note": "backward = segment recompute with the tape + adjoint steps; run_loop = EulerSolver.advance "
                "(graph-replayed device run loop, includes begin_run) over the same steps",
    }


def run_precision(args) -> dict:
    """The precision study: the Sod tube on 2000x200 quads x 2 (K = 800,000),
    hllc/van_leer, to t = 0.2, in the FP32-mixed and the plain FP64 form
    (the FP64 GPU run is the reference: the CPU oracle would take weeks).
    Reports the L1 / Linf density difference between the two final states,
    each form's L1 errors against the exact solution, the shock and contact
    positions from column-averaged density, and the mass / energy
    conservation defects against the time-integrated boundary fluxes."""
    import torch

    from cfd_demo_b200 import sod_shock_tube
    from cfd_demo_b200.cases import SOD_DISCONTINUITY, SOD_GAMMA, SOD_LEFT, SOD_RIGHT
    from cfd_demo_b200.verification import ExactRiemann, column_density, front_position, l1_errors

    torch.cuda.set_device(0)
    nx, ny = args.precision_nx, args.precision_nx // 10
    case = sod_shock_tube(nx, ny, flux="hllc", limiter="van_leer", precision="fp64")
    solvers = {"fp64": case.solver, "fp32_mixed": case.solver.with_precision("fp32_mixed")}
    exact = ExactRiemann((SOD_LEFT[0], SOD_LEFT[1], SOD_LEFT[3]), (SOD_RIGHT[0], SOD_RIGHT[1], SOD_RIGHT[3]),
                         SOD_GAMMA, SOD_DISCONTINUITY)
    t_end = case.final_time
    waves = exact.wave_positions(t_end)
    from cfd_demo_b200.autotune import autotune

    out, states, shapes = {}, {}, {}
    for name, solver in solvers.items():
        if args.variant is None:  # stage-kernel shape picked outside the timed run
            shapes[name] = autotune(solver, case.initial_state)["choice"]
        else:
            solver.set_variant(args.variant)
            shapes[name] = (args.variant, 0)
        initial = solver.integrate(case.initial_state)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = solver.run(case.initial_state, t_end)
        wall = time.perf_counter() - t0
        q = torch.from_numpy(res.state).cuda()
        states[name] = q
        cols, faces = column_density(q, solver.mesh, nx)
        defect = solver.integrate(res.state) - initial + res.boundary_flux_integral
        out[name] = {
            "steps": res.steps, "rejected": res.rejected_steps, "wall_s": wall,
            "dof_steps_per_s": res.steps * solver.mesh.num_elements * NP_NODES / wall,
            "l1_vs_exact": l1_errors(q, solver.mesh, exact, res.time, SOD_GAMMA, n=args.precision_quad),
            "shock_x": front_position(cols, faces, (waves["shock"] - 0.05, waves["shock"] + 0.05)),
            "contact_x": front_position(cols, faces, (waves["contact"] - 0.05, waves["contact"] + 0.05)),
            "mass_defect": float(defect[0]), "energy_defect": float(defect[3]),
            "max_troubled_cells": res.max_troubled_cells, "min_density": res.min_density,
            "min_pressure": res.min_pressure, "stage_kernel": shapes[name],
        }
    d = (states["fp32_mixed"][..., 0] - states["fp64"][..., 0]).abs()
    w = torch.as_tensor(case.solver.reference.cell_weights, device=d.device, dtype=d.dtype)
    l1 = float(torch.einsum("n,nk->", w, d) / (w.sum() * d.shape[1]))  # elements have equal area
    return {
        "metric": "precision study: FP32-mixed vs FP64 on the Sod tube", "unit": "density difference",
        "config": {"workload": f"Sod tube {nx}x{ny} quads x 2 (K={case.solver.mesh.num_elements}), hllc/van_leer, "
                               f"t={t_end}", "quadrature": f"{args.precision_quad}x{args.precision_quad} "
                               "collapsed Gauss per (sub-)triangle, elements cut at the exact waves"},
        "l1_rho_fp32_vs_fp64": l1, "linf_rho_fp32_vs_fp64": float(d.max()),
        "exact_waves": waves, "fp64": out["fp64"], "fp32_mixed": out["fp32_mixed"],
        "fp32_over_fp64_dof_steps": out["fp32_mixed"]["dof_steps_per_s"] / out["fp64"]["dof_steps_per_s"],
    }


def _oblique_oracle_rate(nx: int, ny: int, steps: int) -> float:
    """The oracle's DOF-steps/s on the oblique-shock case (one process)."""
    import oracle
    from oracle.physics import ExactState as OExact, FixedState as OFixed, SlipWall as OSlip

    from cfd_demo_b200.cases import OBLIQUE_GAMMA, OBLIQUE_HEIGHT, OBLIQUE_LENGTH
    from cfd_demo_b200.mesh import sheared_rectangle_mesh
    from cfd_demo_b200.verification import ObliqueShock

    ex = ObliqueShock(2.0, math.radians(10.0), OBLIQUE_GAMMA)
    m = sheared_rectangle_mesh(nx, ny, ex.theta, (0.0, OBLIQUE_LENGTH), (0.0, OBLIQUE_HEIGHT))
    om = oracle.mesh.TriangleMesh(np.array(m.vertices), np.array(m.elements),
                                  {k: np.array(v) for k, v in m.boundary_edges.items()})
    far = OExact(ex.conserved, ex.cell_average)
    s = oracle.OracleSolver(om, {"left": OFixed.from_primitive(*ex.upstream, OBLIQUE_GAMMA), "bottom": OSlip(),
                                 "top": far, "right": far}, flux="rusanov", limiter="minmod", gamma=OBLIQUE_GAMMA)
    q = np.broadcast_to(np.array(OFixed.from_primitive(*ex.upstream, OBLIQUE_GAMMA).state), s.state_shape).copy()
    q, _ = s.step(q, s.time_step(q))  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        q, _ = s.step(q, s.time_step(q))
    return steps * m.num_elements * NP_NODES / (time.perf_counter() - t0)


def run_oblique(args) -> dict:
    """The oblique-shock verification case (exact far-field boundaries on a
    sheared mesh; CFD-demo proposes it in its ADR 0011 / 0012): baseline
    M1 = 2, wall 10 deg, rusanov/minmod, FP64, 200x100 quads x 2 (K = 40,000)
    to t = 2 through EulerSolver.run, timed on the wall clock; the ADR's
    acceptance quantities; the oracle's rate on the same mesh (a few steps,
    one host core) beside it."""
    import torch

    from cfd_demo_b200 import oblique_shock
    from cfd_demo_b200.verification import oblique_l1_errors, shock_angle_at

    nx, ny = args.oblique_nx, args.oblique_nx // 2
    oracle_rate = _oblique_oracle_rate(nx, ny, 3) if not args.no_cpu_baseline else None
    torch.cuda.set_device(0)
    case = oblique_shock(nx, ny, flux="rusanov", limiter="minmod")
    s, ex = case.solver, case.exact
    from cfd_demo_b200.autotune import autotune

    shape = autotune(s, case.initial_state)["choice"] if args.variant is None else (args.variant, 0)
    if args.variant is not None:
        s.set_variant(args.variant)
    s.run(case.initial_state, 0.01)  # warm-up: captures the run loop's graphs
    initial = s.integrate(case.initial_state)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = s.run(case.initial_state, case.final_time)
    wall = time.perf_counter() - t0
    q = torch.from_numpy(res.state).cuda()
    err = oblique_l1_errors(q, s.mesh, ex, 1.4)
    angle = shock_angle_at(q, s.mesh, ex, 0.5 * case.length, case.height)
    defect = s.integrate(res.state) - initial + res.boundary_flux_integral
    rate = res.steps * s.mesh.num_elements * NP_NODES / wall
    return {
        "metric": "oblique-shock run DOF-steps/s (EulerSolver.run, wall clock)", "value": rate,
        "unit": "DOF-steps/s", "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"oblique shock M1 = 2, wall 10 deg, {nx}x{ny} quads x 2 (K={s.mesh.num_elements}), "
                               "rusanov/minmod, exact far-field top and right, t = 0 -> 2"},
        "stage_kernel": list(shape), "steps": res.steps, "seconds": wall,
        "l1": {k: v for k, v in err.items() if k != "area"},
        "shock_angle_deg": math.degrees(angle), "exact_beta_deg": math.degrees(ex.beta),
        "conservation_defect_max": float(np.abs(defect).max()),
        "cpu_oracle": {"value": oracle_rate, "unit": "DOF-steps/s", "cores": 1, "kind": "port",
                       "sample": f"3 RK3 steps of the same {nx}x{ny} case after one warm-up step"},
    }


def run_reference(args) -> dict:
    """The reference arm: the CPU oracle (NumPy restatement of the reference's
    own algorithm; the reference itself is JAX code that cannot be installed
    on the box) on every host core, each worker advancing its own share-sized
    sample of the workload."""
    procs = args.cpu_procs or os.cpu_count() or 1
    nx = args.ref_nx or sample_nx(procs)
    base = cpu_baseline(nx, args.steps, procs, budget_s=args.ref_budget)
    return {
        "metric": METRIC, "value": base["value"], "unit": "DOF-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"1M-triangle RK3 microbenchmark split into {procs} samples of {nx}x{nx} quads x 2 "
                               f"({base['elements_total']} elements in all), roe/unlimited", "flux": "roe",
                   "limiter": "unlimited"},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "DOF-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--ref-nx", type=int, default=0, help="CPU sample quads per side (default: 724/sqrt(processes))")
    ap.add_argument("--ref-budget", type=float, default=90.0, help="seconds of timed CPU work per worker")
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--cpu-baseline-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=None, help="stage-kernel variant (default: autotuned)")
    ap.add_argument("--variant-fp64", type=int, default=None,
                    help="stage-kernel variant of the FP64 form (default: as --variant); fixing both to the "
                         "autotuner's choices reproduces a run's kernels under a profiler, whose serialised "
                         "launches would mislead the autotuner")
    ap.add_argument("--workload", choices=["microbenchmark", "batch", "adjoint", "precision", "oblique"],
                    default="microbenchmark")
    ap.add_argument("--oblique-nx", type=int, default=200)
    ap.add_argument("--precision-nx", type=int, default=2000)
    ap.add_argument("--precision-quad", type=int, default=6)
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint timing of the default line")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-instances timing of the default line")
    ap.add_argument("--min-seconds", type=float, default=1.0,
                    help="repeat the timed block of `steps` steps until the clock samples span this long (0: once)")
    ap.add_argument("--profile-form", choices=["fp32_mixed", "fp64"], default=None,
                    help="time only this form's steps and print a short line (for profiler captures)")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-final-time", type=float, default=0.15)
    ap.add_argument("--batch-chunk", type=int, default=64, help="attempts per graph chunk of the batch run")
    ap.add_argument("--batch-max-attempts", type=int, default=15000,
                    help="attempts after which instances still running are reported as such")
    ap.add_argument("--batch-stride", type=int, default=1, help="time every n-th instance in the sequential arm")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.workload == "batch":
        if rank == 0:
            print(json.dumps(run_batch(args, args.batch_stride)), flush=True)
        return
    if args.workload == "adjoint":
        if rank == 0:
            print(json.dumps(run_adjoint(args)), flush=True)
        return
    if args.workload == "precision":
        if rank == 0:
            print(json.dumps(run_precision(args)), flush=True)
        return
    if args.workload == "oblique":
        if rank == 0:
            print(json.dumps(run_oblique(args)), flush=True)
        return

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return

    # CPU baseline first (spawned workers, before any CUDA context)
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = args.cpu_procs or os.cpu_count() or 1
        base = cpu_baseline(args.ref_nx or sample_nx(procs), args.cpu_baseline_steps, procs, budget_s=20.0)

    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        torch.distributed.barrier()
    line = run_ours(args, rank, world)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        line["cpu_baseline"] = base
        if world == 1 and not args.no_adjoint:
            line["adjoint"] = run_adjoint(args)
        if world == 1 and not args.no_batch:
            # the first 64 instances of the family (the full 256: --workload batch)
            line["batch"] = run_batch(args, sequential_stride=4, count=64)
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
