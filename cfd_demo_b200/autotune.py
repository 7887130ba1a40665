"""Autotuner of the stage-kernel shape (elements per block, tile staging).

The fused stage kernel comes in these shapes (CfdSolver.variant):
  0  tiled, 32 elements (64 threads) per block, state and geometry staged in
     shared memory, stage base read from global memory in the epilogue
  1  tiled, 32 elements per block, stage base staged in shared memory too
  2  register-only pair kernel (block size 64/128/256 threads)
  3  tiled, 64 elements (128 threads) per block
  4  tiled, 32 elements per block, registers capped so that 10 (FP32) / 8
     (FP64) blocks fit on an SM instead of 8 / 6
  5  tiled, 64 elements per block, the FP32 face rounds kept rolled (smaller
     code, LIFT from the constant bank)
  6, 7  variants 3 and 5 with scalar FMAs in the FP32 [Dr|Ds] and LIFT
     contractions, which every other tiled shape issues as packed FP32x2 FMAs
     (bitwise the same results; kept as the reference of that claim, not a
     candidate)
  8  tiled, 64 elements per block, stage base staged in shared memory (FP32:
     four blocks still fit an SM's shared memory, as many as the registers
     allow)
  9  shape 8 with the face-node flux as an out-of-line call, so the eight
     unrolled face rounds share one copy of the flux code (FP32; FP64 runs 8)
  10 shape 3 in the face-job form: the block lists the faces it owns (each
     in-tile interior face once), deals their face nodes out to all threads,
     evaluates each face flux once for both sides and lifts the 15 jump
     inputs of each element from shared memory
  11 shape 8 (staged base rows) in the face-job form
  12, 13  shape 9 with the volume node loop kept rolled ([Dr|Ds] columns from
     the constant bank: a fifteenth of the unrolled loop's code, every entry
     taken), with unrolled / rolled face rounds
  14 shape 5 with the volume node loop kept rolled
  (6, 7 and 12-14 are not among the default candidates)
`autotune(solver, state)` times one RK3 attempt per candidate on the solver's
own buffers (an attempt from the same state recomputes the same step, so the
candidates see identical work), keeps the fastest, and remembers the choice per
(GPU, precision, flux, limiter, size bucket) for the life of the process.
"""

from __future__ import annotations

import ctypes as C
import math

from . import _native

# shapes 12-14 are selectable but not candidates: measured on the 1M-element
# workload they lose in FP32 (12: 1.497, 13: 1.465 ms against 1.284 ms for 9)
# and tie in FP64 (14: 2.941 ms against 2.963 ms for 5)
CANDIDATES = ((0, 0), (1, 0), (3, 0), (4, 0), (5, 0), (8, 0), (9, 0), (10, 0), (11, 0), (2, 64), (2, 128))  # (variant, pair-kernel block size)
_cache: dict = {}


def _key(solver) -> tuple:
    import torch

    name = torch.cuda.get_device_name(solver.operators.device)
    k = solver.operators.num_elements
    return (name, solver.config.precision, solver.config.flux, solver.config.limiter, int(math.log2(max(k, 1))))


def autotune(solver, state, *, repeats: int = 3, candidates=CANDIDATES, use_cache: bool = True) -> dict:
    """Pick the fastest stage-kernel shape for `solver` on `state` (any state
    the solver accepts). Returns {"choice": (variant, block), "ms": {...}}."""
    import torch

    key = _key(solver)
    if use_cache and key in _cache:
        variant, block = _cache[key]["choice"]
        solver.set_variant(variant)
        solver.set_block_size(block)
        return _cache[key]
    solver.begin_run(state, math.inf)
    ws, lib = solver._ws, solver._lib
    stream = torch.cuda.current_stream()
    times = {}
    for variant, block in candidates:
        solver.set_variant(variant)
        solver.set_block_size(block)
        ptr = C.byref(solver.native)
        args = (ws.x0.data_ptr(), ws.x1.data_ptr(), ws.stage.data_ptr(), stream.cuda_stream)
        _native.check(lib.cfd_rk3_attempt(ptr, *args))  # warm-up (first launch configures the kernel)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(repeats):
            _native.check(lib.cfd_rk3_attempt(ptr, *args))
        stop.record(stream)
        stop.synchronize()
        times[f"variant{variant}/bs{block}"] = start.elapsed_time(stop) / repeats
    best = min(candidates, key=lambda vb: times[f"variant{vb[0]}/bs{vb[1]}"])
    solver.set_variant(best[0])
    solver.set_block_size(best[1])
    result = {"choice": best, "ms": times}
    _cache[key] = result
    return result


BATCH_CANDIDATES = (("persistent", 9), ("chunks", 3), ("chunks", 8), ("chunks", 9), ("chunks", 0))


def autotune_batch(batch, states, final_time, *, attempts: int = 16, candidates=BATCH_CANDIDATES) -> dict:
    """Pick the faster execution form of a BatchedEulerSolver: the persistent
    launch (its tile shape is fixed per precision) or CUDA-graph chunks of the
    separate launches with one of the tiled shapes. Each candidate advances
    the same states `attempts` attempts from t = 0 (after a warm-up chunk that
    captures its graph); the batch is left set to the fastest.
    Returns {"choice": (form, variant), "ms": {...}}."""
    import torch

    times = {}
    for form, variant in candidates:
        batch.persistent = form == "persistent"
        batch.set_variant(variant)
        batch.begin_run(states, final_time)
        batch.advance(attempts)  # warm-up: captures the chunk's graph
        batch.begin_run(states, final_time)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        batch.advance(attempts)
        stop.record()
        stop.synchronize()
        times[f"{form}/variant{variant}"] = start.elapsed_time(stop)
    best = min(candidates, key=lambda fv: times[f"{fv[0]}/variant{fv[1]}"])
    batch.persistent = best[0] == "persistent"
    batch.set_variant(best[1])
    return {"choice": best, "ms": times}
