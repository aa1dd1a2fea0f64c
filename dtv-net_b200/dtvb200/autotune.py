"""Launch-parameter autotuner for projector plans.

A plan's tuning keys (DTV_TUNE_*) change how its kernels are launched, not
what they compute (beyond FP32 rounding). ``tune`` times each candidate value
of a key on the plan's own geometry with CUDA events, keeps the fastest, and
remembers the choice per (device, geometry, batch, key) for the rest of the
process, so plans created later for the same workload reuse it without timing.

DTV_TUNE_FP_RAY_TILE picks the forward projector's ray tile: which detector
pixels share a block (256 rays of one view) and a warp (32 rays). The samplers
are bound by the texture / L1 pipe, whose throughput depends on how many cache
lines the 32 samples of one warp instruction touch, and that depends on the
tile and on the geometry (magnification, pixel pitch, volume aspect).

DTV_TUNE_FP_TEX_SHARE applies to "tma" plans: of every 8 ray tiles, that
many sample through the texture unit and the rest from shared memory, so the
texture pipe and the shared-memory/FMA pipes work side by side.

DTV_TUNE_ADJOINT applies to plans with adjoint tables: the exact adjoint
scatters either per 16^3 brick through shared-memory atomics (0) or into
per-cell records with 16-byte vector atomics in L2 (1); which is faster
depends on whether the records fit in L2. It is timed on plan.adjoint.

DTV_TUNE_FP_BAND picks the forward projector's block order: view by view (0),
or bands of B tile rows with every view of a band before the next band, which
keeps the volume slab under a band in L2 across views when the staged volume
is larger than L2.

DTV_TUNE_BP_WARP picks the backprojector's columns per warp (16 x 2, 8 x 4 or
4 x 8). It is timed on plan.backward.
"""
from __future__ import annotations

import torch

from . import _lib
from .geometry import Plan

_CACHE: dict = {}
N_RAY_TILES = 8
CANDIDATES = {_lib.DTV_TUNE_FP_RAY_TILE: range(N_RAY_TILES), _lib.DTV_TUNE_FP_TEX_SHARE: range(9),
              _lib.DTV_TUNE_ADJOINT: range(2), _lib.DTV_TUNE_FP_BAND: (0, 1, 2, 4, 8, 16, 32),
              _lib.DTV_TUNE_BP_WARP: range(5)}


def _key(plan: Plan, batch: int, key: int):
    return (torch.cuda.get_device_name(plan.device), plan.sampler, int(batch),
            plan.geometry.key(), int(key))


def _median_ms(plan: Plan, fn, reps: int, warmup: int) -> float:
    with torch.cuda.device(plan.device):
        for _ in range(warmup):
            fn()
        times = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def time_forward(plan: Plan, vol: torch.Tensor, out: torch.Tensor, reps: int = 5,
                 warmup: int = 2) -> float:
    """Median milliseconds of ``plan.forward(vol, out)`` on the current stream."""
    return _median_ms(plan, lambda: plan.forward(vol, out), reps, warmup)


def tune(plan: Plan, batch: int = 1, key: int = None, candidates=None,
         reps: int = 5, warmup: int = 2, use_cache: bool = True) -> dict:
    """Time ``candidates`` for ``key`` on ``plan`` and set the fastest.

    ``key`` defaults to the key that applies to the plan's sampler
    (DTV_TUNE_FP_TEX_SHARE for "tma", DTV_TUNE_FP_RAY_TILE otherwise).
    Returns {value: milliseconds}. A cached choice is applied without
    timing."""
    if key is None:
        key = _lib.DTV_TUNE_FP_TEX_SHARE if plan.sampler == "tma" else _lib.DTV_TUNE_FP_RAY_TILE
    if key not in CANDIDATES:
        raise ValueError(f"unknown tuning key {key}")
    ck = _key(plan, batch, key)
    if use_cache and ck in _CACHE:
        plan.set_tuning(key, _CACHE[ck][0])
        return dict(_CACHE[ck][1])
    if candidates is None:
        candidates = CANDIDATES[key]
    gen = torch.Generator(device=plan.device).manual_seed(0)
    vol = torch.rand(plan.vol_shape(batch), device=plan.device, generator=gen)
    sino = torch.rand(plan.sino_shape(batch), device=plan.device, generator=gen)
    if key == _lib.DTV_TUNE_ADJOINT:
        fn = lambda: plan.adjoint(sino, vol)  # noqa: E731
    elif key == _lib.DTV_TUNE_BP_WARP:
        fn = lambda: plan.backward(sino, vol)  # noqa: E731
    else:
        fn = lambda: plan.forward(vol, sino)  # noqa: E731
    times = {}
    for c in candidates:
        plan.set_tuning(key, int(c))
        times[int(c)] = _median_ms(plan, fn, reps, warmup)
    best = min(times, key=times.get)
    plan.set_tuning(key, best)
    _CACHE[ck] = (best, dict(times))
    return times


def clear_cache() -> None:
    _CACHE.clear()
