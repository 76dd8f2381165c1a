"""Autotuner for the batched-ensemble kernel.

The tunables are the launch shape and the schedule of the persistent kernel:
warps (systems in flight) per block, the unroll factor of the inner pair loop,
and the order in which warps take systems (largest first, or upload order).
Packing several small systems into one warp is not a tunable: at the C4 size
distribution (n uniform in 3..64) systems of 16 or fewer bodies carry under
2% of the pair work, so it could win at most that. Each candidate
is timed on the caller's own ensemble (the real size distribution) for a short
run with CUDA events inside the library, after one untimed warm-up run, and
the three fastest are timed again for four times as long (neighbouring shapes
differ by about the short runs' own spread); the state is saved before and
restored after, so tuning leaves the ensemble untouched. Results are cached in a JSON file keyed by the name of the
context's GPU, precision, integrator, force law and a histogram of the system
sizes, so later runs of the same configuration skip the search.
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

from .api import MIXED, YOSHIDA4, Context, Params

DEFAULT_SPACE = {"warps_per_block": (1, 2, 4, 8), "unroll": (1, 2, 4), "schedule": (0, 1)}
DEFAULT_CACHE = Path(os.environ.get("ASTER_TUNE_CACHE", Path.home() / ".cache" / "aster_b200" / "ensemble.json"))


def _gpu_name(device: int) -> str:
    """Name of CUDA device `device` (the context's, in CUDA's numbering)."""
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda{device}"


def _key(ctx: Context, offsets, precision, integrator, force_law) -> str:
    sizes = np.diff(np.asarray(offsets, dtype=np.int64))
    hist = np.bincount(sizes, minlength=65)[:65]
    h = hashlib.sha1(hist.tobytes()).hexdigest()[:16]
    return f"{_gpu_name(getattr(ctx, 'device', 0))}|p{precision}|i{integrator}|f{force_law}|n{len(sizes)}|h{h}"


def tune_ensemble(ctx: Context, offsets, p: Params, integrator: int = YOSHIDA4, precision: int = MIXED,
                  steps: int = 40, space: dict | None = None, cache: Path | str | None = DEFAULT_CACHE,
                  force: bool = False, refine: int = 3) -> dict:
    """Return the fastest config for the ensemble currently uploaded to ctx
    (offsets must be the ones uploaded). Every candidate runs `steps` steps;
    the `refine` fastest run again for 4 x `steps`, and the best of those
    wins. Adds "ms_per_step" (and "ms_per_step_long") and "timings"."""
    space = space or DEFAULT_SPACE
    key = _key(ctx, offsets, precision, integrator, p.force_law)
    cache = Path(cache) if cache else None
    if cache and cache.exists() and not force:
        table = json.loads(cache.read_text())
        if key in table:
            return table[key]
    pos0, vel0 = ctx.ensemble_download()
    mass = None
    timings = []
    try:
        for wpb in space["warps_per_block"]:
            for unroll in space["unroll"]:
                for schedule in space.get("schedule", (0,)):
                    cfg = {"warps_per_block": wpb, "unroll": unroll, "check_every": 256, "use_graph": 1,
                           "schedule": schedule}
                    ctx.ensemble_run(p, max(2, steps // 8), integrator, precision, cfg)   # warm-up
                    ctx.ensemble_run(p, steps, integrator, precision, cfg)
                    ms = ctx.stats()["ms_total"] / steps
                    timings.append({**cfg, "ms_per_step": ms})
        # the short runs differ by a few percent between neighbouring shapes, about
        # their own run-to-run spread: time the leading candidates again, longer
        timings.sort(key=lambda t: t["ms_per_step"])
        for t in timings[:refine]:
            cfg = {k: t[k] for k in ("warps_per_block", "unroll", "check_every", "use_graph", "schedule")}
            ctx.ensemble_run(p, steps * 4, integrator, precision, cfg)
            t["ms_per_step_long"] = ctx.stats()["ms_total"] / (steps * 4)
    finally:
        # restore the caller's state (masses are unchanged by a run)
        mass = _masses_of(ctx)
        ctx.ensemble_upload(offsets, pos0, vel0, mass)
    ranked = [t for t in timings if "ms_per_step_long" in t] or timings
    best = min(ranked, key=lambda t: t.get("ms_per_step_long", t["ms_per_step"]))
    result = {**best, "timings": timings, "key": key}
    if cache:
        cache.parent.mkdir(parents=True, exist_ok=True)
        table = json.loads(cache.read_text()) if cache.exists() else {}
        table[key] = result
        cache.write_text(json.dumps(table, indent=1))
    return result


def _masses_of(ctx: Context):
    m = getattr(ctx, "_ens_mass", None)
    if m is None:
        raise RuntimeError("upload the ensemble with Context.ensemble_upload before tuning")
    return m
