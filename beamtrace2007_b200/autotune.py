"""Autotuner (no counterpart in the reference): picks the engine's launch
settings for a workload by timing a probe of it on the GPU.

Two kinds of setting:

* per context (`bt_gpu_config`): CTAs per SM of the persistent grids
  (`blocks_per_sm`, i.e. warps per SM; 0 = as many as fit), the register
  budget of the full-round trace kernel (`trace_ctas`: 3 or 4 CTAs per
  SM, 0 = by scene size), the queue
  length below which rounds become fused tail rounds (`tail_records`), the
  share of exited trace warps at which the records still in flight are
  handed on to the next round (`yield_pct`), and the sub-beam queue
  capacity -- `tune_engine` builds a context for each candidate and times
  soft-shadow frames;
* per call: the primary-visibility tile (pixels per side of a root) --
  `tune_tile` times `bt_gpu_primary_ids` per candidate on an existing
  context.  Fewer, larger tiles mean less re-traversal and fewer splits at
  tile borders; more, smaller tiles keep the GPU busy on small images.

Results do not depend on the context settings (the engine is deterministic
and exact for any of them); the tile changes which polygons are produced,
so a caller that compares images must use the same tile (the reference's
own is 16).
"""
from __future__ import annotations

import itertools
import time

import numpy as np


def _best(timings: dict):
    return min(timings, key=timings.get)


def tune_engine(scene, cam, light, exact: bool = True, blocks_per_sm=(0, 2), tail_records=(0, 30000, -1),
                capacities=(0,), yield_pcts=(0,), budgets=None, trace_ctas=None, reps: int = 2, device: int = 0):
    """Times `reps` soft-shadow frames (after one warm-up) for every
    combination of the candidate settings; returns (best settings as
    GpuRenderer keyword arguments, {settings tuple: best ms}).  `budgets`:
    candidate live sub-beam budgets per root (a root over it is retried with
    16x; dense meshes under large lights prefer larger ones); `trace_ctas`:
    candidate CTAs per SM of the full-round trace kernel.  Each given one
    adds a field to the settings tuple (budget first); None keeps the
    default and the 4-tuple keys."""
    from .renderer import GpuRenderer
    timings = {}
    for bps, tail, cap, yp, bud, tc in itertools.product(blocks_per_sm, tail_records, capacities, yield_pcts,
                                                         budgets or (None,), trace_ctas or (None,)):
        kw = {} if bud is None else {"budget": bud}
        if tc is not None:
            kw["trace_ctas"] = tc
        with GpuRenderer(scene, device=device, blocks_per_sm=bps, tail_records=tail, capacity=cap,
                         yield_pct=yp, **kw) as g:
            g.soft_shadows(cam, light, exact=exact)
            ms = []
            for _ in range(reps):
                ms.append(g.soft_shadows(cam, light, exact=exact).info["ms_total"])
        key = (bps, tail, cap, yp) + (() if budgets is None else (bud,)) + (() if trace_ctas is None else (tc,))
        timings[key] = min(ms)
    best = _best(timings)
    out = {"blocks_per_sm": best[0], "tail_records": best[1], "capacity": best[2], "yield_pct": best[3]}
    rest = list(best[4:])
    if budgets is not None:
        out["budget"] = rest.pop(0)
    if trace_ctas is not None:
        out["trace_ctas"] = rest.pop(0)
    return out, timings


def tune_tile(renderer, cam, tiles=(8, 16, 32), reps: int = 2):
    """The primary tile that gives the fastest `primary_ids` for this
    camera; returns (tile, {tile: best seconds})."""
    timings = {}
    for tile in tiles:
        renderer.primary_ids(cam, tile=tile)
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            renderer.primary_ids(cam, tile=tile)
            ts.append(time.perf_counter() - t)
        timings[tile] = float(np.min(ts))
    return _best(timings), timings
