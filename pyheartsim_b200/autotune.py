"""Autotuner of the step kernel.

Times every compiled step-kernel variant (register budget) at every feasible
CTAs-per-SM setting on the engine's live instances, keeps the fastest and
leaves the engine configured with it.  Tuning advances the instances like any
other call (the steps are real work).  Results are cached per GPU name and
workload bucket (total voxels rounded to a power of two, instance count) for
the lifetime of the process.
"""
import math

import torch

from . import _lib
from .engine import step_variants

_CACHE = {}


def _bucket(engine):
    n = sum(engine.instance(s).n_voxel for s in engine.slots())
    return (torch.cuda.get_device_name(), engine.precision, 1 << max(0, int(math.log2(max(n, 1)))),
            len(engine.slots()))


def tune(engine, steps=10, stream=None, cps_options=None):
    """Pick (variant, ctas_per_sm) for ``engine``; returns the timing table."""
    key = _bucket(engine)
    if key in _CACHE:
        best = _CACHE[key]
        engine.configure(variant=best[0], ctas_per_sm=best[1])
        return {"cached": True, "best": best}
    stream = stream or torch.cuda.current_stream()
    table = []
    for variant, minb, regs in step_variants(engine.precision):
        options = cps_options or sorted({minb, max(1, minb - 1), minb + 1})
        for cps in options:
            engine.configure(variant=variant, ctas_per_sm=cps)
            try:
                engine.advance(steps, stream=stream, sync=True)      # plan + graph capture, warm
            except _lib.PhsError:
                continue
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            engine.advance(steps, stream=stream, sync=False)
            e1.record(stream)
            torch.cuda.synchronize()
            table.append({"variant": variant, "min_ctas": minb, "regs": regs, "ctas_per_sm": cps,
                          "ms_per_step": e0.elapsed_time(e1) / steps})
    best = min(table, key=lambda r: r["ms_per_step"])
    _CACHE[key] = (best["variant"], best["ctas_per_sm"])
    engine.configure(variant=best["variant"], ctas_per_sm=best["ctas_per_sm"])
    return {"cached": False, "best": (best["variant"], best["ctas_per_sm"]), "table": table}
