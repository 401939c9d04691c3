"""Autotuner for batched renders: times one batch of jobs under candidate engine settings and keeps the
fastest.

Knobs (all of them change how the work is scheduled, none changes what a pixel computes):
  * slots   - path slots in flight (the queue capacity of the job-ring wavefront);
  * batch   - (extend, shade) iterations between two host polls (multiples of 6 replay a CUDA graph);
  * drain   - queued slots below which the register-resident drain kernel finishes the batch
              (1: never drain);
  * layout  - BVH node layout: the binary nodes (64 B) or the 4-wide nodes (128 B).

The choice is cached per workload signature (number of images, pixels, traced samples, triangles), so a
serving process tunes once per kind of batch.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass, field, replace

from .scene import FLAG_WIDE_BVH

DEFAULT_SPACE = {
    "slots": [1 << 20, 1 << 21, 1 << 22],
    "batch": [6, 12],
    "drain": [0, 1],
    "layout": ["binary", "wide"],
}


@dataclass
class Tuned:
    slots: int
    batch: int
    drain: int
    layout: str
    ms: float
    table: list = field(default_factory=list)   # (config dict, ms) of every candidate tried

    def batch_params(self) -> dict:
        return {"slots": self.slots, "batch": self.batch, "drain": self.drain}


_cache: dict = {}


def signature(jobs) -> tuple:
    pixels = sum(j.params.width * j.params.height for j in jobs)
    paths = sum(j.params.width * j.params.height * j.params.traced_spp for j in jobs)
    tris = sum(j.scene.info()["num_primitives"] for j in {id(j.scene): j for j in jobs}.values())
    return (len(jobs), pixels, paths, tris, jobs[0].params.mode, jobs[0].params.draw_order)


def with_layout(jobs, layout: str):
    """The jobs with the BVH layout flag set for `layout` ("binary" or "wide")."""
    out = []
    for j in jobs:
        flags = j.params.flags & ~FLAG_WIDE_BVH
        if layout == "wide":
            flags |= FLAG_WIDE_BVH
        out.append(replace(j, params=replace(j.params, flags=flags)))
    return out


def autotune_batch(ctx, jobs, space: dict | None = None, repeats: int = 2, stream: int | None = None,
                   use_cache: bool = True) -> Tuned:
    """Renders `jobs` (a list of renderer.Job) once per candidate configuration (after one untimed run)
    and returns the fastest.  The jobs' output buffers hold the last candidate's images afterwards."""
    sig = signature(jobs)
    if use_cache and sig in _cache:
        return _cache[sig]
    space = {**DEFAULT_SPACE, **(space or {})}
    table = []
    best = None
    for slots, batch, drain, layout in itertools.product(space["slots"], space["batch"], space["drain"],
                                                         space["layout"]):
        js = with_layout(jobs, layout)
        kw = {"slots": slots, "batch": batch, "drain": drain, "stream": stream}
        ctx.render_batch(js, **kw)          # untimed: engine set-up for this configuration
        times = []
        for _ in range(repeats):
            t = time.perf_counter()
            ctx.render_batch(js, **kw)      # synchronous: returns once every image is complete
            times.append((time.perf_counter() - t) * 1e3)
        ms = min(times)
        cfg = {"slots": slots, "batch": batch, "drain": drain, "layout": layout}
        table.append((cfg, ms))
        if best is None or ms < best[1]:
            best = (cfg, ms)
    tuned = Tuned(**best[0], ms=best[1], table=table)
    _cache[sig] = tuned
    return tuned
