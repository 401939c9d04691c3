"""Autotuner for batched renders: times one batch of jobs under candidate engine settings and keeps the
fastest.

Knobs (all of them change how the work is scheduled, none changes what a pixel computes):
  * slots   - path slots in flight (the queue capacity of the job-ring wavefront);
  * batch   - (extend, shade) iterations between two host polls (multiples of 6 replay a CUDA graph);
  * drain   - queued slots below which the register-resident drain kernel finishes the batch
              (1: never drain);
  * layout  - BVH node layout: the binary nodes (64 B) or the 8-wide nodes with quantised child
              boxes (96 B);
  * block   - threads per block of the extend and shade kernels (128, 256 or 512).

Search: coordinate descent by default - each knob in turn is swept with the others held at the best
configuration so far, until a pass over all knobs changes nothing (at most `passes` passes); every
configuration is timed once however often the search meets it.  `search="grid"` times every
combination instead.

The choice is cached per workload signature (number of images, pixels, traced samples, triangles), so a
serving process tunes once per kind of batch.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass, field, replace

from .scene import FLAG_WIDE_BVH

DEFAULT_SPACE = {
    "layout": ["binary", "wide"],
    "slots": [1 << 20, 1 << 21, 1 << 22],
    "batch": [6, 12],
    "drain": [0, 1],
    "block": [128, 256, 512],
}
DEFAULT_START = {"layout": "binary", "slots": 1 << 22, "batch": 12, "drain": 0, "block": 128}


@dataclass
class Tuned:
    slots: int
    batch: int
    drain: int
    layout: str
    block: int
    ms: float
    table: list = field(default_factory=list)   # (config dict, ms) of every candidate tried

    def batch_params(self) -> dict:
        return {"slots": self.slots, "batch": self.batch, "drain": self.drain, "block": self.block}


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
                   use_cache: bool = True, search: str = "descent", passes: int = 2,
                   start: dict | None = None) -> Tuned:
    """Renders `jobs` (a list of renderer.Job) under candidate configurations (each after one untimed
    run) and returns the fastest.  The jobs' output buffers hold the last candidate's images afterwards."""
    sig = signature(jobs)
    if use_cache and sig in _cache:
        return _cache[sig]
    space = {**DEFAULT_SPACE, **(space or {})}
    knobs = list(space)
    timed: dict = {}

    def measure(cfg: dict) -> float:
        key = tuple(cfg[k] for k in knobs)
        if key not in timed:
            js = with_layout(jobs, cfg["layout"])
            kw = {"slots": cfg["slots"], "batch": cfg["batch"], "drain": cfg["drain"], "block": cfg["block"],
                  "stream": stream}
            ctx.render_batch(js, **kw)          # untimed: engine set-up for this configuration
            times = []
            for _ in range(repeats):
                t = time.perf_counter()
                ctx.render_batch(js, **kw)      # synchronous: returns once every image is complete
                times.append((time.perf_counter() - t) * 1e3)
            timed[key] = min(times)
        return timed[key]

    if search == "grid":
        for combo in itertools.product(*(space[k] for k in knobs)):
            measure(dict(zip(knobs, combo)))
    elif search == "descent":
        best = {k: (start or DEFAULT_START).get(k, space[k][0]) for k in knobs}
        best_ms = measure(best)
        for _ in range(passes):
            changed = False
            for k in knobs:
                for v in space[k]:
                    cand = {**best, k: v}
                    ms = measure(cand)
                    if ms < best_ms:
                        best, best_ms, changed = cand, ms, True
            if not changed:
                break
    else:
        raise ValueError(f"unknown search {search!r}")
    table = [(dict(zip(knobs, key)), ms) for key, ms in timed.items()]
    cfg, ms = min(table, key=lambda x: x[1])
    tuned = Tuned(slots=cfg["slots"], batch=cfg["batch"], drain=cfg["drain"], layout=cfg["layout"],
                  block=cfg["block"], ms=ms, table=table)
    _cache[sig] = tuned
    return tuned
