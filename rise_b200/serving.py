"""Progressive render serving with continuous batching.

Requests arrive over time (a Poisson process); each names a resident scene
and asks for a progressive image at a ladder of sample counts (e.g. 16, then
64, then 256 spp).  `serve(mode="continuous")` admits a request as soon as
device memory for its film fits the budget, submits its next level to one
shared engine while other requests are in flight, and reports when each
level is complete; `serve(mode="fifo")` is the plain path: one request at a
time, level after level, on the same engine and kernels.

Latency of a level = wall time from the request's arrival until all samples
of that level are in its film.  The scenes (BVHs, materials) stay resident;
per request the device holds only its film and, while submitted, its slot
in the engine's job table.
"""
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .pathtracer import Engine, SpectralRasterizer


@dataclass
class Request:
    rid: int
    arrival: float
    scene: int                 # index into the resident scene pool
    settings: object           # scenes.RenderSettings
    levels: tuple = (16, 64, 256)
    done_at: list = field(default_factory=list)   # seconds after arrival per level
    job: object = None
    level: int = 0


def poisson_arrivals(rate, duration, seed):
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def serve(ctx, pool, requests, mode="continuous", capacity=1 << 21, step_iters=2, use_graph=True,
          timeout=600.0, max_active=None, max_followup=None):
    """Run `requests` (list of Request, arrival-ordered) against `pool`
    (list of (SceneDesc, committed raycaster.Scene)).  Returns a summary
    dict with per-level latency percentiles and aggregate throughput.
    max_active caps the requests in flight in continuous mode (admission
    waits for a slot; None: only the memory budget limits them).
    max_followup caps, in continuous mode, the requests whose later levels
    (after the first) are in flight at once: first levels always start as
    they arrive, the others wait their turn in order of arrival, so an
    overloaded server keeps fast first previews without interleaving every
    resident scene's paths."""
    eng = Engine(ctx, capacity)
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    later = deque()          # requests whose next level waits for a follow-up slot
    active = []
    finished = []
    samples = 0
    t0 = time.perf_counter()
    try:
        while pending or active or later:
            now = time.perf_counter() - t0
            if now > timeout:
                raise RuntimeError("serving run exceeded its time limit")
            # Admission: arrived requests whose film fits the memory budget.
            limit = 1 if mode == "fifo" else max_active
            inflight = len(active) + len(later)
            while pending and pending[0].arrival <= now and (limit is None or inflight < limit):
                r = pending[0]
                desc, scene = pool[r.scene]
                try:
                    r.job = SpectralRasterizer(ctx, desc, scene=scene, settings=r.settings)
                except _native.RTB200Error as e:
                    if e.code == _native.E_BUDGET:
                        break
                    raise
                pending.popleft()
                eng.submit(r.job, r.levels[0])
                active.append(r)
                inflight += 1
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                continue
            eng.step(step_iters, use_graph)
            now = time.perf_counter() - t0
            for r in list(active):
                done, total = eng.progress(r.job)
                if done < total:
                    continue
                eng.retire(r.job)
                samples += total
                r.done_at.append(now - r.arrival)
                r.level += 1
                active.remove(r)
                if r.level < len(r.levels):
                    later.append(r)
                else:
                    r.job.close()
                    r.job = None
                    finished.append(r)
            # Next levels, within the follow-up cap.
            while later and (mode == "fifo" or max_followup is None or
                             sum(1 for a in active if a.level > 0) < max(1, max_followup)):
                r = later.popleft()
                eng.submit(r.job, r.levels[r.level] - r.levels[r.level - 1])
                active.append(r)
        wall = time.perf_counter() - t0
    finally:
        eng.close()   # detaches any job still submitted
        for r in list(active) + list(later):
            if r.job is not None:
                r.job.close()
                r.job = None
    lat = {}
    for k in range(len(requests[0].levels) if requests else 0):
        v = np.array([r.done_at[k] for r in finished if len(r.done_at) > k])
        lvl = requests[0].levels[k]
        if len(v):
            lat[str(lvl)] = {"p50_s": float(np.percentile(v, 50)), "p99_s": float(np.percentile(v, 99)),
                             "mean_s": float(v.mean())}
    return {"mode": mode, "requests": len(finished), "wall_s": wall, "msamples_s": samples / wall / 1e6,
            "max_active": max_active if mode == "continuous" else 1,
            "max_followup": max_followup if mode == "continuous" else None, "latency": lat}
