"""Autotuner for the wavefront engine.

Two knobs decide how a batch of render jobs maps onto the device: the path
pool capacity (how many paths are in flight, i.e. the queue sizes) and the
number of wavefront iterations between host progress polls
(`rtb200_engine_set_poll`).  A larger pool keeps more rays in flight per
launch but makes each iteration's tail longer; fewer polls save host round
trips but let a finished batch run a few empty iterations.  `tune` renders a
sample of the real job mix under every combination and keeps the fastest;
results are cached per GPU model and workload signature in
rise_b200/_lib/autotune.json, so a service tunes once per device type.

The staging depth of the BVH's top levels in shared memory, the other knob
one could tune, measured slower than no staging at every depth tried on B200
(top nodes stay L1-resident), so the kernels do not stage.
"""
import hashlib
import json
import os
import time
from dataclasses import dataclass

from .pathtracer import Engine, SpectralRasterizer

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "autotune.json")
CAPACITIES = (1 << 18, 1 << 19, 1 << 20, 1 << 21)
POLLS = (2, 4, 8, 16)


@dataclass
class Config:
    capacity: int
    poll: int
    msamples_s: float


def _gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:   # noqa: BLE001 - any failure just means "unknown device"
        return "unknown"


def signature(descs, spp):
    """A stable key for a job mix: resolutions, triangle counts, depths, spp."""
    h = hashlib.sha1()
    for d, s in zip(descs, spp):
        st = d.settings
        lim = (st.max_diffuse_bounce, st.max_glossy_bounce, st.max_transmission_bounce)
        h.update(f"{st.width}x{st.height}:{d.n_tri}:{st.max_depth}:{lim}:{st.nee_per_lambda}:{s};".encode())
    return h.hexdigest()[:16]


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache):
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    tmp = CACHE + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1)
    os.replace(tmp, CACHE)


def tune(ctx, descs, scenes, spp, capacities=CAPACITIES, polls=POLLS, use_graph=True, use_cache=True):
    """Pick (capacity, poll) for rendering jobs `descs` (on committed `scenes`)
    with `spp` samples per pixel each, by timing every combination on that
    mix.  Returns (best Config, list of all Configs tried)."""
    key = f"{_gpu_name()}|{signature(descs, spp)}"
    cache = _load() if use_cache else {}
    if key in cache:
        c = cache[key]
        return Config(c["capacity"], c["poll"], c["msamples_s"]), []
    samples = sum(d.settings.width * d.settings.height * s for d, s in zip(descs, spp))
    tried = []
    for cap in capacities:
        eng = Engine(ctx, cap)
        try:
            warm = SpectralRasterizer(ctx, descs[0], scene=scenes[0])
            eng.render([warm], [1], use_graph=use_graph)
            warm.close()
            for poll in polls:
                eng.set_poll(poll)
                jobs = [SpectralRasterizer(ctx, d, scene=s) for d, s in zip(descs, scenes)]
                try:
                    t0 = time.perf_counter()
                    eng.render(jobs, spp, use_graph=use_graph)
                    dt = time.perf_counter() - t0
                finally:
                    for j in jobs:
                        j.close()
                tried.append(Config(cap, poll, samples / dt / 1e6))
        finally:
            eng.close()
    best = max(tried, key=lambda c: c.msamples_s)
    if use_cache:
        cache[key] = {"capacity": best.capacity, "poll": best.poll, "msamples_s": best.msamples_s}
        _store(cache)
    return best, tried
