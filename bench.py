"""Benchmark: batched BVH ray casting on one B200 (or N replicas).

Workload (one "step"): one pass of 4,194,304 closest-hit rays over a
1,000,000-triangle soup (centroids uniform in the unit cube, vertices offset
by N(0, 0.01^2); rays from a radius-2 sphere towards uniform targets in the
cube; seed 7), through the reference's BVH (SAH 32 bins, leaf 4, collapsed to
4-wide nodes) with FP16-quantised child boxes (binary16 rounded outward,
the configuration's quantised format; the FP32-node and 8-bit-node layouts
are reported as variants; all return the same hits).  Metric: Mrays/s.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank holds the scene and casts its own 4,194,304 rays
(weak scaling, no collective on the data path).  `--impl reference` times
the reference renderer's own CPU BVH (oracle/_ref, or the oracle port where
the reference was not built) on the host cores instead.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TRI = 1_000_000
N_RAYS = 4_194_304
SEED = 7
BYTES_CLOSEST = 48  # ray in 32 B + hit out 16 B
BYTES_ANY = 33      # ray in 32 B + occlusion flag 1 B
WORKLOAD = ("raycast microbench: 1,000,000-triangle soup, 4,194,304 rays from a radius-2 sphere, "
            "closest-hit, reference BVH (SAH 32 bins, leaf 4) collapsed to 4-wide nodes with FP16-quantised "
            "child boxes (binary16, rounded outward)")
METRIC = "Mrays/s"
# The reference arm runs the reference's own BVH, whose child boxes are FP32
# (it has no quantised node format).
REF_WORKLOAD = ("raycast microbench: 1,000,000-triangle soup, 4,194,304 rays from a radius-2 sphere, "
                "closest-hit, the reference's own BVH (SAH 32 bins, leaf 4, FP32 child boxes) and "
                "double-precision ray/triangle test on the host cores")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="rtb200", choices=["rtb200", "reference"])
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-path-tracer", action="store_true")
    p.add_argument("--no-large", action="store_true", help="skip the 3.4M-triangle scene")
    p.add_argument("--no-batch", action="store_true", help="skip the 48-scene batch and the serving run")
    p.add_argument("--pt-only", action="store_true",
                   help="run only the path-tracer measurement and print its JSON (for profiling)")
    p.add_argument("--large-only", action="store_true",
                   help="run only the large-scene path-tracer measurement and print its JSON (for profiling)")
    p.add_argument("--serving-full", action="store_true",
                   help="run only the serving configuration at full size (20 req/s for 60 s over the whole "
                        "batched-scenes distribution, 120 GB device budget; many minutes) and print its JSON")
    p.add_argument("--serving-skip", default="", help="--serving-full: comma list of arms to leave out (continuous, fifo)")
    return p.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled(name, key):
    """A figure of the committed ncu capture of a kernel (its summary under
    profiles/ holds `key: value` lines), or None."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(re.escape(key) + r":\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clock / throttle sampling around a timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_time(tri, rays, seconds=12.0, threads=None):
    """Time the reference CPU BVH (oracle/_ref, else the oracle port) on host
    cores over a bounded sample of the rays.  Returns (Mrays/s, kind, cores, n)."""
    import oracle
    kind = "reference" if oracle.ref() is not None else "port"
    threads = threads or os.cpu_count()
    b = oracle.BVH(tri, "ref" if kind == "reference" else "port")
    probe = rays[:32768]
    t0 = time.perf_counter()
    b.closest(probe, threads=threads)
    rate = len(probe) / max(time.perf_counter() - t0, 1e-6)
    n = int(min(len(rays), max(65536, rate * seconds)))
    t0 = time.perf_counter()
    b.closest(rays[:n], threads=threads)
    dt = time.perf_counter() - t0
    return n / dt / 1e6, kind, threads, n


C1_SCENE = os.path.join(ROOT, "tests", "golden", "cornell_c1.RISEscene")
C1_REF = os.path.join(ROOT, "tests", "golden", "cornell_c1_ref_fp64.npz")
C1_CHECKPOINTS = (16, 64, 256, 512, 1024, 2048)


def relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def convergence(ctx, desc, ref, settings, checkpoints=C1_CHECKPOINTS, crop=None):
    """relMSE against `ref` at each checkpoint spp of one progressive render,
    device seconds at each, and the first checkpoint at relMSE <= 1e-3 with
    its Msamples/s (samples to that point / device seconds to that point)."""
    from rise_b200 import pathtracer
    r = pathtracer.SpectralRasterizer(ctx, desc, settings=settings)
    rel, secs, done = {}, {}, 0
    x0, y0, x1, y1 = crop or (0, 0, settings.width, settings.height)
    for target in checkpoints:
        r.rasterize_scene(target - done)
        done = target
        rel[str(target)] = relmse(r.film()[y0:y1, x0:x1].astype(np.float64), ref)
        secs[str(target)] = r.stats()["seconds"]
    r.close()
    out = {"relmse": rel, "device_seconds": secs}
    reach = [int(k) for k, v in rel.items() if v <= 1e-3]
    if reach:
        k = min(reach)
        out["spp_to_relmse_1e-3"] = k
        out["device_seconds_to_relmse_1e-3"] = secs[str(k)]
        out["msamples_s_at_relmse_1e-3"] = settings.width * settings.height * k / secs[str(k)] / 1e6
    return out


def bench_path_tracer(ctx, rank, cpu_baseline=True):
    """C1 spectral Cornell box, read from its scene file in the reference's
    scene language (tests/golden/cornell_c1.RISEscene: 32 triangles,
    256x256, 16 spp, HWSS 4 wavelengths, at most 7 diffuse bounces, Russian
    roulette from depth 3; Owen-scrambled Sobol with the index shuffled per
    dimension pair).  Device throughput in Msamples/s (the three samplers,
    per-wavelength and shared NEE, 8-bit nodes); relMSE at 16 .. 2048 spp
    against the reference renderer's 16384-spp FP64 image (its integrator
    given independent numbers) with the spp, device time and Msamples/s at
    relMSE <= 1e-3 per sampler; and the reference renderer itself
    (Job::Rasterize, oracle/_ref) timed on the host cores."""
    import dataclasses
    from rise_b200 import pathtracer, scenefile
    ls = scenefile.load_scene(C1_SCENE)
    desc, base = ls.desc, ls.desc.settings
    out = {"workload": "C1 spectral Cornell box from its .RISEscene: 32 triangles, 256x256, 16 spp, HWSS 4 "
                       "wavelengths, at most 7 diffuse bounces (8 vertices), RR from depth 3, Sobol sampler "
                       "(index shuffled per dimension pair)"}
    scene = pathtracer.upload_scene(ctx, desc)
    npix = base.width * base.height

    def throughput(st, dev_scene):
        r = pathtracer.SpectralRasterizer(ctx, desc, scene=dev_scene, settings=st)
        r.rasterize_scene(16)   # warm-up pass
        t0 = r.stats()["seconds"]
        reps = 4
        for _ in range(reps):
            r.rasterize_scene(16)
        stt = r.stats()
        dt = (stt["seconds"] - t0) / reps
        r.close()
        return {"msamples_s": npix * 16 / dt / 1e6, "ms_per_16spp": dt * 1e3,
                "segments_per_sample": stt["segments"] / stt["samples"],
                "shadow_rays_per_sample": stt["shadow_rays"] / stt["samples"]}

    out["nee_per_wavelength"] = throughput(base, scene)
    out["nee_per_wavelength_hash_sampler"] = throughput(dataclasses.replace(base, sampler=0), scene)
    out["nee_per_wavelength_reference_sobol"] = throughput(dataclasses.replace(base, sampler=1), scene)
    out["nee_shared"] = throughput(dataclasses.replace(base, nee_per_lambda=0), scene)
    sq = pathtracer.upload_scene(ctx, desc, "q8")
    out["q8_nodes_msamples_s"] = throughput(base, sq)["msamples_s"]
    sq.close()
    if os.path.exists(C1_REF):
        ref = np.load(C1_REF)["xyz"].astype(np.float64)
        # Sobol as the reference pads it (a pixel stops converging at a
        # relMSE near 2e-3), with the index shuffled per dimension pair, and
        # the counter-based hash.
        out["vs_reference_fp64_16384spp"] = {
            "sobol_shuffled": convergence(ctx, desc, ref, dataclasses.replace(base, seed=7, sampler=2)),
            "sobol_reference": convergence(ctx, desc, ref, dataclasses.replace(base, seed=7, sampler=1)),
            "hash": convergence(ctx, desc, ref, dataclasses.replace(base, seed=7, sampler=0))}
    if cpu_baseline and rank == 0:
        import oracle
        if oracle.rise_ref() is not None:
            # The reference renderer's own pipeline on every host core.
            rr = oracle.RefRenderer(C1_SCENE)
            rr.render()   # scene preparation and first-touch outside the timing
            t0 = time.perf_counter()
            reps = 2
            for _ in range(reps):
                rr.render()
            dt = (time.perf_counter() - t0) / reps
            rr.close()
            out["cpu_baseline"] = {"value": npix * 16 / dt / 1e6, "unit": "Msamples/s",
                                   "cores": oracle.RISE_THREADS, "kind": "reference",
                                   "sample": "the whole 256x256 image at 16 spp through the reference's "
                                             "Job::Rasterize, twice"}
        else:
            oracle.pt_render(desc, 1, crop=(0, 0, 8, 8))   # one-time table setup outside the timing
            t0 = time.perf_counter()
            oracle.pt_render(desc, 16, crop=(0, 96, 256, 160))
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": 256 * 64 * 16 / dt / 1e6, "unit": "Msamples/s",
                                   "cores": os.cpu_count(), "kind": "port",
                                   "sample": "rows 96-159 of the 256x256 image, 16 spp"}
    scene.close()
    return out


def bench_large_scene(ctx, layout="f16"):
    """Large scene: 1024x1024 fBm heightfield (2,093,058 triangles) + 64 spheres
    of 20,000 triangles (half GGX conductors, half glass), area light and sky;
    1024x1024 pixels, 64 spp, 4 wavelengths, max depth 16 (15 bounces of each
    type under a 128-vertex cap, as the reference reads it).  relMSE at 64, 256
    and 1024 spp (shuffled Sobol sampler) over the 128x128 image centre
    against the reference renderer's 4096-spp render of that crop
    (tests/golden/spheres_crop_ref_4096.npz, independent numbers).  Rendered
    over binary16 child boxes, with FP32 and 8-bit boxes timed beside them
    (the same hits, so the same image)."""
    from rise_b200 import pathtracer, scenes
    desc = scenes.spheres_scene()
    t0 = time.perf_counter()
    scene = pathtracer.upload_scene(ctx, desc, layout)
    setup = time.perf_counter() - t0
    info = scene.info()
    r = pathtracer.SpectralRasterizer(ctx, desc, scene=scene)
    r.rasterize_scene(4)      # warm-up
    s0 = r.stats()
    r.rasterize_scene(64)
    s1 = r.stats()
    dt = s1["seconds"] - s0["seconds"]
    n = (s1["samples"] - s0["samples"])
    out = {"workload": "1024^2 fBm heightfield + 64 x 20k-triangle spheres (GGX / glass), area light + sky, "
                       "1024x1024, 64 spp, HWSS 4 wavelengths, max depth 16 (15 bounces of each type, "
                       "as the reference reads it)",
           "n_tri": info["n_tri"], "layout": layout, "bvh_build_and_upload_s": round(setup, 3),
           "msamples_s": n / dt / 1e6, "seconds_64spp": dt,
           "segments_per_sample": (s1["segments"] - s0["segments"]) / n,
           "shadow_rays_per_sample": (s1["shadow_rays"] - s0["shadow_rays"]) / n,
           "mrays_s": ((s1["segments"] - s0["segments"]) + (s1["shadow_rays"] - s0["shadow_rays"])) / dt / 1e6}
    r.close()
    ref_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "spheres_crop_ref_4096.npz")
    if os.path.exists(ref_path):
        z = np.load(ref_path)
        ref = z["xyz"].astype(np.float64)
        x0, y0, x1, y1 = (int(v) for v in z["crop"])
        st = scenes.RenderSettings(**{**desc.settings.__dict__, "sampler": scenes.SAMPLER_SOBOL_SHUFFLED, "seed": 7})
        r = pathtracer.SpectralRasterizer(ctx, desc, scene=scene, settings=st)
        rel, done = {}, 0
        for target in (64, 256, 1024):
            r.rasterize_scene(target - done)
            done = target
            img = r.film()[y0:y1, x0:x1].astype(np.float64)
            rel[str(target)] = float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))
        r.close()
        out["relmse_vs_reference_crop"] = {"crop": [x0, y0, x1, y1], "reference_spp": int(z["spp"]),
                                           "sampler": "sobol_shuffled", **rel}
    scene.close()
    # The same render over the other node layouts: FP32 child boxes (plain)
    # and 8-bit quantised ones (64-byte nodes); every layout gives the same
    # hits, so the same image.
    for lay in ("f32", "q8", "f16"):
        if lay != layout:
            q = pathtracer.upload_scene(ctx, desc, lay)
            r = pathtracer.SpectralRasterizer(ctx, desc, scene=q)
            r.rasterize_scene(4)
            s0 = r.stats()
            r.rasterize_scene(64)
            s1 = r.stats()
            out[lay + "_nodes_msamples_s"] = (s1["samples"] - s0["samples"]) / (s1["seconds"] - s0["seconds"]) / 1e6
            r.close()
            q.close()
    return out


def bench_batch(ctx):
    """48 uneven scenes (heightfield + 16 spheres; triangles log-uniform
    10k-1M, resolutions 128^2..1024^2, spp log-uniform 4-256, max depth
    8-16): one shared engine replaying a captured CUDA graph, with pool
    capacity and poll interval from the autotuner (tuned on every 4th scene
    at 1/8 of its spp), against the same jobs rendered one scene at a time on
    the same engine and kernels, and against the plain path (rtb200_job_render
    per scene: its own default-sized engine, no graph)."""
    from rise_b200 import autotune, pathtracer, scenes
    params = scenes.batch_scene_params()
    t0 = time.perf_counter()
    descs = [scenes.batch_scene(p) for p in params]
    devs = [pathtracer.upload_scene(ctx, d, "q8") for d in descs]
    setup = time.perf_counter() - t0
    spp = [p["spp"] for p in params]
    total = sum(p["res"] ** 2 * p["spp"] for p in params)
    t0 = time.perf_counter()
    best, tried = autotune.tune(ctx, descs[::4], devs[::4], [max(1, s // 8) for s in spp[::4]], use_cache=False)
    tune_s = time.perf_counter() - t0
    eng = pathtracer.Engine(ctx, best.capacity)
    eng.set_poll(best.poll)
    out = {"workload": "48 scenes, triangles log-uniform 10k-1M, resolutions {128,256,512,1024}^2, "
                       "spp log-uniform 4-256, max depth 8-16, BVHs with 8-bit quantised child boxes",
           "samples": total,
           "triangles": int(sum(p["n_tri"] for p in params)), "scene_setup_s": round(setup, 2),
           "autotune": {"capacity": best.capacity, "poll": best.poll, "seconds": round(tune_s, 2),
                        "tried": [[c.capacity, c.poll, round(c.msamples_s, 1)] for c in tried]}}
    try:
        # Warm-up (kernels, graph capture) on a small job.
        w = pathtracer.SpectralRasterizer(ctx, descs[0], scene=devs[0])
        eng.render([w], [1])
        w.close()
        one = [pathtracer.SpectralRasterizer(ctx, d, scene=s) for d, s in zip(descs, devs)]
        per_scene = []
        t0 = time.perf_counter()
        for r, s in zip(one, spp):
            t1 = time.perf_counter()
            eng.render([r], [s], use_graph=False)
            per_scene.append(time.perf_counter() - t1)
        t_one = time.perf_counter() - t0
        bat = [pathtracer.SpectralRasterizer(ctx, d, scene=s) for d, s in zip(descs, devs)]
        t0 = time.perf_counter()
        eng.render(bat, spp, use_graph=True)
        t_bat = time.perf_counter() - t0
        same = all(np.allclose(a.film(), b.film(), rtol=1e-4, atol=1e-6) for a, b in zip(one[:6], bat[:6]))
        plain = [pathtracer.SpectralRasterizer(ctx, d, scene=s) for d, s in zip(descs, devs)]
        t0 = time.perf_counter()
        for r, s in zip(plain, spp):
            r.rasterize_scene(s)
        t_plain = time.perf_counter() - t0
        out.update({"plain_job_render": {"seconds": t_plain, "msamples_s": total / t_plain / 1e6},
                    "one_by_one": {"seconds": t_one, "msamples_s": total / t_one / 1e6},
                    "batched_graph": {"seconds": t_bat, "msamples_s": total / t_bat / 1e6},
                    "speedup": t_one / t_bat, "speedup_vs_plain": t_plain / t_bat,
                    "films_equal_first6": bool(same)})
        # Where the time goes: throughput of each resolution class rendered
        # alone on the engine.  When the classes that hold most samples
        # already run at the batch's rate alone, batching has only the small
        # images' tails to remove.
        by_res = {}
        for p, sec in zip(params, per_scene):
            c = by_res.setdefault(str(p["res"]), {"scenes": 0, "samples": 0, "seconds": 0.0})
            c["scenes"] += 1
            c["samples"] += p["res"] ** 2 * p["spp"]
            c["seconds"] += sec
        for c in by_res.values():
            c["msamples_s_alone"] = c["samples"] / c["seconds"] / 1e6
            c["share_of_samples"] = c["samples"] / total
        big = by_res.get("1024", {})
        out["limiter"] = {"one_by_one_by_resolution": by_res,
                          "batched_over_1024_alone": (total / t_bat / 1e6) / big["msamples_s_alone"] if big else None}
        for r in one + bat + plain:
            r.close()
        # Small requests (the same 48 scenes at 128x128, 16 spp): the plain
        # path pays its per-job tail and host polls 48 times, the engine once.
        small = [scenes.RenderSettings(**{**d.settings.__dict__, "width": 128, "height": 128}) for d in descs]
        n_small = 48 * 128 * 128 * 16
        warm = pathtracer.SpectralRasterizer(ctx, descs[0], scene=devs[0], settings=small[0])
        warm.rasterize_scene(1)
        warm.close()
        plain = [pathtracer.SpectralRasterizer(ctx, d, scene=s, settings=st) for d, s, st in zip(descs, devs, small)]
        t0 = time.perf_counter()
        for r in plain:
            r.rasterize_scene(16)
        t_plain_s = time.perf_counter() - t0
        bat = [pathtracer.SpectralRasterizer(ctx, d, scene=s, settings=st) for d, s, st in zip(descs, devs, small)]
        t0 = time.perf_counter()
        eng.render(bat, [16] * 48, use_graph=True)
        t_bat_s = time.perf_counter() - t0
        out["small_requests"] = {"workload": "the 48 scenes at 128x128, 16 spp each",
                                 "plain_job_render": {"seconds": t_plain_s, "msamples_s": n_small / t_plain_s / 1e6},
                                 "batched_graph": {"seconds": t_bat_s, "msamples_s": n_small / t_bat_s / 1e6},
                                 "speedup_vs_plain": t_plain_s / t_bat_s}
        for r in plain + bat:
            r.close()
    finally:
        eng.close()
        for s in devs:
            s.close()
    return out


def bench_serving(ctx, rate=20.0, duration=8.0, resolutions=(128, 256), n_scenes=12, max_tri=300_000,
                  layout="q8", timeout=600.0, caps=(), followup_caps=(), skip=()):
    """Serving loop: Poisson arrivals, progressive 16 -> 64 -> 256 spp per
    request, scenes drawn from a resident pool of the batched-scenes
    distribution (`n_scenes` scenes of up to `max_tri` triangles at
    `resolutions`); continuous batching vs one request at a time on the same
    engine and kernels."""
    from rise_b200 import pathtracer, scenes, serving
    params = scenes.batch_scene_params(n=n_scenes, seed=5, max_tri=max_tri, resolutions=resolutions)
    descs = [scenes.batch_scene(p) for p in params]
    devs = [pathtracer.upload_scene(ctx, d, layout) for d in descs]
    pool = list(zip(descs, devs))
    arrivals = serving.poisson_arrivals(rate, duration, seed=9)

    def make(times=arrivals):
        rng = np.random.default_rng(10)
        reqs = []
        for i, t in enumerate(times):
            k = int(rng.integers(len(pool)))
            st = scenes.RenderSettings(**{**descs[k].settings.__dict__, "seed": 1000 + i})
            reqs.append(serving.Request(i, t, k, st))
        return reqs
    out = {"workload": f"Poisson {rate}/s for {duration}s, progressive 16/64/256 spp, {n_scenes} resident scenes "
                       f"(triangles 10k-{max_tri // 1000}k, resolutions {list(resolutions)}, depth 8-16, "
                       f"{layout} BVHs)", "requests": len(arrivals)}
    try:
        # Warm-up: first launches of every kernel instantiation serving uses.
        serving.serve(ctx, pool, make(arrivals[:12]), mode="continuous")
        if "continuous" not in skip:
            out["continuous"] = serving.serve(ctx, pool, make(), mode="continuous", timeout=timeout)
        # Continuous batching with at most `cap` requests in flight: under
        # overload an unbounded mix interleaves every resident scene's paths.
        for cap in caps:
            out[f"continuous_max{cap}"] = serving.serve(ctx, pool, make(), mode="continuous", timeout=timeout,
                                                        max_active=cap)
        for cap in followup_caps:
            out[f"continuous_followup{cap}"] = serving.serve(ctx, pool, make(), mode="continuous", timeout=timeout,
                                                             max_followup=cap)
        if "fifo" not in skip:
            out["fifo"] = serving.serve(ctx, pool, make(), mode="fifo", timeout=timeout)
    finally:
        for s in devs:
            s.close()
    return out


def bench_serving_cpu(ctx, n_requests=6, rate=0.2, seed=13):
    """The serving comparison against the reference renderer, on a stated
    subset of the request stream: 6 requests (Poisson, 0.2/s) over 4
    resident scenes of the batched distribution restricted to 128 x 128
    pixels and 10k-60k triangles, each asking for 16, then 64, then 256 spp.
    The reference renders them one at a time on all host cores (its own
    per-pixel integrator through oracle.RefRenderer, pixels in parallel; the
    scenes written in its scene language and loaded before the stream
    starts); the device serves the same requests (same scenes, arrival
    times) continuously and one at a time.  Reported: p50 / p99 latency per
    level on each arm and the ratio of the reference's p99 to the device's."""
    import shutil
    import tempfile
    import oracle
    from oracle.scene_writer import write_risescene
    from rise_b200 import pathtracer, scenes, serving
    if oracle.rise_ref() is None:
        return {"unavailable": "the reference renderer (oracle/_ref/librise_ref.so) is not built"}
    params = scenes.batch_scene_params(n=4, seed=17, max_tri=60_000, resolutions=(128,))
    descs = [scenes.batch_scene(p) for p in params]
    rng = np.random.default_rng(seed)
    times = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    picks = rng.integers(len(descs), size=n_requests)
    levels = (16, 64, 256)
    tmp = tempfile.mkdtemp(prefix="rise_serving_")
    out = {"subset": f"{n_requests} requests, Poisson {rate}/s, 4 resident scenes of the batched distribution "
                     f"at 128x128 with {min(p['n_tri'] for p in params) // 1000}k-"
                     f"{max(p['n_tri'] for p in params) // 1000}k triangles, levels 16/64/256 spp",
           "cpu_threads": oracle.RISE_THREADS}
    try:
        refs = [oracle.RefRenderer(write_risescene(d, tmp, f"s{i}", spp=16)) for i, d in enumerate(descs)]
        lat = {lv: [] for lv in levels}
        t0 = time.perf_counter()
        for i, (t, k) in enumerate(zip(times, picks)):
            now = time.perf_counter() - t0
            if now < t:
                time.sleep(t - now)
            done = 0
            for lv in levels:
                refs[k].integrate(lv - done, batch=1000 * i + lv)
                done = lv
                lat[lv].append(time.perf_counter() - t0 - t)
        wall = time.perf_counter() - t0
        for r in refs:
            r.close()
        samples = sum(256 * 128 * 128 for _ in picks)
        out["cpu_reference"] = {"wall_s": wall, "msamples_s": samples / wall / 1e6, "latency": {
            str(lv): {"p50_s": float(np.percentile(v, 50)), "p99_s": float(np.percentile(v, 99))}
            for lv, v in lat.items()}}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    devs = [pathtracer.upload_scene(ctx, d, "q8") for d in descs]
    try:
        pool = list(zip(descs, devs))

        def make():
            return [serving.Request(i, float(t), int(k), scenes.RenderSettings(
                **{**descs[int(k)].settings.__dict__, "seed": 1000 + i})) for i, (t, k) in enumerate(zip(times, picks))]
        serving.serve(ctx, pool, make()[:2], mode="continuous")   # warm-up
        for mode in ("continuous", "fifo"):
            out["gpu_" + mode] = serving.serve(ctx, pool, make(), mode=mode)
    finally:
        for d in devs:
            d.close()
    out["p99_ratio_cpu_over_gpu"] = {
        mode: {lv: out["cpu_reference"]["latency"][lv]["p99_s"] / out["gpu_" + mode]["latency"][lv]["p99_s"]
               for lv in out["cpu_reference"]["latency"]} for mode in ("continuous", "fifo")}
    return out


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    import oracle
    from rise_b200 import scenes
    tri = scenes.soup_triangles(N_TRI, seed=SEED)
    rays = scenes.sphere_rays(N_RAYS, seed=SEED)
    kind = "reference" if oracle.ref() is not None else "port"
    b = oracle.BVH(tri, "ref" if kind == "reference" else "port")
    threads = os.cpu_count()
    sample = 65536
    for i in range(args.warmup):
        b.closest(rays[(i * sample) % N_RAYS:][:sample], threads=threads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        s = (i * sample) % (N_RAYS - sample)
        b.closest(rays[s:s + sample], threads=threads)
    dt = time.perf_counter() - t0
    v = args.steps * sample / dt / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": {"workload": REF_WORKLOAD, "n_tri": N_TRI, "n_rays": N_RAYS},
        "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} rays per step of the {N_RAYS}-ray set, BVH build excluded"},
        "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    from rise_b200 import raycaster, scenes

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if args.serving_full:
        ctx = raycaster.Context(local, 120 * 10**9)
        res = bench_serving(ctx, rate=20.0, duration=60.0, resolutions=scenes.RESOLUTIONS, n_scenes=48,
                            max_tri=1_000_000, timeout=3600.0, followup_caps=(4,),
                            skip=tuple(x for x in args.serving_skip.split(",") if x))
        res["budget_bytes"] = 120 * 10**9
        print(json.dumps({"serving_full": res}))
        ctx.close()
        return
    if args.pt_only or args.large_only:
        ctx = raycaster.Context(local)
        print(json.dumps(bench_large_scene(ctx) if args.large_only else bench_path_tracer(ctx, rank, cpu_baseline=False)))
        ctx.close()
        return
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    tri = scenes.soup_triangles(N_TRI, seed=SEED)
    rays = scenes.sphere_rays(N_RAYS, seed=SEED + 1000 * rank)
    srays = scenes.sphere_rays(N_RAYS, seed=SEED + 1000 * rank, shadow=True)

    ctx = raycaster.Context(local)
    sf = raycaster.Scene(ctx)
    sf.add_triangles(tri)
    sf.commit("f32")
    sq = raycaster.Scene(ctx)
    sq.add_triangles(tri)
    sq.commit("q8")
    sh16 = raycaster.Scene(ctx)
    sh16.add_triangles(tri)
    sh16.commit("f16")
    rf, rq, rh = raycaster.RayCaster(sf), raycaster.RayCaster(sq), raycaster.RayCaster(sh16)

    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    d_rays = torch.from_numpy(rays).cuda()
    d_srays = torch.from_numpy(srays).cuda()
    d_hits = torch.empty((N_RAYS, 4), dtype=torch.float32, device="cuda")
    d_occ = torch.empty(N_RAYS, dtype=torch.uint8, device="cuda")

    def step_closest(rc):
        rc.cast_rays_device(d_rays.data_ptr(), d_hits.data_ptr(), N_RAYS, sh)

    def step_any(rc):
        rc.cast_shadow_rays_device(d_srays.data_ptr(), d_occ.data_ptr(), N_RAYS, sh)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # Headline: FP16-quantised child boxes (conservative, the same hits as
    # FP32 nodes: tests/test_raycast_gpu.py); FP32 and 8-bit nodes are variants.
    for _ in range(max(3, args.warmup)):
        step_closest(rh)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_closest(rh)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * N_RAYS / (ms_step * 1e-3) / 1e6

    # Variants (same device-resident protocol, shorter runs).
    def timed(fn, rc, n=20):
        for _ in range(3):
            fn(rc)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn(rc)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    variants = {}
    for name, fn, rc in (("closest_f32", step_closest, rf), ("any_f32", step_any, rf), ("closest_q8", step_closest, rq),
                         ("any_q8", step_any, rq), ("any_f16", step_any, rh)):
        variants[name] = N_RAYS / (timed(fn, rc) * 1e-3) / 1e6
    hit_rate = float((d_hits[:, 1].view(torch.int32) >= 0).float().mean())

    # End to end through the public host-buffer API: pinned host rays in,
    # host hits out, copies inside the timed region.
    h_rays = torch.from_numpy(rays).pin_memory().numpy()
    h_hits = torch.empty(N_RAYS * 16, dtype=torch.uint8).pin_memory().numpy().view(raycaster.HIT_DTYPE)
    from rise_b200._native import check, lib
    import ctypes
    for _ in range(2):
        check(lib().rtb200_cast_closest(sh16.h, ctypes.c_void_p(h_rays.ctypes.data), N_RAYS,
                                        ctypes.c_void_p(h_hits.ctypes.data)), ctx.h)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        check(lib().rtb200_cast_closest(sh16.h, ctypes.c_void_p(h_rays.ctypes.data), N_RAYS,
                                        ctypes.c_void_p(h_hits.ctypes.data)), ctx.h)
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * N_RAYS / e2e_s / 1e6

    peak, peak_kind = load_peaks()
    achieved = BYTES_CLOSEST * N_RAYS / (ms_step * 1e-3) / 1e9
    prof = "raycast_closest_f16_soup1M"
    traffic = profiled(prof, "traffic_bytes_per_launch")
    info = sh16.info()

    out = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded: triangles seed 7, rays seed 7 + 1000*rank)",
        "config": {"workload": WORKLOAD, "n_tri": N_TRI, "n_rays_per_gpu": N_RAYS, "layout": "f16",
                   "parallelism": f"replicas x{world}",
                   "l2_policy": "inputs larger than L2 (rays 134 MB per pass); scene (nodes + triangles) stays resident",
                   "bvh_nodes": info["n_nodes"], "scene_device_bytes": info["device_bytes"],
                   "bvh_build_s": round(info["build_seconds"], 3), "hit_rate": round(hit_rate, 6)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "traffic_source": f"ncu capture of this kernel on this workload (profiles/{prof})",
                     "algorithmic_bytes_per_ray": BYTES_CLOSEST,
                     # HBM does not bind this kernel (the scene is L2-resident):
                     # its limiters are the L1/texture pipe and instruction
                     # issue under divergence, from the same ncu capture.
                     "limiter": {"l1tex_throughput_pct": profiled(prof, "l1tex_throughput_pct"),
                                 "issue_active_pct": profiled(prof, "issue_active_pct"),
                                 "threads_per_warp_instruction": profiled(prof, "threads_per_warp_instruction")}},
        "variants_mrays_s": variants,
        "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": 32 * N_RAYS,
                "d2h_bytes_per_step": 16 * N_RAYS},
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, kind, cores, n = cpu_reference_time(tri, rays)
        out["cpu_baseline"] = {"value": v, "unit": "Mrays/s", "cores": cores, "kind": kind,
                               "sample": f"first {n} rays of the {N_RAYS}-ray set, closest-hit, BVH build excluded"}
    sf.close()
    sq.close()
    sh16.close()
    if not args.no_path_tracer:
        out["path_tracer"] = bench_path_tracer(ctx, rank, cpu_baseline=world == 1 and not args.no_cpu_baseline)
        # The headline path-tracing metric: Msamples/s at relMSE <= 1e-3
        # against the reference renderer's FP64 16384-spp image.
        conv = out["path_tracer"].get("vs_reference_fp64_16384spp", {})
        out["msamples_s_at_relmse_1e-3"] = {f"C1_{k}": v.get("msamples_s_at_relmse_1e-3") for k, v in conv.items()}
        if not args.no_large:
            out["path_tracer_large"] = bench_large_scene(ctx)
        if not args.no_batch:
            out["batch"] = bench_batch(ctx)
            out["serving"] = bench_serving(ctx)
            if world == 1 and not args.no_cpu_baseline:
                out["serving_vs_reference"] = bench_serving_cpu(ctx)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
