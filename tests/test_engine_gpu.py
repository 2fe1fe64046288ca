"""Batched and continuously batched rendering (through the C ABI).

Every job draws its random numbers from (its seed, pixel, sample,
dimension) only, so a job's film must not depend on what else shares the
wavefront: the same job rendered alone, in a batch, from a captured CUDA
graph, or submitted while other jobs are in flight gives the same image up
to the order of floating-point film additions (relative 1e-5).
"""
import dataclasses

import numpy as np
import pytest

from rise_b200 import pathtracer, raycaster, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = raycaster.Context(0)
    yield c
    c.close()


def mixed_descs():
    a = scenes.cornell_box(32, 32)
    b = scenes.spheres_scene(grid=48, n_spheres=6, sphere_tris=600, width=40, height=24, max_depth=10)
    c = scenes.cornell_box(48, 32, spp_seed=7, nee_per_lambda=0)
    return [a, b, c]


def alone(ctx, desc, spp):
    r = pathtracer.SpectralRasterizer(ctx, desc)
    try:
        r.rasterize_scene(spp)
        return r.film()
    finally:
        r.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_equals_alone(ctx, use_graph):
    descs = mixed_descs()
    spp = [8, 4, 12]
    ref = [alone(ctx, d, s) for d, s in zip(descs, spp)]
    eng = pathtracer.Engine(ctx, capacity=1 << 15)
    rs = [pathtracer.SpectralRasterizer(ctx, d) for d in descs]
    try:
        eng.render(rs, spp, use_graph=use_graph)
        for r, f in zip(rs, ref):
            assert np.allclose(r.film(), f, rtol=1e-5, atol=1e-7)
            assert r.stats()["spp"] in spp
    finally:
        for r in rs:
            r.close()
        eng.close()


def test_continuous_submission_equals_alone(ctx):
    descs = mixed_descs()
    ref0 = alone(ctx, descs[0], 16)
    ref1 = alone(ctx, descs[1], 8)
    ref2 = alone(ctx, descs[2], 4)
    eng = pathtracer.Engine(ctx, capacity=1 << 14)
    r0, r1, r2 = (pathtracer.SpectralRasterizer(ctx, d) for d in descs)
    try:
        eng.submit(r0, 16)
        eng.step(2)
        eng.submit(r1, 8)          # arrives while r0 is in flight
        eng.step(2)
        eng.submit(r2, 4)
        live = {0: r0, 1: r1, 2: r2}
        for _ in range(10000):
            eng.step(2)
            for k in list(live):
                done, total = eng.progress(live[k])
                if done == total:
                    eng.retire(live.pop(k))
            if not live:
                break
        assert not live
        assert np.allclose(r0.film(), ref0, rtol=1e-5, atol=1e-7)
        assert np.allclose(r1.film(), ref1, rtol=1e-5, atol=1e-7)
        assert np.allclose(r2.film(), ref2, rtol=1e-5, atol=1e-7)
        # Progressive: a second request continues the same sample sequence.
        eng.submit(r1, 8)
        for _ in range(10000):
            eng.step(2)
            d, t = eng.progress(r1)
            if d == t:
                break
        eng.retire(r1)
        assert np.allclose(r1.film(), alone(ctx, descs[1], 16), rtol=1e-5, atol=1e-7)
    finally:
        for r in (r0, r1, r2):
            r.close()
        eng.close()


@pytest.mark.parametrize("mode,caps", [("continuous", {}), ("fifo", {}), ("continuous", {"max_active": 2}),
                                       ("continuous", {"max_followup": 1})])
def test_serving_levels_complete_and_match_alone(ctx, mode, caps):
    from rise_b200 import serving
    descs = [scenes.cornell_box(32, 32), scenes.spheres_scene(grid=32, n_spheres=4, sphere_tris=400,
                                                              width=24, height=24, max_depth=8)]
    devs = [pathtracer.upload_scene(ctx, d) for d in descs]
    pool = list(zip(descs, devs))
    reqs = []
    for i, t in enumerate([0.0, 0.005, 0.01, 0.02, 0.03]):
        k = i % 2
        st = scenes.RenderSettings(**{**descs[k].settings.__dict__, "seed": 500 + i})
        reqs.append(serving.Request(i, t, k, st, levels=(4, 8)))
    try:
        res = serving.serve(ctx, pool, reqs, mode=mode, capacity=1 << 14, **caps)
        assert res["requests"] == 5 and set(res["latency"]) == {"4", "8"}
        assert all(len(r.done_at) == 2 and r.done_at[0] <= r.done_at[1] for r in reqs)
        assert res["latency"]["8"]["p99_s"] >= res["latency"]["4"]["p50_s"]
    finally:
        for s in devs:
            s.close()


def test_retire_before_done_is_refused(ctx):
    d = scenes.cornell_box(64, 64)
    eng = pathtracer.Engine(ctx, capacity=1 << 12)
    r = pathtracer.SpectralRasterizer(ctx, d)
    try:
        eng.submit(r, 64)
        eng.step(2)
        with pytest.raises(Exception) as ei:
            eng.retire(r)
        assert "E_NOT_READY" in str(ei.value)
        for _ in range(100000):
            eng.step(4)
            a, b = eng.progress(r)
            if a == b:
                break
        eng.retire(r)
    finally:
        r.close()
        eng.close()


def test_autotune_picks_a_config_and_poll_does_not_change_images(ctx):
    from rise_b200 import autotune
    descs = mixed_descs()
    devs = [pathtracer.upload_scene(ctx, d) for d in descs]
    spp = [4, 2, 4]
    try:
        best, tried = autotune.tune(ctx, descs, devs, spp, capacities=(1 << 14, 1 << 16), polls=(2, 8),
                                    use_cache=False)
        assert len(tried) == 4 and best in tried and best.msamples_s > 0
        films = []
        for poll in (2, 8):
            eng = pathtracer.Engine(ctx, best.capacity)
            eng.set_poll(poll)
            rs = [pathtracer.SpectralRasterizer(ctx, d, scene=s) for d, s in zip(descs, devs)]
            eng.render(rs, spp)
            films.append([r.film() for r in rs])
            for r in rs:
                r.close()
            eng.close()
        for a, b in zip(*films):
            assert np.allclose(a, b, rtol=1e-5, atol=1e-7)
    finally:
        for s in devs:
            s.close()


def test_progress_callback_reports_and_can_stop_a_render(ctx):
    """IProgressCallback semantics: progress grows to the total; a callback
    that returns True leaves the image unchanged; one that returns False
    stops the pass with every pixel at the same whole number of samples, so
    the film equals an uninterrupted render of that many samples."""
    d = scenes.cornell_box(128, 128)
    scene = pathtracer.upload_scene(ctx, d)
    try:
        ref = pathtracer.SpectralRasterizer(ctx, d, scene=scene)
        ref.rasterize_scene(64)
        seen = []
        r = pathtracer.SpectralRasterizer(ctx, d, scene=scene)
        r.set_progress(lambda p, t: seen.append((p, t)) or True)
        assert r.rasterize_scene(64)
        assert seen and all(t == 64 for _, t in seen) and seen[-1][0] == 64
        assert all(a[0] <= b[0] for a, b in zip(seen, seen[1:]))
        assert np.allclose(r.film(), ref.film(), rtol=1e-5, atol=1e-7)
        stop = pathtracer.SpectralRasterizer(ctx, d, scene=scene)
        stop.set_progress(lambda p, t: False)
        assert stop.rasterize_scene(4096) is False
        k = stop.stats()["spp"]
        assert 0 < k < 4096
        part = pathtracer.SpectralRasterizer(ctx, d, scene=scene)
        part.rasterize_scene(k)
        assert np.allclose(stop.film(), part.film(), rtol=1e-5, atol=1e-7)
        # The next pass continues from sample k.
        stop.set_progress(None)
        assert stop.rasterize_scene(8)
        assert stop.stats()["spp"] == k + 8
        for x in (ref, r, stop, part):
            x.close()
    finally:
        scene.close()


def test_engine_cancel_stops_a_served_request(ctx):
    d = scenes.cornell_box(128, 128)
    scene = pathtracer.upload_scene(ctx, d)
    eng = pathtracer.Engine(ctx)
    try:
        a = pathtracer.SpectralRasterizer(ctx, d, scene=scene)
        b = pathtracer.SpectralRasterizer(ctx, d, scene=scene, settings=dataclasses.replace(d.settings, seed=5))
        eng.submit(a, 4096)
        eng.submit(b, 16)
        eng.step(4)
        eng.cancel(a)
        for _ in range(10000):
            da, ta = eng.progress(a)
            db, tb = eng.progress(b)
            if da >= ta and db >= tb:
                break
            eng.step(4)
        assert da == ta and ta < 4096 * 128 * 128 and ta % (128 * 128) == 0
        eng.retire(a)
        eng.retire(b)
        assert a.stats()["spp"] == ta // (128 * 128) and b.stats()["spp"] == 16
        assert np.isfinite(a.film()).all()
        a.close()
        b.close()
    finally:
        eng.close()
        scene.close()
