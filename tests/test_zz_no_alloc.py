"""rtb200_cast_closest_noalloc: closest hit without any device allocation.

This entry point is for callers that cannot call cudaMalloc/cudaFree when
they cast rays (a host application whose pool allocator owns all device
memory, or a latency-critical thread that cannot afford the device-wide
synchronisation those calls may cause).  Its kernel scratch lives in a
static device array instead of scene-owned memory.  The test calls it
through the C ABI twice in a row on each node layout (the second call must
see a cleared work counter, not the first call's leftovers) and compares
each result with the regular device entry point and with the reference BVH
(through the oracle, under the ray-cast parity rules of tests/parity.py);
a deep BVH runs the local-memory-stack kernel through the same scratch; an
empty batch, a misaligned buffer and a batch beyond the stated maximum are
refused or ignored before any launch.  The file is named to be collected
last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from parity import closest_report
from rise_b200 import _native, raycaster, scenes

pytestmark = pytest.mark.gpu


def _cast(L, fn, s, d_rays, n, d_out, st, ctx):
    _native.check(fn(s.h, ctypes.c_void_p(d_rays.data_ptr()), n, ctypes.c_void_p(d_out.data_ptr()), st), ctx.h)


@pytest.mark.parametrize("case", ["f32", "q8", "f16", "deep"])
def test_noalloc_matches_device_entry_point_and_reference_twice(case):
    torch = pytest.importorskip("torch")
    L = _native.lib()
    if case == "deep":
        tri = scenes.nested_clusters()
        rays = scenes.cluster_rays(tri, 100000, seed=22)
    else:
        tri = scenes.soup_triangles(50000, seed=21)
        rays = scenes.sphere_rays(300000, seed=21)
    with raycaster.Context(0) as ctx:
        s = raycaster.Scene(ctx)
        s.add_triangles(tri)
        s.commit(case if case in ("q8", "f16") else "f32")
        d_rays = torch.from_numpy(rays).cuda()
        d_ref = torch.empty((len(rays), 4), dtype=torch.float32, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _cast(L, L.rtb200_cast_closest_device, s, d_rays, len(rays), d_ref, st, ctx)
        torch.cuda.synchronize()
        assert L.rtb200_scene_device_status(s.h, st) == _native.OK
        ref = d_ref.cpu().numpy().view(raycaster.HIT_DTYPE).reshape(-1)
        assert (ref["prim"] >= 0).mean() > 0.3
        b = oracle.BVH(tri, "port")
        ref_ids, ref_t = b.closest(rays)
        for call in range(2):
            d_out = torch.full((len(rays), 4), -7.0, dtype=torch.float32, device="cuda")
            _cast(L, L.rtb200_cast_closest_noalloc, s, d_rays, len(rays), d_out, st, ctx)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(raycaster.HIT_DTYPE).reshape(-1)
            # Same kernel, same inputs as the device entry point: identical
            # ids, distances within the 4-ulp tolerance of the ray-cast tests.
            assert (got["prim"] == ref["prim"]).all(), call
            hit = ref["prim"] >= 0
            ulps = np.abs(got["t"][hit].astype(np.float64) - ref["t"][hit]) / np.spacing(np.abs(ref["t"][hit]))
            assert ulps.max() <= 4, call
            # And the reference BVH's hits under the parity rules.
            rep = closest_report(tri, rays, got, ref_ids, ref_t)
            assert not rep["bad"] and rep["t_over"] == 0, (call, rep["bad"][:5], rep["t_over"])
        s.close()


def test_noalloc_refuses_bad_calls_without_launching():
    torch = pytest.importorskip("torch")
    L = _native.lib()
    tri = scenes.soup_triangles(1000, seed=3)
    rays = scenes.sphere_rays(1024, seed=3)
    with raycaster.Context(0) as ctx:
        s = raycaster.Scene(ctx)
        s.add_triangles(tri)
        s.commit("f32")
        d_rays = torch.from_numpy(rays).cuda()
        d_out = torch.full((len(rays), 4), -7.0, dtype=torch.float32, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        # An empty batch is a no-op.
        assert L.rtb200_cast_closest_noalloc(s.h, ctypes.c_void_p(d_rays.data_ptr()), 0,
                                             ctypes.c_void_p(d_out.data_ptr()), st) == _native.OK
        torch.cuda.synchronize()
        assert (d_out.cpu().numpy() == -7.0).all()
        # Buffers off the 16-byte alignment of the ray and hit records.
        rc = L.rtb200_cast_closest_noalloc(s.h, ctypes.c_void_p(d_rays.data_ptr() + 4), 8,
                                           ctypes.c_void_p(d_out.data_ptr()), st)
        assert rc == _native.E_INVALID and b"aligned" in L.rtb200_last_error(ctx.h)
        # Sizes beyond the stated maximum are rejected before any launch.
        rc = L.rtb200_cast_closest_noalloc(s.h, ctypes.c_void_p(d_rays.data_ptr()),
                                           _native.NOALLOC_MAX_RAYS + 1, ctypes.c_void_p(d_out.data_ptr()), st)
        assert rc == _native.E_INVALID
        assert b"exceed" in L.rtb200_last_error(ctx.h)
        torch.cuda.synchronize()
        assert (d_out.cpu().numpy() == -7.0).all()
        s.close()
