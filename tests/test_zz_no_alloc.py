"""rtb200_cast_closest_noalloc: closest hit without any device allocation.

This entry point is for callers that cannot call cudaMalloc/cudaFree when
they cast rays (a host application whose pool allocator owns all device
memory, or a latency-critical thread that cannot afford the device-wide
synchronisation those calls may cause).  Its kernel scratch lives in a
static device array instead of scene-owned memory; this test calls it
through the C ABI twice in a row (the second call must see a cleared work
counter, not the first call's leftovers) and compares each result with the
regular device entry point.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from rise_b200 import _native, raycaster, scenes

pytestmark = pytest.mark.gpu


def test_noalloc_matches_device_entry_point_twice():
    torch = pytest.importorskip("torch")
    L = _native.lib()
    tri = scenes.soup_triangles(50000, seed=21)
    rays = scenes.sphere_rays(300000, seed=21)
    with raycaster.Context(0) as ctx:
        s = raycaster.Scene(ctx)
        s.add_triangles(tri)
        s.commit("f32")
        d_rays = torch.from_numpy(rays).cuda()
        d_ref = torch.empty((len(rays), 4), dtype=torch.float32, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _native.check(L.rtb200_cast_closest_device(s.h, ctypes.c_void_p(d_rays.data_ptr()), len(rays),
                                                   ctypes.c_void_p(d_ref.data_ptr()), st), ctx.h)
        torch.cuda.synchronize()
        ref = d_ref.cpu().numpy().view(raycaster.HIT_DTYPE).reshape(-1)
        assert (ref["prim"] >= 0).mean() > 0.5
        for call in range(2):
            d_out = torch.full((len(rays), 4), -7.0, dtype=torch.float32, device="cuda")
            _native.check(L.rtb200_cast_closest_noalloc(s.h, ctypes.c_void_p(d_rays.data_ptr()), len(rays),
                                                        ctypes.c_void_p(d_out.data_ptr()), st), ctx.h)
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(raycaster.HIT_DTYPE).reshape(-1)
            # Same kernel, same inputs: identical ids; distances within the
            # 4-ulp tolerance the other ray-cast tests use (here exact).
            assert (got["prim"] == ref["prim"]).all(), call
            hit = ref["prim"] >= 0
            ulps = np.abs(got["t"][hit].astype(np.float64) - ref["t"][hit]) / np.spacing(np.abs(ref["t"][hit]))
            assert ulps.max() <= 4, call
        # Sizes beyond the stated maximum are rejected before any launch.
        rc = L.rtb200_cast_closest_noalloc(s.h, ctypes.c_void_p(d_rays.data_ptr()),
                                           _native.NOALLOC_MAX_RAYS + 1, ctypes.c_void_p(d_ref.data_ptr()), st)
        assert rc == _native.E_INVALID
        assert b"exceed" in L.rtb200_last_error(ctx.h)
        s.close()
