"""A scene read from the reference's scene format renders on the device as
the oracle renders it (same random numbers)."""
import numpy as np
import pytest

import oracle
from rise_b200 import pathtracer, raycaster, scenefile

from test_scenefile import SCENE

pytestmark = pytest.mark.gpu


OMNI = """
omni_light
{
	name		bulb
	power		0.5
	position	0.3 0.8 0.4
	color		1.0 0.9 0.7
}
"""


@pytest.mark.parametrize("extra", ["", OMNI], ids=["area", "area+omni"])
def test_ingested_scene_matches_oracle(extra):
    s = scenefile.load_scene(text=SCENE.replace("\tpixel_filter\tbox\n", "") + extra)
    assert len(s.desc.point_lights) == (1 if extra else 0)
    ctx = raycaster.Context(0)
    try:
        r = pathtracer.SpectralRasterizer(ctx, s.desc)
        try:
            r.rasterize_scene(s.spp)
            g = r.film().astype(np.float64)
        finally:
            r.close()
    finally:
        ctx.close()
    o = oracle.pt_render(s.desc, s.spp)
    assert np.isfinite(g).all() and g[..., 1].mean() > 0
    close = (np.abs(g - o) <= 1e-3 * (np.abs(o) + 1e-3)).all(axis=2)
    assert close.mean() > 0.9, close.mean()
    assert np.mean((g - o) ** 2 / (o ** 2 + 1e-2)) < 1e-3
