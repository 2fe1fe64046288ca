""".RISEscene ingest (host side): chunk grammar, the supported chunks'
semantics, and refusals for what the renderer cannot draw."""
import math
import os

import numpy as np
import pytest

from rise_b200 import scenefile, scenes

REF = "/root/reference"

SCENE = """RISE ASCII SCENE 7
# a small test scene in the reference's chunk format
/* block
   comment */
pathtracing_spectral_rasterizer
{
	samples			16
	nmbegin			400
	nmend			700
	pixel_filter	box
	rr_min_depth	2
}

film
{
	width	40
	height	30
}

pinhole_camera
{
	location	0.5 0.5 -1.5
	lookat		0.5 0.5 0
	up			0 1 0
	fov			40
}

spectral_painter
{
	name	white
	cp		400 0.5
	cp		700 0.9
	nmbegin	400
	nmend	700
}

spectral_painter
{
	name	light
	cp		400 10
	cp		700 10
	scale	4
}

lambertian_material
{
	name		matte
	reflectance	white
}

lambertian_luminaire_material
{
	name		lamp
	exitance	light
	scale		3.0
	material	none
}

clippedplane_geometry
{
	name	floor
	pta		0 0 0
	ptb		0 0 1
	ptc		1 0 1
	ptd		1 0 0
}

clippedplane_geometry
{
	name	lightquad
	pta		0.4 0.99 0.4
	ptb		0.6 0.99 0.4
	ptc		0.6 0.99 0.6
	ptd		0.4 0.99 0.6
}

box_geometry
{
	name	cube
	width	0.2
	height	0.4
	depth	0.2
}

standard_object
{
	name		floor
	geometry	floor
	material	matte
}

standard_object
{
	name		lamp
	geometry	lightquad
	material	lamp
}

standard_object
{
	name		cube
	geometry	cube
	material	matte
	position	0.5 0.2 0.5
	orientation	0 30 0
	scale		1 1 1
}
"""


def test_small_scene_loads_with_reference_semantics():
    s = scenefile.load_scene(text=SCENE)
    d, st = s.desc, s.desc.settings
    assert s.spp == 16 and (st.width, st.height) == (40, 30) and st.fov_deg == 40.0
    assert (st.lambda_min, st.lambda_max, st.filter, st.rr_min_depth, st.max_depth) == (400, 700, 0, 2, 128)
    assert d.n_tri == 2 + 2 + 12 and len(d.meshes) == 3
    # Spectral painter: 2 control points -> 2 bins over 400..700 sampled at 400 and 550 nm.
    white = d.spectra[d.materials[0].reflectance]
    assert np.allclose(white.amps, [0.5, 0.5 + 0.4 * 150 / 300]) and (white.begin, white.end) == (400, 700)
    assert np.allclose(white.value_at([399, 400, 549, 551, 700, 701]), [0, 0.5, 0.5, 0.7, 0.7, 0])
    # Luminaire: radiance = exitance * scale / pi; the painter's scale does not touch the spectrum.
    lamp = d.spectra[d.materials[1].emission]
    assert np.allclose(lamp.amps, 10 * 3.0 / math.pi)
    # Clipped plane: triangles (a, b, c), (a, c, d), double sided by default.
    assert np.allclose(d.tri9[0], [0, 0, 0, 0, 0, 1, 1, 0, 1]) and d.meshes[0][3] == 1
    # Light quad normal (b - a) x (c - a) points down.
    t = d.tri9[2].reshape(3, 3)
    assert np.cross(t[1] - t[0], t[2] - t[0])[1] < 0
    # Box: centred, rotated 30 degrees about y, moved to (0.5, 0.2, 0.5); outward normals.
    cube = d.tri9[4:].reshape(-1, 3, 3).astype(np.float64)
    centre = np.array([0.5, 0.2, 0.5])
    assert np.allclose(cube.reshape(-1, 3).mean(axis=0), centre, atol=1e-6)
    assert np.allclose(cube[..., 1].min(), 0.0, atol=1e-6) and np.allclose(cube[..., 1].max(), 0.4, atol=1e-6)
    n = np.cross(cube[:, 1] - cube[:, 0], cube[:, 2] - cube[:, 0])
    assert ((n * (cube.mean(axis=1) - centre)).sum(axis=1) > 0).all()
    a = math.radians(30)
    corner = np.array([-0.1, -0.2, -0.1])
    rot = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    assert np.isclose(np.linalg.norm(cube.reshape(-1, 3) - (rot @ corner + centre), axis=1), 0, atol=1e-6).any()


def test_defaults_gaussian_filter_and_notes():
    s = scenefile.load_scene(text=SCENE.replace("\tpixel_filter\tbox\n", ""))
    st = s.desc.settings
    assert (st.filter, st.filter_size, st.filter_sigma) == (1, 2.0, 0.35)
    assert any("not denoised" in n for n in s.notes)


@pytest.mark.parametrize("edit,word", [
    (("box_geometry", "sphere_geometry"), "sphere_geometry"),
    (("\tfov\t\t\t40\n", "\tfov\t\t\t40\n\ttheta 10\n"), "theta"),
    (("\tpixel_filter\tbox\n", "\tpixel_filter\tmitchell-netravali\n"), "pixel filter"),
    (("\tmaterial\tmatte\n\tposition", "\tmaterial\tnothere\n\tposition"), "nothere"),
    (("RISE ASCII SCENE 7", "RISE ASCII SCENE 3"), "RISE ASCII SCENE"),
    (("film\n{\n\twidth\t40\n", "film\n{\n\twidth\t40\n\tpixelAR\t2\n"), "pixel aspect"),
])
def test_unsupported_input_is_refused(edit, word):
    with pytest.raises(scenefile.SceneFileError, match=word):
        scenefile.load_scene(text=SCENE.replace(*edit))


def test_rawmesh_and_risemesh_files(tmp_path):
    from risemesh_io import risemesh_bytes
    (tmp_path / "blk.rawmesh").write_text("quad 0 0 0  1 0 0  1 1 0  0 1 0\ntri 0 0 1  1 0 1  0 1 1\n")
    pts = np.array([[0, 0, 2], [1, 0, 2], [0, 1, 2]], np.float64)
    (tmp_path / "t.risemesh").write_bytes(risemesh_bytes(pts, [[0, 1, 2]], double_sided=True))
    text = SCENE + """
rawmesh_geometry
{
	name	blk
	file	blk.rawmesh
}

risemesh_geometry
{
	name	rm
	file	t.risemesh
}

standard_object
{
	name		blk
	geometry	blk
	material	matte
}

standard_object
{
	name		rm
	geometry	rm
	material	matte
	position	0 0 1
}
"""
    s = scenefile.load_scene(text=text, search=[str(tmp_path)])
    d = s.desc
    assert d.n_tri == 16 + 3 + 1
    assert np.allclose(d.tri9[16:19], [[0, 0, 0, 1, 0, 0, 1, 1, 0], [0, 0, 0, 1, 1, 0, 0, 1, 0],
                                       [0, 0, 1, 1, 0, 1, 0, 1, 1]])
    assert d.meshes[3][3] == 0 and d.meshes[4][3] == 1          # rawmesh one-sided, risemesh from its file
    assert np.allclose(d.tri9[19], [0, 0, 3, 1, 0, 3, 0, 1, 3])


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_reference_cornell_scene_loads():
    """The reference's own HWSS Cornell box scene: 6 clipped planes and two
    rawmesh blocks (32 triangles), spectral painters from its data files."""
    p = os.path.join(REF, "scenes", "Tests", "Spectral", "hwss_cornellbox_pt.RISEscene")
    s = scenefile.load_scene(p, search=[REF])
    d = s.desc
    assert d.n_tri == 32 and len(d.meshes) == 8 and s.spp == 256
    assert (d.settings.width, d.settings.height, d.settings.fov_deg) == (512, 512, 37.0)
    emit = [m for m in d.materials if m.emission >= 0]
    assert len(emit) == 1
    assert all(isinstance(sp, scenes.SpectralPacket) for sp in d.spectra)


def test_uniformcolor_painters_become_rgb_spectra():
    text = SCENE.replace("""spectral_painter
{
	name	white
	cp		400 0.5
	cp		700 0.9
	nmbegin	400
	nmend	700
}""", """uniformcolor_painter
{
	name		white
	color		0.8 0.6 0.2
}

uniformcolor_painter
{
	name		srgbwhite
	color		0.5 0.5 0.5
	colorspace	sRGB
}""")
    s = scenefile.load_scene(text=text)
    sp = s.desc.spectra[s.desc.materials[0].reflectance]
    assert isinstance(sp, scenes.SigmoidSpectrum) and sp.scale == 1.0
    want = scenes.rgb_spectrum([0.8, 0.6, 0.2])
    assert (sp.c0, sp.c1, sp.c2) == (want.c0, want.c1, want.c2)
    lin = ((0.5 + 0.055) / 1.055) ** 2.4
    g = [x for x in s.desc.spectra if isinstance(x, scenes.SigmoidSpectrum)][1]
    assert abs(g.value_at([550.0])[0] - lin) < 0.02
    with pytest.raises(scenefile.SceneFileError, match="colour space"):
        scenefile.load_scene(text=text.replace("colorspace	sRGB", "colorspace	ProPhotoRGB"))


def test_blackbody_painter_and_scene_options():
    text = SCENE.replace("""spectral_painter
{
	name	light
	cp		400 10
	cp		700 10
	scale	4
}""", """scene_options
{
	scene_unit	0.001
}

blackbody_painter
{
	name		light
	temperature	3000
	scale		20
}""")
    s = scenefile.load_scene(text=text)
    emit = s.desc.spectra[s.desc.materials[1].emission]
    assert isinstance(emit, scenes.BlackbodySpectrum) and emit.normalize
    # Unit peak at 0.0029 / T metres, times the painter and luminaire scales over pi.
    peak = 0.0029 / 3000 * 1e9
    assert abs(emit.value_at([peak])[0] / (20 * 3.0 / math.pi) - 1) < 1e-6
    nm = np.array([400.0, 550.0, 700.0])
    h, c, k = 6.6260755e-34, 2.99792458e8, 1.380658e-23
    lam = nm * 1e-9
    planck = 2 * math.pi * h * c * c / lam ** 5 / (np.exp(h * c / (k * lam * 3000)) - 1)
    assert np.allclose(emit.value_at(nm) / planck, planck[1] * 0 + emit.value_at([550.0])[0] / planck[1], rtol=1e-6)


def test_omni_light_becomes_point_light():
    text = SCENE + """
omni_light
{
	name		bulb
	power		2.5
	position	0.1 0.2 0.3
	color		1.0 0.5 0.25
	shootphotons	FALSE
}
"""
    s = scenefile.load_scene(text=text)
    assert s.desc.point_lights == [((0.1, 0.2, 0.3), (1.0, 0.5, 0.25), 2.5)]


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference scenes not present")
def test_reference_pointlight_cornell_loads():
    p = os.path.join(REF, "scenes", "Tests", "Spectral", "cornellbox_pointlight_spectral.RISEscene")
    s = scenefile.load_scene(p, search=[REF])
    assert len(s.desc.point_lights) == 1 and s.desc.n_tri > 0


def test_written_scene_keeps_the_depth_semantics(tmp_path):
    """A scene description written in the reference's scene language
    (oracle/scene_writer.py, the input of the reference-renderer fixtures)
    reads back with the same depth settings: the reference's file format has
    no total path cap (its rasterizer caps paths at 128 vertices) and takes
    max depth N as per-type bounce limits of N - 1, which is how
    scenes.spheres_scene() sets its own; materials and the sky read back
    too."""
    from oracle.scene_writer import write_risescene
    d = scenes.spheres_scene(grid=8, n_spheres=2, sphere_tris=80, width=16, height=12, max_depth=10)
    st = d.settings
    assert (st.max_depth, st.max_diffuse_bounce, st.max_glossy_bounce, st.max_transmission_bounce) == (128, 9, 9, 9)
    back = scenefile.load_scene(write_risescene(d, str(tmp_path), "s"))
    bs = back.desc.settings
    assert (bs.max_depth, bs.max_diffuse_bounce, bs.max_glossy_bounce, bs.max_transmission_bounce) == (128, 9, 9, 9)
    assert (bs.width, bs.height) == (16, 12)
    assert [m.type for m in back.desc.materials if m.emission < 0] == [m.type for m in d.materials if m.emission < 0]
    assert back.desc.n_tri == d.n_tri and back.desc.env >= 0
