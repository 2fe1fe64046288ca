"""The path-tracing oracle against the reference renderer itself (CPU).

The reference fixtures (tests/golden/cornell_c1_ref_k16.npz: per-pixel mean
and variance of XYZ over 16 independent batches of 16 samples per pixel;
generator tests/golden/make_cornell_reference.py) come from the reference
renderer's own integrator (oracle/_ref/librise_ref.so, built from its
sources) on the C1 Cornell box scene tests/golden/cornell_c1.RISEscene, which
this package's scene ingest reads too.  The oracle restates the device path
tracer in FP64 with the same Sobol sampler, so holding it to the reference
here pins the restatement that the GPU tests compare against sample by
sample.
"""
import dataclasses
import os

import numpy as np
import pytest

import oracle
from rise_b200 import scenefile
from parity import Z_ALLOWED_RATE, Z_LIMIT, rel_mse, z_scores

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SCENE = os.path.join(GOLDEN, "cornell_c1.RISEscene")
ROWS = (96, 160)   # 64 rows x 256 columns keeps the CPU test short


def ref_k16(independent=False):
    f = np.load(os.path.join(GOLDEN, "cornell_c1_ref_k16_independent.npz" if independent else "cornell_c1_ref_k16.npz"))
    return f["mean"].astype(np.float64), f["var"].astype(np.float64), int(f["k"]), int(f["spp"])


# The reference's padded Sobol sampler makes its images about 0.1-0.3 %
# brighter than the same integrator given independent numbers (measured with
# the harness's IndependentSampler switch); the restatement's own Sobol draws
# land about 0.2 % below its hash-sampler images.  Image means against the
# Sobol fixture are therefore held to 0.5 %, against the independent-sampler
# fixture to the statistics alone.
SOBOL_MEAN_TOL = 5e-3


def test_scene_ingest_reads_the_reference_settings():
    ls = scenefile.load_scene(SCENE)
    st = ls.desc.settings
    assert (st.width, st.height, ls.spp) == (256, 256, 16)
    assert st.sampler == 2 and st.max_diffuse_bounce == 7 and st.rr_min_depth == 3
    assert (st.lambda_min, st.lambda_max) == (400.0, 700.0) and st.filter == 0
    assert ls.desc.n_tri == 32


@pytest.mark.parametrize("sampler", [0, 1, 2], ids=["hash_vs_independent", "sobol_vs_sobol", "shuffled_vs_independent"])
def test_oracle_matches_reference_renderer_z_test(sampler):
    """16 batches of 16 spp of the restatement against the reference's 16:
    the hash sampler and the shuffled Sobol sampler against the reference
    with independent numbers, the reference's Sobol sampler against the
    reference's own."""
    mr, vr, k, spp = ref_k16(independent=sampler != 1)
    ls = scenefile.load_scene(SCENE)
    st = ls.desc.settings
    y0, y1 = ROWS
    crop = (0, y0, st.width, y1)
    g = np.array([oracle.pt_render(ls.desc, spp, crop=crop,
                                   settings=dataclasses.replace(st, seed=500 + b, sampler=sampler))
                  for b in range(k)])
    z, _ = z_scores(g.mean(0), g.var(0, ddof=1), k, mr[y0:y1], vr[y0:y1], k)
    assert (np.abs(z) > Z_LIMIT).mean() <= Z_ALLOWED_RATE, (np.abs(z) > Z_LIMIT).mean()
    # Image mean: within 4 standard errors of the batch-to-batch spread.
    se = np.sqrt(g[..., 1].mean(axis=(1, 2)).var(ddof=1) / k + vr[y0:y1, :, 1].mean() / k / g[0, ..., 1].size)
    tol = 4 * se + (SOBOL_MEAN_TOL * mr[y0:y1, :, 1].mean() if sampler == 1 else 0.0)
    assert abs(g[..., 1].mean() - mr[y0:y1, :, 1].mean()) < tol


def test_harness_pixel_loop_matches_the_reference_pipeline():
    """The fixtures come from the reference's per-sample function under a
    box-filter pixel loop restated in the harness; the reference's own
    Job::Rasterize of the same scene must give the same picture: image means
    within 1 %, and its relMSE against the 256-spp fixture (converted to
    Rec.709 like the reference's film) at the level of one 16-spp batch."""
    if oracle.rise_ref() is None:
        pytest.skip("oracle/_ref/librise_ref.so not built (no reference tree)")
    mr, vr, k, spp = ref_k16()
    lib = oracle.port_blocks()
    to_rgb = lambda xyz: oracle.xyz_to_rec709(lib, "orc_pt_", xyz.reshape(-1, 3)).reshape(xyz.shape)
    r = oracle.RefRenderer(SCENE)
    try:
        full = r.render()
        one = r.integrate(spp, batch=99)
    finally:
        r.close()
    ref_rgb = to_rgb(mr)
    assert abs(full.mean() / ref_rgb.mean() - 1) < 0.01
    e_full, e_one = rel_mse(full, ref_rgb), rel_mse(to_rgb(one), ref_rgb)
    assert 0.6 < e_full / e_one < 1.6, (e_full, e_one)


def test_smooth_shading_normals_match_the_reference():
    """Interpolated vertex normals (a smooth Lambertian sphere and a smooth
    glass sphere read from RAW2 files): the restatement's 16 batches against
    the reference's 16 (independent numbers) on the rows through both
    spheres; the same scene shaded with face normals fails the same test."""
    f = np.load(os.path.join(GOLDEN, "cornell_smooth_ref_k16_independent.npz"))
    mr, vr, k, spp = f["mean"].astype(np.float64), f["var"].astype(np.float64), int(f["k"]), int(f["spp"])
    ls = scenefile.load_scene(os.path.join(GOLDEN, "cornell_smooth.RISEscene"))
    st = ls.desc.settings
    assert sum(n is not None for n in ls.desc._nrms) == 2
    y0, y1 = 128, 192
    crop = (0, y0, st.width, y1)

    def rate(desc):
        g = np.array([oracle.pt_render(desc, spp, crop=crop, settings=dataclasses.replace(st, seed=700 + b, sampler=0))
                      for b in range(k)])
        z, _ = z_scores(g.mean(0), g.var(0, ddof=1), k, mr[y0:y1], vr[y0:y1], k)
        return float((np.abs(z) > Z_LIMIT).mean())

    assert rate(ls.desc) <= Z_ALLOWED_RATE
    flat = dataclasses.replace(ls.desc)
    flat._nrms = [None] * len(ls.desc._nrms)
    assert rate(flat) > 2 * Z_ALLOWED_RATE


def _variant(name):
    f = np.load(os.path.join(GOLDEN, name + "_ref_k16_independent.npz"))
    ls = scenefile.load_scene(os.path.join(GOLDEN, name + ".RISEscene"))
    return ls, f["mean"].astype(np.float64), f["var"].astype(np.float64), int(f["k"]), int(f["spp"])


def _z_rate(desc, st, mr, vr, k, spp, rows, seed0):
    y0, y1 = rows
    g = np.array([oracle.pt_render(desc, spp, crop=(0, y0, st.width, y1),
                                   settings=dataclasses.replace(st, seed=seed0 + b, sampler=0))
                  for b in range(k)])
    z, _ = z_scores(g.mean(0), g.var(0, ddof=1), k, mr[y0:y1], vr[y0:y1], k)
    return float((np.abs(z) > Z_LIMIT).mean()), g


def test_single_wavelength_mode_matches_the_reference():
    """`hwss false` (the reference's default): one wavelength per path from
    10 bins of 30 nm (IntegrateRayNM).  The restatement's 16 batches against
    the reference's 16; the same scene rendered with continuous hero bundles
    fails the test (the bins shift Z by about 3 %)."""
    ls, mr, vr, k, spp = _variant("cornell_nm")
    st = ls.desc.settings
    assert (st.spectral_mode, st.num_wavelengths, st.spectral_samples) == (1, 10, 1)
    rate, g = _z_rate(ls.desc, st, mr, vr, k, spp, ROWS, 900)
    assert rate <= Z_ALLOWED_RATE, rate
    y0, y1 = ROWS
    se = np.sqrt(g[..., 2].mean(axis=(1, 2)).var(ddof=1) / k + vr[y0:y1, :, 2].mean() / k / g[0, ..., 2].size)
    assert abs(g[..., 2].mean() - mr[y0:y1, :, 2].mean()) < 4 * se
    hwss = dataclasses.replace(st, spectral_mode=0)
    assert _z_rate(ls.desc, hwss, mr, vr, k, spp, ROWS, 900)[0] > 2 * Z_ALLOWED_RATE


@pytest.mark.parametrize("name", ["cornell_prism", "cornell_prism_nm"])
def test_dispersive_glass_matches_the_reference(name):
    """A glass prism whose index runs from 2.0 (450 nm) to 1.3 (650 nm):
    under hero bundles the companions end at the prism and the hero goes on
    alone; one wavelength per path (30 bins, two spectral samples per pixel
    sample) refracts each at its own index.  The restatement against the
    reference (16 batches of 64 samples per pixel: the caustics make single
    samples heavy-tailed) on the rows through the prism; the prism read with
    a constant index of 1.5 fails the same test."""
    ls, mr, vr, k, spp = _variant(name)
    st = ls.desc.settings
    glass = [m for m in ls.desc.materials if m.type == 2]
    assert len(glass) == 1 and glass[0].eta >= 0
    rows = (192, 224)   # the prism's lower half and the floor in front of it
    rate, _ = _z_rate(ls.desc, st, mr, vr, k, spp, rows, 1100)
    assert rate <= Z_ALLOWED_RATE, rate
    const = dataclasses.replace(ls.desc)
    const.materials = [dataclasses.replace(m, eta=-1, ior=1.5) if m.type == 2 else m for m in ls.desc.materials]
    assert _z_rate(const, st, mr, vr, k, spp, rows, 1100)[0] > 2 * Z_ALLOWED_RATE


def test_overlapping_media_match_the_reference():
    """Two overlapping glass spheres (indices 1.5 and 1.33) and a GGX
    conductor cutting into the first: the reference keeps an index-of-
    refraction stack per path (IORStack.h), so a ray crossing from the first
    sphere into the second refracts from 1.5 to 1.33, leaves the first for
    the second's 1.33, and the conductor's Fresnel inside the glass takes 1.5
    as its incident index.  The restatement's 16 batches against the
    reference's 16 on the rows through the overlaps."""
    ls, mr, vr, k, spp = _variant("cornell_overlap")
    st = ls.desc.settings
    assert sorted(m.ior for m in ls.desc.materials if m.type == 2) == [1.33, 1.5]
    rows = (160, 192)
    rate, g = _z_rate(ls.desc, st, mr, vr, k, spp, rows, 1500)
    assert rate <= Z_ALLOWED_RATE, rate
    y0, y1 = rows
    for c in range(3):
        se = np.sqrt(g[..., c].mean(axis=(1, 2)).var(ddof=1) / k + vr[y0:y1, :, c].mean() / k / g[0, ..., c].size)
        assert abs(g[..., c].mean() - mr[y0:y1, :, c].mean()) < 4 * se, c


def test_double_sided_glass_matches_the_reference():
    """A glass sphere on a double-sided mesh: the reference turns both of its
    normals towards the ray (TriangleMeshGeometry.cpp:94-120) while the
    dielectric reads inside / outside from the index-of-refraction stack, so
    from inside the refracted ray fails the crossing test and only total
    internal reflection goes on (DielectricSPF.cpp:177-279).  The
    restatement's 16 batches against the reference's 16 on the rows through
    the sphere; the same sphere read as single-sided fails the test."""
    ls, mr, vr, k, spp = _variant("cornell_dsglass")
    st = ls.desc.settings
    glass = [i for i, (_, _, mat, ds) in enumerate(ls.desc.meshes) if ls.desc.materials[mat].type == 2]
    assert len(glass) == 1 and ls.desc.meshes[glass[0]][3] == 1
    rows = (176, 208)
    rate, _ = _z_rate(ls.desc, st, mr, vr, k, spp, rows, 1700)
    assert rate <= Z_ALLOWED_RATE, rate
    single = dataclasses.replace(ls.desc)
    single.meshes = [(f, c, m, 0 if i == glass[0] else ds) for i, (f, c, m, ds) in enumerate(ls.desc.meshes)]
    assert _z_rate(single, st, mr, vr, k, spp, rows, 1700)[0] > 2 * Z_ALLOWED_RATE


def test_image_environment_matches_the_reference():
    """A scene lit only by an HDR light probe: the angular mapping after a
    30-degree turn about y, bilinear texels, the unbounded spectral uplift per
    lookup, radiance scale 1.5, next events from the 64 x 64 importance
    tables with power-heuristic MIS.  The restatement's 16 batches against
    the reference's 16; the probe left unturned fails the same test."""
    ls, mr, vr, k, spp = _variant("cornell_env")
    st = ls.desc.settings
    em = ls.desc.env_map
    assert em is not None and em.orient_deg == (0.0, 30.0, 0.0) and em.scale == 1.5
    rows = (0, st.height)
    rate, g = _z_rate(ls.desc, st, mr, vr, k, spp, rows, 1300)
    assert rate <= Z_ALLOWED_RATE, rate
    for c in range(3):
        se = np.sqrt(g[..., c].mean(axis=(1, 2)).var(ddof=1) / k + vr[..., c].mean() / k / g[0, ..., c].size)
        assert abs(g[..., c].mean() - mr[..., c].mean()) < 4 * se, c
    plain = dataclasses.replace(ls.desc, env_map=dataclasses.replace(em, orient_deg=(0.0, 0.0, 0.0)))
    assert _z_rate(plain, st, mr, vr, k, spp, rows, 1300)[0] > 2 * Z_ALLOWED_RATE


def test_hdr_reader_decodes_rgbe_as_the_reference(tmp_path):
    """The probe file through rtb200_hdr_decode against a direct decode of
    its run-length RGBE bytes: value = 2^(e - 136) (byte + 1/2), 0 for e = 0
    (HDRReader::ReadColor); a truncated file is refused."""
    path = os.path.join(GOLDEN, "cornell_env_probe.hdr")
    img = scenefile.read_hdr(path)
    data = open(path, "rb").read()
    head = data.index(b"-Y ")
    line_end = data.index(b"\n", head)
    h, w = int(data[head:line_end].split()[1]), int(data[head:line_end].split()[3])
    assert img.shape == (h, w, 3)
    pos = line_end + 1
    px = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        assert data[pos:pos + 2] == b"\x02\x02"
        pos += 4
        for comp in range(4):
            x = 0
            while x < w:
                n = data[pos]
                pos += 1
                if n > 128:
                    px[y, x:x + n - 128, comp] = data[pos]
                    pos += 1
                    x += n - 128
                else:
                    px[y, x:x + n, comp] = np.frombuffer(data[pos:pos + n], np.uint8)
                    pos += n
                    x += n
    e = px[..., 3].astype(np.int32)
    want = np.where(e[..., None] == 0, 0.0, np.ldexp(1.0, e[..., None] - 136) * (px[..., :3] + 0.5))
    assert np.array_equal(img, want.astype(np.float32))
    bad = tmp_path / "truncated.hdr"
    bad.write_bytes(data[:len(data) // 2])
    with pytest.raises(scenefile.SceneFileError):
        scenefile.read_hdr(str(bad))
