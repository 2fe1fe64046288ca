"""The path-tracing oracle's building blocks against the reference's own code.

Each function the oracle restates (wavelength sampling, CIE lookup, GGX terms,
visible-normal sampling, Fresnel, the energy-table lookups and the
multiple-scattering lobe sampler, Russian roulette, MIS) is checked on the
committed golden cases from the reference (tests/golden/pt_blocks.json, made
by tests/golden/make_pt_golden.py) and, where oracle/_ref/libref_pt.so was
built from the reference tree, on thousands of random inputs.

Tolerances: 1e-12 relative for closed-form double arithmetic; 1e-9 where the
oracle uses an algebraically equal but differently rounded form (isotropic
vs anisotropic GGX terms).  The energy tables themselves are computed by the
oracle (deterministic quadrature of the reference's estimator) and must match
the reference's Monte Carlo table within its sampling noise; the lookups and
the sampler are checked bit-for-bit on the reference's table values.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle

# The reference's tabulated 21-point Gauss-Legendre weights
# (MicrofacetEnergyLUT.h:370-378) sum to 1 + 7.4e-8; the oracle computes the
# exact nodes and weights, so Fresnel averages agree to ~1e-7 relative.
FAVG_REL = 2e-7
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pt_blocks.json")))
F64P = ctypes.POINTER(ctypes.c_double)


def p64(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(F64P)


@pytest.fixture(scope="module")
def port():
    return oracle.port_blocks()


@pytest.fixture
def ref_tables(port):
    """Swap the reference's E_ss / E_avg values into the oracle for one test."""
    own = oracle.energy_tables(port, "orc_pt_")
    t = GOLDEN["energy_tables"]
    ess, pe = p64(np.array(t["ess"]).ravel())
    eavg, pa = p64(np.array(t["eavg"]))
    port.orc_pt_set_tables(pe, pa)
    yield
    ess, pe = p64(own[0].ravel())
    eavg, pa = p64(own[1])
    port.orc_pt_set_tables(pe, pa)


def close(a, b, rel=1e-12, abs_=1e-300):
    return abs(a - b) <= max(abs_, rel * max(abs(a), abs(b)))


# ---- golden cases (always) ---------------------------------------------------

def test_golden_wavelengths(port):
    for u, lo, hi, want in GOLDEN["sample_wavelengths"]:
        lam, p = p64(np.zeros(4))
        port.orc_pt_sample_wavelengths(u, lo, hi, p)
        assert np.allclose(lam, want, rtol=1e-14, atol=0), (u, lo, hi)


def test_golden_cie(port):
    cie, pc = p64(oracle.cie_table().ravel())
    for nm, ok, want in GOLDEN["xyz_from_nm"]:
        xyz, p = p64(np.zeros(3))
        assert port.orc_pt_xyz_from_nm(nm, pc, p) == ok
        assert np.allclose(xyz, want, rtol=1e-14, atol=1e-300), nm
    y = oracle.cie_table()[1]
    for a, b, want in GOLDEN["cie_y_integral"]:
        lo, hi = max(a, 380.0), min(b, 780.0)
        i0, i1 = int((lo - 380) / 5), int((hi - 380) / 5)
        got = sum(0.5 * (y[i] + y[i + 1]) * 5.0 for i in range(i0, i1)) if hi > lo else 0.0
        assert close(got, want, 1e-13), (a, b)


@pytest.mark.parametrize("name", ["ggx_d", "ggx_lambda"])
def test_golden_ggx_terms(port, name):
    f = getattr(port, "orc_pt_" + name)
    for a, c, want in GOLDEN[name]:
        assert close(f(a, c), want, 1e-12), (a, c)


def test_golden_g2_vndf(port):
    for a, ci, co, want in GOLDEN["ggx_g2"]:
        assert close(port.orc_pt_ggx_g2(a, ci, co), want, 1e-12)
    for wi, n, a, u1, u2, want, onb in GOLDEN["vndf_sample"]:
        m, pm = p64(np.zeros(3))
        port.orc_pt_vndf_sample(p64(wi)[1], p64(onb[0:3])[1], p64(onb[3:6])[1], p64(onb[6:9])[1], a, u1, u2, pm)
        assert np.allclose(m, want, rtol=0, atol=1e-12)
    for wi, wo, n, a, want in GOLDEN["vndf_pdf"]:
        assert close(port.orc_pt_vndf_pdf(p64(wi)[1], p64(wo)[1], p64(n)[1], a), want, 1e-9)


def test_golden_fresnel(port):
    for v, n, ni, nt, k, want in GOLDEN["conductor_f"]:
        assert close(port.orc_pt_conductor_f(float(np.dot(v, n)), ni, nt, k), want, 1e-12)
    for ci, ct, ni, nt, want in GOLDEN["dielectric_r"]:
        assert close(port.orc_pt_dielectric_r(ci, ct, ni, nt), want, 1e-12)
    for ni, nt, k, want in GOLDEN["fresnel_avg"]:
        assert close(port.orc_pt_fresnel_avg(ni, nt, k), want, FAVG_REL)
    for f, e, want in GOLDEN["fms"]:
        assert close(port.orc_pt_fms(f, e), want, 1e-15)


def test_golden_mis_and_roulette(port):
    for a, b, want in GOLDEN["power_heuristic"]:
        assert port.orc_pt_power_heuristic(a, b) == want
    for depth, mind, thr, cur, prev, u, term, surv in GOLDEN["russian_roulette"]:
        s = ctypes.c_double()
        assert port.orc_pt_russian_roulette(depth, mind, thr, cur, prev, u, ctypes.byref(s)) == term
        if not term:
            assert s.value == surv


def test_golden_colour_resolve_and_display(port):
    """XYZ -> linear Rec.709 with the gamut move, and the 8-bit encode with
    exposure and each tone curve: bit-exact against the reference."""
    for xyz, want in GOLDEN["xyz_to_rec709"]:
        got = oracle.xyz_to_rec709(port, "orc_pt_", np.array(xyz))
        assert np.array_equal(got, np.array(want)), (xyz, got, want)
    for rgb, ev, tone, want in GOLDEN["display"]:
        got = oracle.display8(port, "orc_pt_", np.array(rgb), ev, tone)
        assert got.tolist() == want, (rgb, ev, tone, got, want)


def test_golden_sobol_and_hash_combine():
    # The reference's padded Owen-scrambled Sobol and its pixel-seed hash
    # (Sampling/SobolSequence.h:55-206), bit for bit.
    g = np.array(GOLDEN["sobol"], np.uint64)
    got = oracle.sobol(g[:, 0].astype(np.uint32), g[:, 1].astype(np.uint32), g[:, 2].astype(np.uint32))
    assert np.array_equal(got.astype(np.uint64), g[:, 3])
    h = np.array(GOLDEN["hash_combine"], np.uint64)
    assert np.array_equal(oracle.hash_combine(h[:, 0].astype(np.uint32), h[:, 1].astype(np.uint32)).astype(np.uint64),
                          h[:, 2])


def test_golden_gaussian_filter(port):
    for size, sigma, dx, dy, want in GOLDEN["gaussian_filter"]:
        assert close(port.orc_pt_gaussian_weight(size, sigma, dx, dy), want, 1e-14), (size, sigma, dx, dy)


def test_energy_tables_match_reference_within_its_noise(port):
    ess, eavg = oracle.energy_tables(port, "orc_pt_")
    ref = np.array(GOLDEN["energy_tables"]["ess"])
    d = np.abs(ess - ref)
    assert d.max() < 3e-3 and np.sqrt((d ** 2).mean()) < 1e-3, (d.max(), np.sqrt((d ** 2).mean()))
    assert np.abs(eavg - np.array(GOLDEN["energy_tables"]["eavg"])).max() < 2e-3


def test_golden_lut_lookups_and_ms_sampler(port, ref_tables):
    for c, a, want in GOLDEN["lookup_ess"]:
        assert close(port.orc_pt_lookup_ess(c, a), want, 1e-7), (c, a)   # table stored to 8 decimals
    for a, want in GOLDEN["lookup_eavg"]:
        assert close(port.orc_pt_lookup_eavg(a), want, 1e-7)
    for a, want in GOLDEN["ms_z"]:
        assert close(port.orc_pt_ms_z(a), want, 1e-6)
    for c, a, want in GOLDEN["ms_pdf"]:
        assert close(port.orc_pt_ms_pdf(c, a, port.orc_pt_ms_z(a)), want, 1e-6, 1e-300)
    for a, u, want in GOLDEN["ms_sample_cos"]:
        assert abs(port.orc_pt_ms_sample_cos(a, u) - want) < 1e-6, (a, u)


# ---- random inputs against the live reference (where built) ------------------

@pytest.fixture(scope="module")
def ref():
    r = oracle.ref_blocks()
    if r is None:
        pytest.skip("oracle/_ref/libref_pt.so not built (no reference tree)")
    return r


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_random_wavelengths_and_cie(port, ref):
    rng = np.random.default_rng(1)
    cie, pc = p64(oracle.cie_table().ravel())
    for u, lo, w in zip(rng.random(2000), rng.uniform(360, 500, 2000), rng.uniform(50, 400, 2000)):
        a, pa = p64(np.zeros(4))
        b, pb = p64(np.zeros(4))
        port.orc_pt_sample_wavelengths(u, lo, lo + w, pa)
        ref.ref_pt_sample_wavelengths(u, lo, lo + w, pb)
        assert np.array_equal(a, b)
    for nm in rng.uniform(370, 790, 5000):
        a, pa = p64(np.zeros(3))
        b, pb = p64(np.zeros(3))
        assert port.orc_pt_xyz_from_nm(nm, pc, pa) == ref.ref_pt_xyz_from_nm(nm, pb)
        assert np.allclose(a, b, rtol=1e-14, atol=1e-300)


def test_random_ggx(port, ref):
    rng = np.random.default_rng(2)
    for a, c1, c2 in zip(rng.uniform(1e-4, 1, 5000), rng.random(5000), rng.random(5000)):
        assert close(port.orc_pt_ggx_d(a, c1), ref.ref_pt_ggx_d(a, c1), 1e-12)
        assert close(port.orc_pt_ggx_lambda(a, c1), ref.ref_pt_ggx_lambda(a, c1), 1e-12)
        assert close(port.orc_pt_ggx_g2(a, c1, c2), ref.ref_pt_ggx_g2(a, c1, c2), 1e-12)
    ns = unit(rng, 3000)
    for n in ns:
        wi = unit(rng, 1)[0]
        wi = wi if wi @ n > 0 else -wi
        wo = unit(rng, 1)[0]
        wo = wo if wo @ n > 0 else -wo
        a, u1, u2 = rng.uniform(0.01, 1.0), rng.random(), rng.random()
        m, pm = p64(np.zeros(3))
        onb, po = p64(np.zeros(9))
        ref.ref_pt_vndf_sample(p64(wi)[1], p64(n)[1], a, u1, u2, pm, po)
        m2, pm2 = p64(np.zeros(3))
        port.orc_pt_vndf_sample(p64(wi)[1], p64(onb[0:3])[1], p64(onb[3:6])[1], p64(onb[6:9])[1], a, u1, u2, pm2)
        assert np.allclose(m, m2, rtol=0, atol=1e-12)
        assert close(port.orc_pt_vndf_pdf(p64(wi)[1], p64(wo)[1], p64(n)[1], a),
                     ref.ref_pt_vndf_pdf(p64(wi)[1], p64(wo)[1], p64(n)[1], a), 1e-9, 1e-300)


def test_random_fresnel(port, ref):
    rng = np.random.default_rng(3)
    for _ in range(3000):
        n = unit(rng, 1)[0]
        v = unit(rng, 1)[0]
        nt, k = rng.uniform(0.1, 4), rng.uniform(0, 6)
        assert close(port.orc_pt_conductor_f(float(v @ n), 1.0, nt, k),
                     ref.ref_pt_conductor_f(p64(v)[1], p64(n)[1], 1.0, nt, k), 1e-12)
    for ci, ni, nt in zip(rng.uniform(0.001, 1, 3000), rng.uniform(1, 2, 3000), rng.uniform(1, 2, 3000)):
        s2 = (ni / nt) ** 2 * (1 - ci * ci)
        if s2 >= 1:
            continue
        ct = np.sqrt(1 - s2)
        v = np.array([np.sqrt(1 - ci * ci), 0, -ci])
        tv = np.array([np.sqrt(s2), 0, -ct])
        assert close(port.orc_pt_dielectric_r(ci, ct, ni, nt),
                     ref.ref_pt_dielectric_r(p64(v)[1], p64(tv)[1], p64([0, 0, 1.0])[1], ni, nt), 1e-12)
    for nt, k in zip(rng.uniform(0.1, 4, 500), rng.uniform(0, 6, 500)):
        assert close(port.orc_pt_fresnel_avg(1.0, nt, k), ref.ref_pt_fresnel_avg(1.0, nt, k), FAVG_REL)


def test_random_lut_and_ms_sampler_on_reference_tables(port, ref, ref_tables):
    rng = np.random.default_rng(4)
    ess, pe = p64(np.zeros(1024))
    eavg, pa = p64(np.zeros(32))
    ref.ref_pt_tables(pe, pa)
    port.orc_pt_set_tables(pe, pa)     # exact reference values (the fixture restores ours)
    for c, a in zip(rng.uniform(-0.1, 1.1, 5000), rng.uniform(0, 1.2, 5000)):
        assert port.orc_pt_lookup_ess(c, a) == ref.ref_pt_lookup_ess(c, a)
        assert port.orc_pt_lookup_eavg(a) == ref.ref_pt_lookup_eavg(a)
        z = ref.ref_pt_ms_z(a)
        assert close(port.orc_pt_ms_z(a), z, 1e-13)
        assert close(port.orc_pt_ms_pdf(c, a, z), ref.ref_pt_ms_pdf(c, a, z), 1e-13, 1e-300)
    for a, u in zip(rng.uniform(0.01, 1, 3000), rng.random(3000)):
        assert abs(port.orc_pt_ms_sample_cos(a, u) - ref.ref_pt_ms_sample_cos(a, u)) < 1e-12


def test_ms_sampler_matches_its_pdf(port):
    # The sampled mu_o histogram follows MSPdf(mu) * 2 pi (solid angle -> mu).
    rng = np.random.default_rng(5)
    for a in (0.05, 0.3, 0.9):
        mus = np.array([port.orc_pt_ms_sample_cos(a, u) for u in rng.random(40000)])
        z = port.orc_pt_ms_z(a)
        edges = np.linspace(0, 1, 21)
        hist, _ = np.histogram(mus, edges)
        mid = 0.5 * (edges[1:] + edges[:-1])
        dens = np.array([port.orc_pt_ms_pdf(m, a, z) for m in mid]) * 2 * np.pi / 20
        assert np.allclose(hist / len(mus), dens, atol=0.004), a


def test_random_roulette_and_mis(port, ref):
    rng = np.random.default_rng(6)
    s1, s2 = ctypes.c_double(), ctypes.c_double()
    for _ in range(5000):
        d, m = int(rng.integers(0, 8)), int(rng.integers(0, 5))
        thr, cur, prev, u = rng.uniform(0, 0.2), rng.exponential(0.5), rng.exponential(0.5), rng.random()
        t1 = port.orc_pt_russian_roulette(d, m, thr, cur, prev, u, ctypes.byref(s1))
        t2 = ref.ref_pt_russian_roulette(d, m, thr, cur, prev, u, ctypes.byref(s2))
        assert t1 == t2 and (t1 or s1.value == s2.value)
        a, b = rng.exponential(1, 2)
        assert port.orc_pt_power_heuristic(a, b) == ref.ref_pt_power_heuristic(a, b)


def test_random_sobol_and_hash_combine(ref):
    rng = np.random.default_rng(5)
    n = 200000
    idx = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    dim = rng.integers(0, 4096, n).astype(np.uint32)
    seed = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(oracle.sobol(idx, dim, seed).astype(np.float64) / 4294967296.0,
                          oracle.sobol(idx, dim, seed, "ref"))
    assert np.array_equal(oracle.hash_combine(idx, seed), oracle.hash_combine(idx, seed, "ref"))


def test_random_gaussian_filter(port, ref):
    rng = np.random.default_rng(8)
    for _ in range(2000):
        size, sigma = rng.uniform(0.5, 6.0), rng.uniform(0.1, 2.0)
        dx, dy = rng.uniform(-0.6, 0.6, 2) * size
        a = port.orc_pt_gaussian_weight(size, sigma, dx, dy)
        b = ref.ref_pt_gaussian_weight(size, sigma, dx, dy)
        assert close(a, b, 1e-14), (size, sigma, dx, dy, a, b)


def _gaussian(desc, size, sigma):
    from rise_b200 import scenes
    desc.settings = scenes.RenderSettings(**{**desc.settings.__dict__, "filter": 1, "filter_size": size,
                                             "filter_sigma": sigma})
    return desc


def test_filtered_render_crop_equals_full_image():
    """The splatting oracle renders the samples of the pixels around a crop,
    so a crop equals the same pixels of the full image."""
    from rise_b200 import scenes
    d = _gaussian(scenes.cornell_box(32, 32), 3.0, 0.8)
    full = oracle.pt_render(d, 4)
    crop = oracle.pt_render(d, 4, crop=(0, 8, 12, 20))
    assert np.allclose(crop, full[8:20, 0:12], rtol=1e-12, atol=1e-300)
    box = oracle.pt_render(scenes.cornell_box(32, 32), 4)
    assert np.isfinite(full).all() and not np.allclose(full, box)


def test_narrow_gaussian_warps_camera_samples():
    """A Gaussian of half-width <= 0.501 pixel moves the camera samples (a
    different image from the box film's) and keeps a per-pixel mean (a crop
    equals the full image exactly)."""
    from rise_b200 import scenes
    d = _gaussian(scenes.cornell_box(32, 32), 1.0, 0.3)
    full = oracle.pt_render(d, 4)
    crop = oracle.pt_render(d, 4, crop=(4, 4, 20, 12))
    assert np.array_equal(crop, full[4:12, 4:20])
    box = oracle.pt_render(scenes.cornell_box(32, 32), 4)
    assert np.isfinite(full).all() and not np.allclose(full, box)
    assert abs(full[..., 1].mean() / box[..., 1].mean() - 1) < 0.1


def _adaptive(desc, max_spp, threshold):
    from rise_b200 import scenes
    desc.settings = scenes.RenderSettings(**{**desc.settings.__dict__, "adaptive_max_spp": max_spp,
                                             "adaptive_threshold": threshold})
    return desc


def test_adaptive_sampling_follows_the_reference_rule():
    """Each pixel's sample count equals a direct restatement of the
    reference's loop (PathTracingSpectralRasterizer.cpp:379-408) run on the
    pixel's own per-sample luminances, and its value is the mean of those
    samples."""
    from rise_b200 import scenes
    d = _adaptive(scenes.cornell_box(24, 24), 128, 0.2)
    img, counts = oracle.pt_render(d, 8, return_counts=True)
    assert ((counts % 8 == 0) | (counts == 128)).all()
    assert (counts < 128).mean() > 0.2 and (counts == 128).mean() > 0.05, np.bincount(counts.ravel())
    plain = scenes.cornell_box(24, 24)
    for (x, y) in [(3, 3), (12, 12), (20, 5), (5, 20), (12, 2), (23, 23)]:
        ys, acc = [], np.zeros(3)
        mean = m2 = 0.0
        n = 0
        idx = 0
        converged = False
        while idx < 128 and not converged:
            for s in range(idx, min(idx + 8, 128)):
                v = oracle.pt_render(plain, 1, sample_begin=s, crop=(x, y, x + 1, y + 1), threads=1)[0, 0]
                acc += v
                n += 1
                delta = v[1] - mean
                mean += delta / n
                m2 += delta * (v[1] - mean)
            idx = min(idx + 8, 128)
            if n >= 32:
                se = np.sqrt(m2 / (n - 1) / n)
                if abs(mean) > 1e-12:
                    converged = se / abs(mean) < 0.2 * (1 - 4 / n)
                else:
                    converged = m2 < 1e-12 and n >= 64
        assert counts[y, x] == idx, (x, y, counts[y, x], idx)
        assert np.allclose(img[y, x], acc / idx, rtol=1e-12, atol=1e-300)


def test_random_colour_resolve_and_display(port, ref):
    rng = np.random.default_rng(9)
    x = np.concatenate([rng.exponential(1.0, (4000, 3)),
                        rng.exponential(1.0, (1000, 1)) * np.array([[1.0, 0.02, 0.01]]),
                        rng.exponential(1.0, (1000, 1)) * np.array([[0.01, 1.0, 0.03]]),
                        rng.exponential(1.0, (1000, 1)) * np.array([[0.2, 0.05, 1.0]]),
                        rng.normal(size=(500, 3)), np.zeros((2, 3))])
    a = oracle.xyz_to_rec709(port, "orc_pt_", x)
    b = oracle.xyz_to_rec709(ref, "ref_pt_", x)
    assert np.array_equal(a, b, equal_nan=True)
    for tone in range(5):
        ev = float(rng.uniform(-3, 3))
        assert np.array_equal(oracle.display8(port, "orc_pt_", b[:2000], ev, tone),
                              oracle.display8(ref, "ref_pt_", b[:2000], ev, tone)), tone


def test_golden_spectral_painter_packets():
    """spectral_painter's binned spectrum (piecewise-linear control points
    sampled into n bins, step lookup, 0 outside) against the reference's
    PiecewiseLinearFunction1D + SpectralPacket; amplitudes are stored as
    FP32."""
    from rise_b200 import scenes
    for nm, amp, lo, hi, q, want in GOLDEN["spectral_packet"]:
        got = scenes.spectral_painter(nm, amp, lo, hi).value_at(np.array(q))
        assert np.allclose(got, want, rtol=1e-7, atol=0), (nm, lo, hi)


def test_random_spectral_painter_packets(ref):
    from rise_b200 import scenes
    rng = np.random.default_rng(10)
    for _ in range(200):
        n = int(rng.integers(1, 40))
        nm = rng.uniform(360, 800, n)
        amp = rng.exponential(1.0, n)
        lo = float(rng.uniform(360, 500))
        hi = float(lo + rng.uniform(50, 400))
        q = np.concatenate([rng.uniform(lo - 20, hi, 200), [lo]])
        q = q[q < hi]
        want = np.zeros(len(q))
        ref.ref_pt_spectral_packet(nm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   amp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, lo, hi,
                                   q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(q),
                                   want.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        got = scenes.spectral_painter(nm, amp, lo, hi).value_at(q)
        assert np.allclose(got, want, rtol=1e-7, atol=0)


def test_golden_light_bvh(port):
    """Light BVH build, stochastic pick and pdf against the reference's
    LightBVH (point lights; one set lies in a plane)."""
    for pos, power, pts, xi, picked, pdf, pdf_all in GOLDEN["light_bvh"]:
        p, d, a = oracle.light_bvh(port, "orc_pt_", pos, power, pts, xi)
        assert p.tolist() == picked
        assert np.allclose(d, pdf, rtol=1e-12, atol=0) and np.allclose(a, pdf_all, rtol=1e-12, atol=0)
        assert np.allclose(np.array(pdf_all).sum(axis=1), 1.0)


def test_random_light_bvh(port, ref):
    rng = np.random.default_rng(11)
    for n in (2, 5, 16, 100, 333):
        pos = rng.normal(size=(n, 3)) * rng.uniform(0.1, 10)
        power = rng.exponential(1.0, n) * (rng.random(n) < 0.9)
        pts = rng.normal(size=(60, 3)) * 3
        xi = rng.random(60)
        a = oracle.light_bvh(port, "orc_pt_", pos, power, pts, xi)
        b = oracle.light_bvh(ref, "ref_pt_", pos, power, pts, xi)
        assert np.array_equal(a[0], b[0])
        assert np.allclose(a[1], b[1], rtol=1e-12, atol=0) and np.allclose(a[2], b[2], rtol=1e-12, atol=0)


REF_LUT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "rec709.coeff")


def test_rgb_uplift_table_equals_the_reference_generators():
    """The library's RGB -> spectrum table, built by the reference generator's
    steps, equals the table the reference's own generator writes, bit for
    bit."""
    if not os.path.exists(REF_LUT):
        pytest.skip("reference table not generated (no reference tree)")
    from rise_b200._native import lib
    ours = np.zeros(3 * 64 ** 3 * 3, np.float32)
    lib().rtb200_rgb_uplift_table(ours.ctypes.data)
    ref = np.fromfile(REF_LUT, dtype=np.uint8)[20:].view(np.float32)
    assert np.array_equal(ours, ref)


def test_rgb_uplift_lookup_matches_reference(ref):
    """Albedo and unbounded spectra of random colours: the library's lookup
    against the reference's RGBToSpectrumTable / RGB*Spectrum on the same
    table."""
    if not os.path.exists(REF_LUT):
        pytest.skip("reference table not generated (no reference tree)")
    from rise_b200 import scenes
    table = np.ascontiguousarray(np.fromfile(REF_LUT, dtype=np.uint8)[20:].view(np.float32))
    f = ref.ref_pt_rgb_uplift
    f.restype = ctypes.c_int
    P = ctypes.c_void_p
    rng = np.random.default_rng(12)
    nm = np.linspace(370, 790, 60)
    colours = [rng.random(3) for _ in range(150)] + [rng.random(3) * rng.uniform(1, 20) for _ in range(50)] + \
        [np.array(v, np.float64) for v in ([0, 0, 0], [1, 1, 1], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0.5, 0.5])]
    for rgb in colours:
        rgb = np.ascontiguousarray(rgb, np.float64)
        for kind in (0, 1):
            coeffs, vals = np.zeros(3), np.zeros(len(nm))
            assert f(table.ctypes.data_as(P), ctypes.c_uint(table.size), rgb.ctypes.data_as(P), kind,
                     nm.ctypes.data_as(P), len(nm), coeffs.ctypes.data_as(P), vals.ctypes.data_as(P)) == 1
            s = scenes.rgb_spectrum(rgb, kind)
            if kind == 0:
                assert np.array_equal([s.c0, s.c1, s.c2], coeffs), (rgb, s, coeffs)
            assert np.allclose(s.value_at(nm), vals, rtol=1e-12, atol=1e-300), (rgb, kind)


def test_golden_rgb_uplift():
    """RGB -> spectrum of fixed colours (albedo and unbounded) against values
    from the reference's own table code and generator."""
    from rise_b200 import scenes
    for rgb, kind, coeffs, nm, vals in GOLDEN["rgb_uplift"]:
        s = scenes.rgb_spectrum(rgb, kind)
        if kind == 0:
            assert [s.c0, s.c1, s.c2] == coeffs, (rgb, kind)
        assert np.allclose(s.value_at(nm), vals, rtol=1e-12, atol=1e-300), (rgb, kind)
