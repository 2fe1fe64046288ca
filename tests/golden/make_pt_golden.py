"""Generate tests/golden/pt_blocks.json from the reference renderer's own code.

Evaluates the reference's path-tracer building blocks (compiled from its
sources into oracle/_ref/libref_pt.so by oracle/Makefile) on seeded inputs and
stores inputs and outputs, so tests/test_oracle_pt.py can hold the oracle to
the reference on machines without the reference tree.

    make -C oracle && python tests/golden/make_pt_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

F64P = ctypes.POINTER(ctypes.c_double)


def vec(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(F64P)


def hemi(rng, n):
    """Random unit vector in the hemisphere around unit n."""
    while True:
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        if v @ n > 0.05:
            return v


def main():
    r = oracle.ref_blocks()
    if r is None:
        raise SystemExit("oracle/_ref/libref_pt.so not built (needs the reference tree)")
    rng = np.random.default_rng(20240611)
    out = {}

    rows = []
    for u, lo, hi in [(0.0, 400, 700), (0.37, 400, 700), (0.999, 380, 780), (0.5, 360, 830), (0.81, 450, 650)]:
        lam, p = vec(np.zeros(4))
        r.ref_pt_sample_wavelengths(u, lo, hi, p)
        rows.append([u, lo, hi, lam.tolist()])
    out["sample_wavelengths"] = rows

    rows = []
    for nm in [380.0, 381.3, 455.0, 512.7, 555.0, 699.99, 700.0, 779.0, 780.0, 379.0, 781.0]:
        xyz, p = vec(np.zeros(3))
        ok = r.ref_pt_xyz_from_nm(nm, p)
        rows.append([nm, ok, xyz.tolist()])
    out["xyz_from_nm"] = rows
    out["cie_y_integral"] = [[a, b, r.ref_pt_cie_y_integral(a, b)]
                             for a, b in [(380, 780), (400, 700), (402.5, 697.5), (360, 830), (500, 500)]]

    al = [1e-4, 0.01, 0.05, 0.2, 0.5, 1.0]
    cs = [0.0, 1e-11, 0.01, 0.3, 0.7, 0.999, 1.0]
    out["ggx_d"] = [[a, c, r.ref_pt_ggx_d(a, c)] for a in al for c in cs]
    out["ggx_lambda"] = [[a, c, r.ref_pt_ggx_lambda(a, c)] for a in al for c in cs]
    out["ggx_g2"] = [[a, ci, co, r.ref_pt_ggx_g2(a, ci, co)] for a in al for ci, co in [(0.3, 0.8), (0.05, 0.9), (1.0, 0.5)]]

    rows, prows = [], []
    for _ in range(16):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        wi = hemi(rng, n)
        a = float(rng.uniform(0.02, 0.9))
        u1, u2 = float(rng.random()), float(rng.random())
        m, pm = vec(np.zeros(3))
        onb, po = vec(np.zeros(9))
        _, pwi = vec(wi)
        _, pn = vec(n)
        r.ref_pt_vndf_sample(pwi, pn, a, u1, u2, pm, po)
        rows.append([wi.tolist(), n.tolist(), a, u1, u2, m.tolist(), onb.tolist()])
        wo = hemi(rng, n)
        _, pwo = vec(wo)
        prows.append([wi.tolist(), wo.tolist(), n.tolist(), a, r.ref_pt_vndf_pdf(pwi, pwo, pn, a)])
    out["vndf_sample"] = rows
    out["vndf_pdf"] = prows

    rows = []
    for _ in range(12):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        v = -hemi(rng, n)
        ni, nt, k = 1.0, float(rng.uniform(0.2, 3.0)), float(rng.uniform(0.0, 5.0))
        _, pv = vec(v)
        _, pn = vec(n)
        rows.append([v.tolist(), n.tolist(), ni, nt, k, r.ref_pt_conductor_f(pv, pn, ni, nt, k)])
    out["conductor_f"] = rows

    rows = []
    for _ in range(12):
        ci = float(rng.uniform(0.01, 1.0))
        ni, nt = [(1.0, 1.5), (1.5, 1.0), (1.0, 1.33)][int(rng.integers(0, 3))]
        s2 = (ni / nt) ** 2 * (1 - ci * ci)
        if s2 >= 1:
            continue
        ct = float(np.sqrt(1 - s2))
        n = np.array([0.0, 0.0, 1.0])
        v = np.array([np.sqrt(1 - ci * ci), 0.0, -ci])
        tv = np.array([np.sqrt(s2), 0.0, -ct])
        _, pv = vec(v)
        _, ptv = vec(tv)
        _, pn = vec(n)
        rows.append([ci, ct, ni, nt, r.ref_pt_dielectric_r(pv, ptv, pn, ni, nt)])
    out["dielectric_r"] = rows

    out["lookup_ess"] = [[c, a, r.ref_pt_lookup_ess(c, a)] for c in [0.0, 0.01, 0.3, 0.77, 1.0] for a in [0.0, 0.05, 0.33, 1.0, 1.2]]
    out["lookup_eavg"] = [[a, r.ref_pt_lookup_eavg(a)] for a in [0.0, 0.01, 0.05, 0.33, 0.999, 1.0]]
    out["ms_z"] = [[a, r.ref_pt_ms_z(a)] for a in [0.01, 0.05, 0.2, 0.5, 1.0]]
    out["ms_pdf"] = [[c, a, r.ref_pt_ms_pdf(c, a, r.ref_pt_ms_z(a))] for c in [0.0, 0.1, 0.5, 1.0] for a in [0.05, 0.4]]
    out["ms_sample_cos"] = [[a, u, r.ref_pt_ms_sample_cos(a, u)] for a in [0.02, 0.1, 0.3, 0.8] for u in [0.0, 0.1, 0.5, 0.9, 0.999999]]
    out["fresnel_avg"] = [[ni, nt, k, r.ref_pt_fresnel_avg(ni, nt, k)] for ni, nt, k in [(1, 0.2, 3.0), (1, 1.5, 0.0), (1, 2.9, 3.1)]]
    out["fms"] = [[f, e, r.ref_pt_fms(f, e)] for f, e in [(0.9, 0.6), (0.3, 0.99), (1.0, 0.3)]]
    out["power_heuristic"] = [[a, b, r.ref_pt_power_heuristic(a, b)] for a, b in [(1, 1), (0.2, 5), (3, 0.01)]]
    cases = [[0.3, 0.5, 0.1], [0.9505, 1.0, 1.089], [0.0, 0.0, 0.0], [0.6, 0.05, 0.02], [0.05, 0.6, 0.01],
             [0.1, 0.02, 0.9], [0.25, 0.1, 0.5], [1e-9, 2e-9, 3e-9], [2.5, 3.0, 0.2], [0.4, 0.4, -0.05]]
    cases += rng.exponential(0.5, (30, 3)).tolist()
    rows = []
    for xyz in cases:
        rgb, p = vec(np.zeros(3))
        _, px = vec(xyz)
        r.ref_pt_xyz_to_rec709(px, p)
        rows.append([xyz, rgb.tolist()])
    out["xyz_to_rec709"] = rows
    rows = []
    for xyz, rgb in out["xyz_to_rec709"]:
        for tone in range(5):
            for ev in (0.0, 1.0, -1.5):
                o = (ctypes.c_ubyte * 3)()
                _, pr = vec(rgb)
                r.ref_pt_display(pr, ev, tone, o)
                rows.append([rgb, ev, tone, list(o)])
    out["display"] = rows
    rows = []
    for nm, amp, lo, hi in [([400, 450, 500, 600, 700], [0.1, 0.5, 0.2, 0.9, 0.3], 400, 700),
                            ([380, 420, 430, 700, 780], [1.0, 0.0, 2.0, 0.5, 0.25], 390, 710),
                            ([550], [0.7], 400, 700), ([700, 400, 550], [3.0, 1.0, 2.0], 380, 780),
                            (list(np.arange(400, 701, 4.0)), list(rng.random(76)), 400, 700)]:
        q = np.concatenate([np.linspace(lo - 10, hi - 1e-6, 41), [lo, lo + 1e-9]])
        o, po = vec(np.zeros(len(q)))
        _, pn = vec(nm)
        _, pa = vec(amp)
        _, pq = vec(q)
        r.ref_pt_spectral_packet(pn, pa, len(nm), float(lo), float(hi), pq, len(q), po)
        rows.append([list(map(float, nm)), list(map(float, amp)), lo, hi, q.tolist(), o.tolist()])
    out["spectral_packet"] = rows
    lrng = np.random.default_rng(77)
    rows = []
    for n in (2, 3, 7, 40):
        pos = lrng.uniform(-1, 1, (n, 3))
        if n == 7:
            pos[:, 1] = 0.5                      # a flat row of lights (zero extent on one axis)
        power = lrng.exponential(1.0, n)
        pts = lrng.uniform(-1.5, 1.5, (25, 3))
        xi = lrng.random(25)
        picked, pdf, pdf_all = oracle.light_bvh(r, "ref_pt_", pos, power, pts, xi)
        rows.append([pos.tolist(), power.tolist(), pts.tolist(), xi.tolist(), picked.tolist(), pdf.tolist(),
                     pdf_all.tolist()])
    out["light_bvh"] = rows
    lut_path = os.path.join(os.path.dirname(HERE), "..", "oracle", "_ref", "rec709.coeff")
    table = np.ascontiguousarray(np.fromfile(lut_path, dtype=np.uint8)[20:].view(np.float32))
    urng = np.random.default_rng(91)
    colours = [[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.8, 0.1, 0.05], [0.1, 0.7, 0.2], [0.05, 0.1, 0.9],
               [0.5, 0.5, 0.5], [0.18, 0.18, 0.18], [3.0, 2.0, 1.0], [15.0, 15.0, 15.0]]
    colours += urng.random((12, 3)).tolist()
    qnm = np.linspace(375, 785, 42)
    rows = []
    P = ctypes.c_void_p
    for rgb in colours:
        for kind in (0, 1):
            c, vals = np.zeros(3), np.zeros(len(qnm))
            rr = np.ascontiguousarray(rgb, np.float64)
            r.ref_pt_rgb_uplift(table.ctypes.data_as(P), ctypes.c_uint(table.size), rr.ctypes.data_as(P), kind,
                                qnm.ctypes.data_as(P), len(qnm), c.ctypes.data_as(P), vals.ctypes.data_as(P))
            rows.append([rgb, kind, c.tolist(), qnm.tolist(), vals.tolist()])
    out["rgb_uplift"] = rows
    out["gaussian_filter"] = [[s, g, dx, dy, r.ref_pt_gaussian_weight(s, g, dx, dy)]
                              for s, g in [(2.0, 0.5), (3.0, 1.0), (1.0, 0.3)]
                              for dx, dy in [(0, 0), (0.3, -0.2), (0.99, 0.5), (1.0, 0.0), (-1.01, 0.1), (1.4, 1.4)]]
    rows = []
    for depth, mind, thr, cur, prev, u in [(2, 3, 0.05, 0.1, 1.0, 0.9), (3, 3, 0.05, 0.1, 1.0, 0.05), (3, 3, 0.05, 0.1, 1.0, 0.5),
                                           (5, 3, 0.05, 0.01, 0.02, 0.3), (4, 3, 0.05, 2.0, 1.0, 0.99), (6, 3, 0.05, 0.0, 0.5, 0.0)]:
        s = ctypes.c_double()
        t = r.ref_pt_russian_roulette(depth, mind, thr, cur, prev, u, ctypes.byref(s))
        rows.append([depth, mind, thr, cur, prev, u, t, s.value])
    out["russian_roulette"] = rows

    # Owen-scrambled Sobol (Sampling/SobolSequence.h): value * 2^32 as an
    # integer, for indices, dimensions and seeds including the edges.
    srng = np.random.default_rng(17)
    idx = np.concatenate([[0, 1, 2, 3, 255, 256, 65535, 2**31, 2**32 - 1],
                          srng.integers(0, 2**32, 55, dtype=np.uint64)]).astype(np.uint32)
    dim = np.concatenate([[0, 1, 2, 3, 31, 32, 543, 544, 1023], srng.integers(0, 1024, 55)]).astype(np.uint32)
    seed = srng.integers(0, 2**32, idx.size, dtype=np.uint64).astype(np.uint32)
    vals = oracle.sobol(idx, dim, seed, "ref")
    out["sobol"] = [[int(a), int(b), int(c), int(round(v * 4294967296.0))] for a, b, c, v in zip(idx, dim, seed, vals)]
    hc = oracle.hash_combine(idx, seed, "ref")
    out["hash_combine"] = [[int(a), int(c), int(h)] for a, c, h in zip(idx, seed, hc)]

    ess, eavg = oracle.energy_tables(r, "ref_pt_")
    out["energy_tables"] = {"ess": ess.round(8).tolist(), "eavg": eavg.round(8).tolist()}

    path = os.path.join(HERE, "pt_blocks.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
