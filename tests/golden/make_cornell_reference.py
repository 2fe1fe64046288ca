"""Generate the C1 Cornell box fixtures from the reference renderer itself
(oracle/_ref/librise_ref.so, built from the reference sources by
oracle/rise_ref.mk), on tests/golden/cornell_c1.RISEscene:

* cornell_c1_ref_fp64.npz -- the converged image: mean XYZ (256, 256, 3)
  of 16384 samples per pixel in FP64 (stored as float32), through the
  reference's per-sample function given independent numbers (its
  IndependentSampler; oracle.RefRenderer.integrate(independent=True)).  With
  its own Sobol sampler a pixel does not converge: one seed per pixel and
  dimensions that reuse two Sobol dimensions with only the scrambling
  changed leave a per-pixel error that more samples do not remove (relMSE
  about 2e-3 against this image at any sample count).  This image's noise
  (relMSE ~3e-5) is far below the 1e-3 level that relMSE figures are judged
  at, so a GPU image's relMSE against it measures the GPU's noise plus any
  bias.
* cornell_c1_ref_k16.npz -- per-pixel mean and variance (ddof 1) of XYZ over
  16 independent batches of 16 samples per pixel (batches 1..16: the batch
  number mixed into the Sobol seed), for the per-pixel z-test of the GPU
  path tracer against the reference at equal samples per pixel.
* cornell_c1_ref_k16_independent.npz -- the same with the reference's
  IndependentSampler (uniform numbers from a Mersenne twister) in place of
  its Sobol sampler: the reference integrator's estimate without the small
  bias its padded Sobol sequence carries (images about 0.1-0.3 % brighter
  than with independent numbers), for a tight test of the image mean.
* cornell_smooth_ref_k16_independent.npz -- 16 x 16 spp with independent
  numbers of tests/golden/cornell_smooth.RISEscene, the box with a smooth-
  shaded Lambertian sphere and a smooth-shaded glass sphere (vertex normals
  from RAW2 files): the z-test of interpolated shading normals.
* cornell_nm_ref_k16_independent.npz, cornell_prism_ref_k16_independent.npz,
  cornell_prism_nm_ref_k16_independent.npz -- the same for the wavelength-
  sampling variants (tests/golden/make_cornell_scene.py variants): one
  wavelength per path in 10 bins; a dispersive glass prism under hero-
  wavelength bundles; the prism with one wavelength per path in 30 bins and
  two spectral samples per pixel sample (the prism scenes at 16 batches of 64
  samples per pixel).
* cornell_overlap_ref_k16_independent.npz -- 16 x 64 spp with independent
  numbers of tests/golden/cornell_overlap.RISEscene (make_cornell_scene.py
  overlap): overlapping glass spheres of indices 1.5 and 1.33 and a GGX
  conductor cutting into one of them, the z-test of the index-of-refraction
  stack.
* cornell_dsglass_ref_k16_independent.npz -- 16 x 64 spp with independent
  numbers of tests/golden/cornell_dsglass.RISEscene (make_cornell_scene.py
  dsglass): a double-sided glass sphere, whose normals turn towards the ray
  while its dielectric reads inside / outside from the stack.
* cornell_env_ref_k16_independent.npz -- the same for
  tests/golden/cornell_env.RISEscene (tests/golden/make_env_scene.py): a
  scene lit only by an HDR light probe, rotated and scaled, 128 x 128.

    make -C oracle && python tests/golden/make_cornell_reference.py [k16|k16i|smooth|variants|overlap|dsglass|env|fp64]
    (k16, k16i: ~40 s each, fp64: ~45 min on 8 cores; rows are checkpointed under
    oracle/_ref/ so an interrupted run resumes)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

SCENE = os.path.join(HERE, "cornell_c1.RISEscene")
K, K_SPP = 16, 16
FP64_SPP = 16384
ROWS = 8


def make_k16(r, independent=False, name=None, spp=K_SPP):
    t0 = time.time()
    b = np.array([r.integrate(spp, batch=k, independent=independent) for k in range(1, K + 1)])
    name = name or ("cornell_c1_ref_k16_independent.npz" if independent else "cornell_c1_ref_k16.npz")
    np.savez_compressed(os.path.join(HERE, name), mean=b.mean(0).astype(np.float32),
                        var=b.var(0, ddof=1).astype(np.float32), k=K, spp=spp)
    print(f"{name}: {time.time() - t0:.0f} s", flush=True)


def make_fp64(r):
    ck = os.path.join(ROOT, "oracle", "_ref", "cornell_c1_fp64_independent_rows.npy")
    img = np.load(ck) if os.path.exists(ck) else np.full((r.height, r.width, 3), np.nan)
    t0 = time.time()
    for y0 in range(0, r.height, ROWS):
        if not np.isnan(img[y0:y0 + ROWS]).any():
            continue
        img[y0:y0 + ROWS] = r.integrate(FP64_SPP, batch=0, rect=(0, y0, r.width, y0 + ROWS), independent=True)
        np.save(ck, img)
        print(f"rows {y0 + ROWS}/{r.height}, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "cornell_c1_ref_fp64.npz"), xyz=img.astype(np.float32), spp=FP64_SPP)


def main():
    which = sys.argv[1:] or ["k16", "k16i", "smooth", "variants", "overlap", "dsglass", "env", "fp64"]
    r = oracle.RefRenderer(SCENE)
    if "k16" in which:
        make_k16(r)
    if "k16i" in which:
        make_k16(r, independent=True)
    if "fp64" in which:
        make_fp64(r)
    if "smooth" in which:
        make_k16(oracle.RefRenderer(os.path.join(HERE, "cornell_smooth.RISEscene")), independent=True,
                 name="cornell_smooth_ref_k16_independent.npz")
    if "env" in which:
        make_k16(oracle.RefRenderer(os.path.join(HERE, "cornell_env.RISEscene")), independent=True,
                 name="cornell_env_ref_k16_independent.npz")
    if "variants" in which:
        # The prism's caustics make single pixels heavy-tailed; 64 samples
        # per batch bring the batch means nearer to normal for the z-test.
        for v, spp in (("cornell_nm", K_SPP), ("cornell_prism", 64), ("cornell_prism_nm", 64)):
            make_k16(oracle.RefRenderer(os.path.join(HERE, v + ".RISEscene")), independent=True,
                     name=v + "_ref_k16_independent.npz", spp=spp)
    if "overlap" in which:
        make_k16(oracle.RefRenderer(os.path.join(HERE, "cornell_overlap.RISEscene")), independent=True,
                 name="cornell_overlap_ref_k16_independent.npz", spp=64)
    if "dsglass" in which:
        make_k16(oracle.RefRenderer(os.path.join(HERE, "cornell_dsglass.RISEscene")), independent=True,
                 name="cornell_dsglass_ref_k16_independent.npz", spp=64)


if __name__ == "__main__":
    main()
