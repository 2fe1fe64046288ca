"""Reference-renderer fixtures for the large scene (the 1024 x 1024 fBm
heightfield with 64 GGX / glass spheres, an area light and a uniform sky:
rise_b200.scenes.spheres_scene(), 3,373,060 triangles), on its 128 x 128
centre crop (pixels 448..575 in x and y):

* spheres_crop_ref_k16_independent.npz -- per-pixel mean and variance of XYZ
  over 16 independent batches of 16 samples per pixel, for the z-test;
* spheres_crop_ref_4096.npz -- the crop at 4096 samples per pixel, the
  reference for the large scene's relMSE (the full image at 16384 samples
  per pixel would take days of host time).

The scene goes to the reference renderer in its own scene language through
oracle/scene_writer.py (written to a scratch folder, about 300 MB of RAW
meshes), loaded by oracle.RefRenderer (oracle/_ref/librise_ref.so, built by
oracle/rise_ref.mk); the reference's integrator is given independent numbers.

    make -C oracle && python tests/golden/make_spheres_reference.py [k16|4096]
    (k16: ~2 min, 4096: ~25 min on 16 cores; rows of the 4096 image are
    checkpointed under oracle/_ref/ so an interrupted run resumes)
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle.scene_writer import write_risescene  # noqa: E402
from rise_b200 import scenes  # noqa: E402

CROP = (448, 448, 576, 576)
K, K_SPP, BIG_SPP, ROWS = 16, 16, 4096, 16


def main():
    which = sys.argv[1:] or ["k16", "4096"]
    tmp = tempfile.mkdtemp(prefix="spheres_ref_")
    r = oracle.RefRenderer(write_risescene(scenes.spheres_scene(), tmp, "spheres", spp=16))
    if "k16" in which:
        t0 = time.time()
        b = np.array([r.integrate(K_SPP, batch=k, rect=CROP, independent=True) for k in range(1, K + 1)])
        np.savez_compressed(os.path.join(HERE, "spheres_crop_ref_k16_independent.npz"), mean=b.mean(0).astype(np.float32),
                            var=b.var(0, ddof=1).astype(np.float32), k=K, spp=K_SPP, crop=np.array(CROP))
        print(f"k16: {time.time() - t0:.0f} s", flush=True)
    if "4096" in which:
        ck = os.path.join(ROOT, "oracle", "_ref", "spheres_crop_4096_rows.npy")
        h, w = CROP[3] - CROP[1], CROP[2] - CROP[0]
        img = np.load(ck) if os.path.exists(ck) else np.full((h, w, 3), np.nan)
        t0 = time.time()
        for y0 in range(0, h, ROWS):
            if not np.isnan(img[y0:y0 + ROWS]).any():
                continue
            rect = (CROP[0], CROP[1] + y0, CROP[2], CROP[1] + y0 + ROWS)
            img[y0:y0 + ROWS] = r.integrate(BIG_SPP, batch=0, rect=rect, independent=True)
            np.save(ck, img)
            print(f"rows {y0 + ROWS}/{h}, {time.time() - t0:.0f} s", flush=True)
        np.savez_compressed(os.path.join(HERE, "spheres_crop_ref_4096.npz"), xyz=img.astype(np.float32), spp=BIG_SPP,
                            crop=np.array(CROP))
    r.close()


if __name__ == "__main__":
    main()
