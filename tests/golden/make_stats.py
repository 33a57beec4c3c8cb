"""Generates the high-sample statistics fixtures from the compiled reference.

Run from the repository root after ``make -C oracle ref`` (needs the
reference sources, so it only runs where they are mounted):

    python tests/golden/make_stats.py

For every case it renders the scene K times with the reference's own renderer
(oracle/_ref: the reference sources with their own flags and the project's CPU
BVH in place of Embree), each time with a different seed at spp samples per
pixel, and stores the per-pixel and per-parameter mean and standard error of
the mean over the K renders in tests/golden/stats/<case>.npz.  K * spp is the
total sample count (4096 per pixel).  The GPU test renders the same scenes
with its own random streams and checks that the means agree within a few
standard errors: the reference's random numbers (mt19937 per image tile) and
the product's (Philox per sample) differ, so only the expectations can match.

The reference keeps one secondary-edge position derivative per shading point,
the last one in edge order (delta_ray.cpp:975-1002), and orders edges by
Shape* address, which changes between calls; the expected gradient depends on
that order.  So every render's shape order is identified (the oracle in the
reference's own random-number mode reproduces the render sample for sample
only with the right order) and stored, and the tests render with the same
orders.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from make_golden import build_case, scene_checksum  # noqa: E402

K = 8
CASES = [
    # name, builder, kwargs (spp per render), first seed
    ("soft_shadow", "soft_shadow", dict(seed=2, resolution=(32, 32), spp=512, max_bounces=1), 100),
    ("glossy_shadow", "glossy_shadow", dict(seed=4, resolution=(24, 20), spp=512, max_bounces=2), 200),
]


def main():
    import oracle
    import ref_runner
    os.makedirs(os.path.join(HERE, "stats"), exist_ok=True)
    for name, builder, kwargs, seed0 in CASES:
        wl = build_case(builder, kwargs)
        W, H = wl.resolution
        dimg = np.ones((H, W, 3), np.float32)
        ltc = np.fromfile(os.path.join(ROOT, "oracle", "_ref", "ltc_tabM.f32"), np.float32)
        cores = os.cpu_count()  # the reference's num_system_cores() (parallel.cpp:203-210)
        imgs, grads, orders, errs = [], [], [], []
        for k in range(K):
            out = ref_runner.render_reference(wl, seed0 + k, d_image=dimg, strict=True)
            rank, _, err = oracle.match_reference_order(wl, out, seed0 + k, dimg, cores=cores, ltc_table=ltc)
            imgs.append(out["image"].astype(np.float64))
            grads.append(oracle.flat_from_parts(wl, out).astype(np.float64))
            orders.append(np.asarray(rank, np.int32))
            errs.append(float(err))
        imgs, grads = np.stack(imgs), np.stack(grads)
        meta = dict(name=name, builder=builder, kwargs=kwargs, renders=K, seeds=[seed0 + k for k in range(K)],
                    spp_total=K * wl.spp, checksum=scene_checksum(wl), reference_build="oracle/_ref/strict",
                    adjoint="ones", order_match_err=max(errs))
        np.savez_compressed(os.path.join(HERE, "stats", name + ".npz"), meta=json.dumps(meta),
                            image_mean=imgs.mean(0), image_se=imgs.std(0, ddof=1) / np.sqrt(K),
                            grad_mean=grads.mean(0), grad_se=grads.std(0, ddof=1) / np.sqrt(K),
                            orders=np.stack(orders))
        print(f"{name}: {K} x {wl.spp} spp, |grad| max {np.abs(grads.mean(0)).max():.3g}, "
              f"orders {[o.tolist() for o in orders]}, worst order match {max(errs):.2e}")


if __name__ == "__main__":
    main()
