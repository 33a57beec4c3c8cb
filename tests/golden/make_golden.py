"""Generates the golden fixtures of the parity tests from the compiled reference.

Run from the repository root after ``make -C oracle ref`` (needs the
reference sources, so it only runs where they are mounted):

    python tests/golden/make_golden.py

For every case it renders the scene with the reference's own renderer
(oracle/_ref/strict: the reference sources compiled with IEEE arithmetic and
the project's CPU BVH in place of Embree), forward and backward, and stores the
image, the backward image and the flat gradient (product layout) in
tests/golden/<case>.npz.  The reference orders its edges by Shape* address,
which varies between calls, so the generator also records the shape order the
call used (found by matching the oracle's renders); the oracle tests replay
that order.  Scenes are rebuilt from their seeded builders at test time; a
checksum of the scene arrays guards against builder drift.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

CASES = [
    # name, builder, kwargs, render seed
    ("single_triangle", "single_triangle", dict(seed=1, resolution=(32, 32), spp=4, max_bounces=1), 3),
    ("soft_shadow", "soft_shadow", dict(seed=2, resolution=(32, 32), spp=4, max_bounces=1), 5),
    ("soft_shadow_b3", "soft_shadow", dict(seed=3, resolution=(24, 20), spp=2, max_bounces=3), 7),
    ("glossy_shadow", "glossy_shadow", dict(seed=4, resolution=(24, 20), spp=2, max_bounces=2), 11),
    ("textured", "textured", dict(seed=5, resolution=(24, 24), spp=2, max_bounces=2), 13),
    ("smooth_sphere", "smooth_sphere", dict(seed=6, resolution=(24, 24), spp=2, max_bounces=1), 17),
    ("fisheye", "fisheye", dict(seed=7, resolution=(24, 24), spp=2, max_bounces=1), 19),
    ("heightfield_small", "heightfield_small", dict(seed=8, resolution=(24, 20), spp=2, max_bounces=2), 23),
    ("mirror_shadow", "mirror_shadow", dict(seed=10, resolution=(24, 20), spp=2, max_bounces=3), 29),
    ("mirror_hall", "mirror_hall", dict(seed=11, resolution=(24, 20), spp=2, max_bounces=5), 31),
]


def build_case(builder, kwargs):
    from delta_ray_b200 import workloads
    import scenes
    fn = workloads.BUILDERS.get(builder) or scenes.SCENES[builder]
    kw = dict(kwargs)
    if "resolution" in kw:
        kw["resolution"] = tuple(kw["resolution"])
    return fn(**kw)


def scene_checksum(wl):
    h = hashlib.sha256()
    for a in wl.serialize():
        if hasattr(a, "detach"):
            h.update(np.ascontiguousarray(a.detach().cpu().numpy()).tobytes())
        else:
            h.update(repr(a).encode())
    return h.hexdigest()[:16]


def adjoint_image(wl, seed):
    W, H = wl.resolution
    return np.random.default_rng(1000 + seed).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)


def main():
    import oracle
    import ref_runner
    ltc = np.fromfile(os.path.join(ROOT, "oracle", "_ref", "ltc_tabM.f32"), np.float32)
    only = set(sys.argv[1:])  # optional case names: regenerate those only
    for name, builder, kwargs, seed in CASES:
        if only and name not in only:
            continue
        wl = build_case(builder, kwargs)
        dimg = adjoint_image(wl, seed)
        fwd = ref_runner.render_reference(wl, seed, strict=True)
        bwd = ref_runner.render_reference(wl, seed, d_image=dimg, strict=True)
        cores = os.cpu_count()  # the reference's num_system_cores() (parallel.cpp:203-210)
        rank, _, err = oracle.match_reference_order(wl, bwd, seed, dimg, cores=cores, ltc_table=ltc)
        flat = oracle.flat_from_parts(wl, bwd)
        meta = dict(name=name, builder=builder, kwargs=kwargs, seed=seed, checksum=scene_checksum(wl),
                    reference_build="oracle/_ref/strict", cores=cores, match_err=err)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=json.dumps(meta), image=fwd["image"],
                            image_bwd=bwd["image"], grad=flat, shape_rank=rank, d_image=dimg)
        print(f"{name}: rank {rank.tolist()} oracle match {err:.2e}")


if __name__ == "__main__":
    main()
