"""Helpers of the statistical tests: shape-order permutation and z-scores.

The edge order of a scene follows its shape order.  The reference orders its
edges by Shape* address instead (a sort key per shape, `rank`), so a render of
the reference with order `rank` corresponds to a render of this library whose
shape list is sorted by `rank`.  `permuted(wl, rank)` builds that workload and
`to_original(flat)` maps its flat gradient back to the original layout.
"""
import dataclasses
import json
import os

import numpy as np

from conftest import GOLDEN

STATS = os.path.join(GOLDEN, "stats")


def stats_cases():
    return sorted(f[:-4] for f in os.listdir(STATS) if f.endswith(".npz"))


def load_stats(name):
    z = np.load(os.path.join(STATS, name + ".npz"))
    return json.loads(str(z["meta"])), {k: z[k] for k in z.files if k != "meta"}


def _grad_blocks(wl):
    from delta_ray_b200 import _abi
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts)
    blocks, o = {}, 0
    for kind, i, n in sd.grad_sizes:
        blocks[(kind, i)] = (o, n)
        o += n
    return blocks, o


def permuted(wl, rank):
    """(workload with shapes sorted by rank, function mapping its flat gradient to wl's layout)."""
    from delta_ray_b200.light import Light
    order = [int(i) for i in np.argsort(np.asarray(rank), kind="stable")]  # new index j <- old shape order[j]
    new_of_old = {old: new for new, old in enumerate(order)}
    wl2 = dataclasses.replace(wl, shapes=[wl.shapes[i] for i in order],
                              lights=[Light(new_of_old[l.shape_id], l.intensity) for l in wl.lights])
    b1, total = _grad_blocks(wl)
    b2, _ = _grad_blocks(wl2)

    def to_original(flat):
        flat = np.asarray(flat)
        out = np.empty(total, flat.dtype)
        for (kind, i), (o2, n) in b2.items():
            key = (kind, order[i]) if kind in ("vertices", "normals") else (kind, i)
            o1, n1 = b1[key]
            assert n1 == n
            out[o1:o1 + n] = flat[o2:o2 + n]
        return out

    return wl2, to_original


def zscores(mean_a, se_a, mean_b, se_b, floor):
    """(a - b) / combined standard error, with an absolute floor for entries
    that are zero up to rounding on both sides."""
    s = np.sqrt(np.asarray(se_a, np.float64) ** 2 + np.asarray(se_b, np.float64) ** 2 + floor ** 2)
    return (np.asarray(mean_a, np.float64) - np.asarray(mean_b, np.float64)) / s


def agree(z, rms_max, frac3_min, max_abs):
    """Means agree: z-scores look like unit noise (K = 8 renders a side, so the
    standard errors are themselves noisy: t tails, not normal ones)."""
    z = np.ravel(z)
    rms = float(np.sqrt(np.mean(z ** 2)))
    frac3 = float(np.mean(np.abs(z) < 3))
    mx = float(np.abs(z).max())
    return rms < rms_max and frac3 >= frac3_min and mx < max_abs, dict(rms=rms, frac3=frac3, max=mx)
