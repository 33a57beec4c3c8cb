"""dr_scene_update: a scene updated with new parameters renders exactly as a
scene built from scratch with them.  With unchanged triangle indices the
update reuses the edge topology and refits the LBVH; with re-indexed
triangles it rebuilds both."""
import copy

import numpy as np
import pytest
import torch

from conftest import rel_err


def _scene(wl):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, None)


def _update(sc, wl):
    from delta_ray_b200 import _abi
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sc.update(cam, mats, shps, lts)


def _render(sc, wl, seed=17):
    W, H = wl.resolution
    img = sc.forward(W, H, wl.spp, wl.max_bounces, seed).cpu().numpy()
    grad, img_b = sc.backward(W, H, wl.spp, wl.max_bounces, seed, torch.ones((H, W, 3), device="cuda"),
                              want_image=True)
    return img, img_b.cpu().numpy(), grad.cpu().numpy()


def _check(a, b):
    assert np.array_equal(a[0], b[0])  # forward image: same samples, same hits
    assert np.array_equal(a[1], b[1])
    assert rel_err(a[2], b[2]) < 1e-5  # gradient: float atomics reorder sums


def _moved(wl, seed):
    rng = np.random.default_rng(seed)
    w2 = copy.deepcopy(wl)
    for s in w2.shapes[:-1]:  # not the light
        s.vertices = s.vertices + torch.from_numpy(rng.normal(0, 0.05, tuple(s.vertices.shape)).astype(np.float32))
    w2.lights[0].intensity = w2.lights[0].intensity * 1.5
    w2.materials[0].diffuse_reflectance = w2.materials[0].diffuse_reflectance * 0.8
    return w2


@pytest.mark.gpu
@pytest.mark.parametrize("builder", ["soft_shadow", "heightfield_small"])
def test_update_matches_fresh_scene(builder):
    from golden.make_golden import build_case
    kw = dict(seed=3, resolution=(48, 40), spp=4, max_bounces=2)
    wl = build_case(builder, kw)
    sc = _scene(wl)
    for k in range(2):  # two updates in a row
        w2 = _moved(wl, 10 + k)
        _update(sc, w2)
        fresh = _scene(w2)
        _check(_render(sc, w2), _render(fresh, w2))
        fresh.close()
    sc.close()


@pytest.mark.gpu
def test_update_with_reindexed_triangles_rebuilds():
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(3, (48, 40), 4, 1)
    sc = _scene(wl)
    w2 = copy.deepcopy(wl)
    w2.shapes[1].indices = w2.shapes[1].indices[:, [1, 2, 0]].contiguous()  # same triangles, rotated corners
    _update(sc, w2)
    fresh = _scene(w2)
    _check(_render(sc, w2), _render(fresh, w2))
    fresh.close()
    sc.close()
