"""dr_render_backward_views: several cameras, resolutions and sample counts
in one call, against one dr_render_backward per view on scenes created with
that view's camera (the gradients of every non-camera parameter sum over the
views; each view's camera gradient comes back on its own)."""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _views(wl, around=False):
    from delta_ray_b200 import workloads
    specs = [([0, 5, -4.5], [0, 3, 0], 60.0, (48, 40), 4, 3),
             ([3.5, 6, -3], [0, 2, 0.5], 55.0, (32, 32), 2, 5),
             ([-3, 2.5, 3.5], [0.5, 2.5, -1], 70.0, (40, 24), 8, 7)]
    if around:  # looking at the origin from a circle (the heightfield)
        specs = [([0, 7, -10.5], [0, 0, 0], 45.0, (48, 40), 4, 3),
                 ([9.1, 7, 5.25], [0, 0, 0], 45.0, (32, 32), 2, 5),
                 ([-9.1, 7, 5.25], [0, 0, 0], 45.0, (40, 24), 8, 7)]
    rng = np.random.default_rng(2)
    views = []
    for eye, tgt, fov, res, spp, seed in specs:
        cam = workloads._camera(eye, tgt, [0, 1, 0], fov, list(res))
        views.append(dict(camera=cam, width=res[0], height=res[1], spp=spp, max_bounces=wl.max_bounces,
                          seed=seed, d_image=rng.uniform(0.5, 1.5, (res[1], res[0], 3)).astype(np.float32)))
    return views


def _case(name):
    import scenes
    from delta_ray_b200 import workloads
    if name == "icosphere_room":
        return scenes.icosphere_room(seed=3, n_spheres=8, subdiv=(1, 2), max_bounces=2)
    # 7,938 triangles: GPU-built edge trees, subtrees walked by the second stage
    return workloads.heightfield(seed=2, resolution=(48, 40), spp=2, max_bounces=2, grid=64, patch=16)


@pytest.mark.parametrize("name,mixed", [("icosphere_room", False), ("heightfield", False), ("icosphere_room", True)])
def test_views_match_one_call_per_view(name, mixed):
    """Views with the same bounce count and flags run batched (their points
    share one edge stage); `mixed` gives one view another bounce count, which
    runs the views one after another."""
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    wl = _case(name)
    views = _views(wl, around=name == "heightfield")
    if mixed:
        views[1]["max_bounces"] = wl.max_bounces + 1
    _, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sc = Scene(_abi.scene_dicts(wl.camera, [], [], [])[0], mats, shps, lts, 0, None)
    for _ in range(2):  # the second call reuses the queues and the view buffers
        grad, cam_grads = sc.backward_views(views)
        counts = tuple(sc.last_counts())
        grad, cam_grads = grad.cpu().numpy(), cam_grads.cpu().numpy()
        assert np.all(grad[:64] == 0) and np.isfinite(grad).all()
        ref = np.zeros_like(grad)
        ref_counts = np.zeros(2, np.int64)
        for k, v in enumerate(views):
            s1 = Scene(_abi.scene_dicts(v["camera"], [], [], [])[0], mats, shps, lts, 0, None)
            g1, _ = s1.backward(v["width"], v["height"], v["spp"], v["max_bounces"], v["seed"],
                                torch.from_numpy(v["d_image"]))
            ref_counts += np.array(s1.last_counts())
            g1 = g1.cpu().numpy()
            ref[64:] += g1[64:]
            assert rel_err(cam_grads[k], g1[:64]) < 1e-4, k
            s1.close()
        assert counts == tuple(ref_counts)
        assert np.abs(ref).max() > 0
        assert rel_err(grad, ref) < 1e-4
    sc.close()


@pytest.mark.parametrize("seed", [6, 7, 8])
def test_icosphere_room_matches_oracle(seed):
    """The multi-view stand-in scene (closed room, icospheres with shading
    normals, glossy lobes, two bounces) against the oracle: its shading points
    sit near many small triangles, where one edge-tree choice decided
    differently would move the gradient of a handful of vertices by a lot;
    counts and every gradient entry."""
    import oracle
    import scenes
    from conftest import assert_grad_parity
    from test_backward_gpu import product_scene
    wl = scenes.icosphere_room(seed=3, n_spheres=8, subdiv=(1, 2), resolution=(32, 24), spp=2, max_bounces=2)
    W, H = wl.resolution
    d = np.random.default_rng(1).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = product_scene(wl)
    grad, _ = sc.backward(W, H, wl.spp, wl.max_bounces, seed, torch.from_numpy(d))
    o = oracle.oracle_render(wl, seed, d, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()
