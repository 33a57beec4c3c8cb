"""Queue settings of a scene and their autotuner (dr_scene_set_tuning,
dr_scene_autotune).  The settings decide how the subtrees of the edge trees
are walked (level by level, or depth first in rounds) and how many edge
items a chunk of the edge stage holds, never which edges are sampled: every
setting gives the same counts and image, and the gradient up to float
round-off (atomic adds sum in another order)."""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _heightfield():
    from delta_ray_b200 import _abi, workloads
    from delta_ray_b200.render_pytorch import Scene
    # 64 x 64 vertices: 7,938 triangles, edge trees walked in two stages
    wl = workloads.heightfield(seed=2, resolution=(48, 40), spp=2, max_bounces=2, grid=64, patch=16)
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return wl, Scene(cam, mats, shps, lts, 0, None)


def _call(sc, wl, d_image):
    W, H = wl.resolution
    g, img = sc.backward(W, H, wl.spp, wl.max_bounces, 11, d_image, want_image=True)
    return g.cpu().numpy(), img.cpu().numpy(), tuple(sc.last_counts())


def test_settings_leave_the_results_unchanged():
    from delta_ray_b200 import _lib
    wl, sc = _heightfield()
    W, H = wl.resolution
    d_image = torch.from_numpy(np.random.default_rng(5).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)).cuda()
    try:
        assert sc.tuning() == {"hand_steps": 64, "task_rounds": 3, "queue_items": 0, "depth_first": 0}
        g0, img0, c0 = _call(sc, wl, d_image)  # the level walk
        assert sc.last_work()["tasks"] > 0
        small = max(65536, c0[1] // 3)
        for hand, rounds, queue, df in ((64, 3, 0, 1), (1, 8, 0, 1), (4096, 1, 0, 1), (16, 2, small, 1),
                                        (64, 3, small, 0)):
            sc.set_tuning(hand, rounds, queue, df)
            assert sc.tuning() == {"hand_steps": hand, "task_rounds": rounds, "queue_items": queue,
                                   "depth_first": df}
            g, img, c = _call(sc, wl, d_image)
            assert c == c0 and np.array_equal(img, img0), (hand, rounds, queue, df)
            assert rel_err(g, g0) < 1e-5, (hand, rounds, queue, df)
        for bad in ((0, 3, 0, 0), (64, 0, 0, 0), (64, 9, 0, 0), (64, 3, -1, 0), (64, 3, 0, 2)):
            with pytest.raises(_lib.DrError):
                sc.set_tuning(*bad)
        assert sc.tuning()["queue_items"] == small  # a rejected setting changes nothing
    finally:
        sc.close()


def test_autotune_keeps_the_fastest_setting():
    wl, sc = _heightfield()
    W, H = wl.resolution
    d_image = torch.from_numpy(np.random.default_rng(6).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)).cuda()
    try:
        g0, img0, c0 = _call(sc, wl, d_image)
        rep = sc.autotune(W, H, wl.spp, wl.max_bounces, 11, d_image, max_trials=10)
        assert 1 <= rep["trials"] <= 10
        assert 0 < rep["best_ms"] <= rep["start_ms"]
        best = {k: rep[k] for k in ("hand_steps", "task_rounds", "queue_items", "depth_first")}
        assert sc.tuning() == best
        assert best["task_rounds"] in (1, 2, 3, 4) and best["hand_steps"] in (16, 32, 64, 128, 256)
        assert best["depth_first"] in (0, 1)
        g, img, c = _call(sc, wl, d_image)
        assert c == c0 and np.array_equal(img, img0)
        assert rel_err(g, g0) < 1e-5
    finally:
        sc.close()
