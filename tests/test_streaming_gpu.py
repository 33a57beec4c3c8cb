"""The edge stage streamed in chunks of shading points.  With the item queue
bounded (dr_set_item_queue_limit) below what a call's points sample, the
call traverses and evaluates its edges chunk by chunk; the sampled edges,
their count and the gradient are those of the unbounded call (the gradient to
float round-off: atomics sum in another order).  Covered: the one-stage
traversal (small edge trees) and the two-stage one (subtree tasks); chunks
planned from the call's own full pass (a scene's first call), from the
previous call's edge counts per range of points, and from its edges per point
alone (after an unbounded call); bounds small enough that forecast chunks
overflow and are cut."""
import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _scene(wl):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, None)


def _case(name):
    from delta_ray_b200 import workloads
    if name == "soft_shadow":
        return workloads.soft_shadow(3, (64, 48), 4, 1)
    # 64 x 64 vertices: 7,938 triangles, edge trees walked in two stages
    return workloads.heightfield(seed=2, resolution=(48, 40), spp=2, max_bounces=2, grid=64, patch=16)


@pytest.mark.parametrize("name", ["soft_shadow", "heightfield"])
def test_streamed_edge_stage_matches_one_pass(name):
    from delta_ray_b200.render_pytorch import set_item_queue_limit
    wl = _case(name)
    W, H = wl.resolution
    d_image = torch.from_numpy(np.random.default_rng(5).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)).cuda()

    def call(sc):
        g, img = sc.backward(W, H, wl.spp, wl.max_bounces, 11, d_image, want_image=True)
        return g.cpu().numpy(), img.cpu().numpy(), tuple(sc.last_counts())

    sc = _scene(wl)
    try:
        g0, img0, counts = call(sc)
        if name == "heightfield":
            assert sc.last_work()["tasks"] > 0  # subtrees handed to the second stage
        items = counts[1]
        # forecast from the unbounded call's edges per point
        set_item_queue_limit(max(1024, items // 6))
        g, img, c = call(sc)
        assert c == counts and np.array_equal(img, img0) and rel_err(g, g0) < 1e-5
    finally:
        set_item_queue_limit(0)
        sc.close()
    for div in (5, 40):
        set_item_queue_limit(max(1024, items // div))
        sc = _scene(wl)  # fresh statistics: the first call plans from its own full pass
        try:
            for k in range(2):  # then from the first call's counts per range of points
                g, img, c = call(sc)
                assert c == counts, (div, k)
                assert np.array_equal(img, img0)
                assert rel_err(g, g0) < 1e-5, (div, k)
        finally:
            set_item_queue_limit(0)
            sc.close()


def test_first_call_probe_forecasts_the_edge_counts():
    """A scene's first call of 2^20 or more pixel samples has no edge counts
    to plan its edge stage from: it walks every 32nd shading point first and
    forecasts the others' counts from theirs.  With room for the forecast it
    then walks every point in one pass; without (a bounded item queue) it
    streams chunks planned from the forecast, cutting those that overflow.
    Either way the call gives the results of a later call on the same scene,
    which plans from its predecessor's counts."""
    from delta_ray_b200 import workloads
    from delta_ray_b200.render_pytorch import set_item_queue_limit
    wl = workloads.heightfield(seed=3, resolution=(256, 256), spp=16, max_bounces=1, grid=32, patch=8)
    W, H = wl.resolution
    assert W * H * wl.spp >= 1 << 20
    d_image = torch.from_numpy(np.random.default_rng(7).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)).cuda()

    def call(sc):
        g, img = sc.backward(W, H, wl.spp, wl.max_bounces, 13, d_image, want_image=True)
        return g.cpu().numpy(), img.cpu().numpy(), tuple(sc.last_counts())

    sc = _scene(wl)
    try:
        g1, img1, c1 = call(sc)  # probe, then one pass
        g0, img0, counts = call(sc)  # planned from the first call's counts
        assert c1 == counts and np.array_equal(img1, img0) and rel_err(g1, g0) < 1e-5
    finally:
        sc.close()
    items = counts[1]
    for div in (3, 12):
        set_item_queue_limit(max(1 << 16, items // div))
        sc = _scene(wl)
        try:
            g, img, c = call(sc)  # probe, then chunks from its forecast
            assert c == counts, div
            assert np.array_equal(img, img0), div
            assert rel_err(g, g0) < 1e-5, div
        finally:
            set_item_queue_limit(0)
            sc.close()
