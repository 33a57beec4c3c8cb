"""Backward parity on the GPU: every gradient against the oracle.

The oracle (tape AD, Philox streams) and the CUDA backward draw the same random
numbers and evaluate the same float operations in the same order, so each
sample takes the same branches: the sets of shading points and sampled edges
are equal, and every gradient entry agrees to 1e-4 of its size (the order of
the float atomic sums is all that differs; see conftest.assert_grad_parity).
"""
import numpy as np
import pytest
import torch

from conftest import assert_grad_parity, build_golden_scene, golden_cases, load_golden
import oracle

pytestmark = pytest.mark.gpu


def product_scene(wl, ltc=None):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, ltc)


@pytest.mark.parametrize("case", golden_cases())
def test_backward_matches_oracle(case, ltc_table):
    meta, gold = load_golden(case)
    wl = build_golden_scene(meta)
    W, H = wl.resolution
    sc = product_scene(wl, ltc_table)
    grad, img = sc.backward(W, H, wl.spp, wl.max_bounces, meta["seed"], torch.from_numpy(gold["d_image"]),
                            want_image=True)
    grad = grad.cpu().numpy()
    o = oracle.oracle_render(wl, meta["seed"], gold["d_image"], rng_mode=oracle.PHILOX, ltc_table=ltc_table)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert_grad_parity(grad, o["grad"], what=case)
    assert sc.launch_count() >= 4


def test_backward_larger_image_matches_oracle():
    """A larger image: more points, items and primary-edge samples per launch."""
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(seed=0, resolution=(64, 48), spp=4)
    dimg = np.random.default_rng(3).uniform(0.5, 1.5, (48, 64, 3)).astype(np.float32)
    sc = product_scene(wl)
    grad, _ = sc.backward(64, 48, 4, 1, 21, torch.from_numpy(dimg))
    o_all = oracle.oracle_render(wl, 21, dimg, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o_all["stats"])
    assert_grad_parity(grad.cpu().numpy(), o_all["grad"])


def test_renderfunction_autograd_roundtrip():
    """RenderFunction.apply / backward through torch autograd (the drop-in path)."""
    from delta_ray_b200 import RenderFunction, workloads
    wl = workloads.single_triangle(seed=0, resolution=(48, 48), spp=4)
    wl.shapes[0].vertices.requires_grad_(True)
    wl.lights[0].intensity.requires_grad_(True)
    args = wl.serialize()
    img = RenderFunction.apply(5, *args)
    assert img.is_cuda and img.shape == (48, 48, 3)
    loss = img.sum()
    loss.backward()
    gv = wl.shapes[0].vertices.grad
    assert gv is not None and gv.device.type == "cpu" and torch.isfinite(gv).all()
    assert gv.abs().max() > 0
    ref = oracle.oracle_render(wl, 5, np.ones((48, 48, 3), np.float32), rng_mode=oracle.PHILOX)
    assert_grad_parity(gv.numpy().ravel(), np.asarray(ref["d_vertices"][0]).ravel(), what="d_vertices")
    assert_grad_parity(wl.lights[0].intensity.grad.numpy(), ref["d_intensity"][0], what="d_intensity")


def test_backward_is_deterministic_in_expectation():
    """Two seeds: gradients differ (Monte Carlo) but agree within noise."""
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(seed=0, resolution=(64, 64), spp=16)
    sc = product_scene(wl)
    d = torch.ones(64, 64, 3)
    g1, _ = sc.backward(64, 64, 16, 1, 1, d)
    g2, _ = sc.backward(64, 64, 16, 1, 2, d)
    g1, g2 = g1.cpu().numpy(), g2.cpu().numpy()
    assert not np.array_equal(g1, g2)
    big = np.abs(g1) > 0.1 * np.abs(g1).max()
    assert np.median(np.abs(g1[big] - g2[big]) / np.abs(g1[big])) < 0.5


def test_specular_chains_grow_the_point_queue():
    """Specular chains in a hall of mirrors: up to max_bounces shading points
    per pixel sample, more than the point queue starts with, so the path stage
    runs again with a grown queue; gradients in both dp modes against the
    oracle, and a second call that starts with the grown queue."""
    import scenes
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import RenderOptions
    wl = scenes.mirror_hall(seed=4, resolution=(40, 32), spp=2, max_bounces=5)
    W, H = wl.resolution
    dimg = np.random.default_rng(5).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = product_scene(wl)
    for mode in (_abi.DR_DP_REFERENCE_LAST, _abi.DR_DP_SUM):
        opts = RenderOptions(dp_mode=mode)
        grad, _ = sc.backward(W, H, 2, 5, 8, torch.from_numpy(dimg), opts)
        points, items = sc.last_counts()
        first_launches = sc.launch_count()
        o = oracle.oracle_render(wl, 8, dimg, rng_mode=oracle.PHILOX, dp_mode=mode)
        assert (points, items) == tuple(o["stats"])
        assert points > 2 * W * H * 2
        assert_grad_parity(grad.cpu().numpy(), o["grad"], what=f"dp mode {mode}")
        grad2, _ = sc.backward(W, H, 2, 5, 8, torch.from_numpy(dimg), opts)
        assert sc.launch_count() <= first_launches
        assert_grad_parity(grad2.cpu().numpy(), o["grad"], what=f"dp mode {mode}, second call")
    sc.close()


def test_single_triangle_config_at_full_size():
    """The single-triangle configuration at its configured size (256 x 256,
    4 spp, max_bounces 1, all-ones adjoint): image, work counts and every
    gradient against the oracle."""
    from delta_ray_b200 import workloads
    from conftest import assert_image_parity
    wl = workloads.single_triangle(seed=0)
    W, H = wl.resolution
    assert (W, H, wl.spp, wl.max_bounces) == (256, 256, 4, 1)
    d = np.ones((H, W, 3), np.float32)
    sc = product_scene(wl)
    grad, img = sc.backward(W, H, wl.spp, wl.max_bounces, 1, torch.from_numpy(d), want_image=True)
    o = oracle.oracle_render(wl, 1, d, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert_image_parity(img.cpu().numpy(), o["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()


def test_soft_shadow_config_at_full_size():
    """The soft-shadow configuration at its configured size (512 x 512, 16 spp,
    max_bounces 1; the benchmark's workload): 3.6 M shading points and 39 M
    sampled edges, every one the oracle's; image and gradients against the
    oracle."""
    from delta_ray_b200 import workloads
    from conftest import assert_image_parity
    wl = workloads.soft_shadow(seed=0)
    W, H = wl.resolution
    assert (W, H, wl.spp, wl.max_bounces) == (512, 512, 16, 1)
    d = np.ones((H, W, 3), np.float32)
    sc = product_scene(wl)
    grad, img = sc.backward(W, H, wl.spp, wl.max_bounces, 1, torch.from_numpy(d), want_image=True)
    o = oracle.oracle_render(wl, 1, d, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert o["stats"][1] > 30_000_000
    assert_image_parity(img.cpu().numpy(), o["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_glossy_heightfield_mesh_matches_oracle(seed):
    """The glossy heightfield configuration's full mesh (256 x 256 vertices,
    130,050 triangles plus two light quads, 64 roughness patches, max_bounces
    3) at a small image (32 x 24, 1 spp): its shading points sample ~2,000
    edges each from the large edge trees (two-stage traversal), and the rays
    walk the deep LBVH; counts, image and all 208,056 gradient entries against
    the oracle."""
    from delta_ray_b200 import workloads
    from conftest import assert_image_parity
    wl = workloads.heightfield(seed=0, resolution=(32, 24), spp=1)
    W, H = wl.resolution
    assert sum(s.indices.shape[0] for s in wl.shapes) == 130054 and wl.max_bounces == 3
    d = np.random.default_rng(seed).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = product_scene(wl)
    grad, img = sc.backward(W, H, wl.spp, wl.max_bounces, seed, torch.from_numpy(d), want_image=True)
    o = oracle.oracle_render(wl, seed, d, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert o["stats"][1] > 1_000_000
    assert_image_parity(img.cpu().numpy(), o["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()


@pytest.mark.parametrize("builder", ["glossy_shadow", "mirror_shadow", "icosphere_room"])
def test_deep_paths_match_oracle(builder):
    """Paths of up to 32 bounces (deeper than the reference's demo settings,
    which go to 16; Russian roulette from bounce 5 ends most paths earlier, the
    closed room keeps some going): each bounce's record is kept for the
    adjoint replay; counts, image and every gradient entry against the
    oracle."""
    import scenes
    from conftest import assert_image_parity
    kw = dict(n_spheres=4, subdiv=(1, 1)) if builder == "icosphere_room" else {}
    wl = scenes.SCENES[builder](seed=5, resolution=(32, 24), spp=2, max_bounces=32, **kw)
    W, H = wl.resolution
    d = np.random.default_rng(6).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = product_scene(wl)
    grad, img = sc.backward(W, H, wl.spp, 32, 41, torch.from_numpy(d), want_image=True)
    o = oracle.oracle_render(wl, 41, d, rng_mode=oracle.PHILOX)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert_image_parity(img.cpu().numpy(), o["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()
