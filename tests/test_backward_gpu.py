"""Backward parity on the GPU: every gradient against the oracle.

The oracle (tape AD, Philox streams) and the CUDA backward draw the same random
numbers, so the flat gradient (camera, materials, vertices, normals, lights)
must agree.  The tolerance covers float round-off of a different summation
order plus the rare sample whose branch a transcendental function's last bit
decides differently on the GPU.
"""
import numpy as np
import pytest
import torch

from conftest import build_golden_scene, golden_cases, load_golden, rel_err
import oracle

pytestmark = pytest.mark.gpu

TOL = 2e-3
# mirror_hall's lobes raise a cosine to the power 2 / roughness = 667 at five
# bounces in a row, so the GPU's FMA contraction and transcendental last bits
# are amplified several hundred fold (the same kernel logic compiled for the CPU
# matches the oracle to 5e-5)
CASE_TOL = {"mirror_hall": 6e-3}


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
    assert np.isfinite(grad).all()
    assert rel_err(grad, o["grad"]) < CASE_TOL.get(case, TOL)
    assert sc.launch_count() >= 4


def test_backward_larger_image_matches_oracle():
    """A larger image: more points, items and primary-edge samples per launch."""
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(seed=0, resolution=(64, 48), spp=4)
    dimg = np.random.default_rng(3).uniform(0.5, 1.5, (48, 64, 3)).astype(np.float32)
    sc = product_scene(wl)
    grad, _ = sc.backward(64, 48, 4, 1, 21, torch.from_numpy(dimg))
    o_all = oracle.oracle_render(wl, 21, dimg, rng_mode=oracle.PHILOX)
    assert rel_err(grad.cpu().numpy(), o_all["grad"]) < TOL


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
    assert rel_err(gv.numpy(), ref["d_vertices"][0]) < TOL
    assert rel_err(wl.lights[0].intensity.grad.numpy(), ref["d_intensity"][0]) < TOL


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
        # the edge culling bound raises cosines to the power 2 / roughness
        # (667): the GPU's last bits of powf decide a few rare edges differently
        assert points == o["stats"][0] and abs(items - o["stats"][1]) <= 0.005 * o["stats"][1]
        assert points > 2 * W * H * 2
        assert rel_err(grad.cpu().numpy(), o["grad"]) < TOL
        grad2, _ = sc.backward(W, H, 2, 5, 8, torch.from_numpy(dimg), opts)
        assert sc.launch_count() <= first_launches
        assert rel_err(grad2.cpu().numpy(), o["grad"]) < TOL
    sc.close()
