"""Forward parity on the GPU: the CUDA renderer against the oracle.

Both sides draw from the same Philox streams and evaluate the same float
operations in the same order (no FMA contraction; the same reproducible
transcendental functions), so each pixel sample takes the same branches and
gives the same radiance up to the order of the per-pixel sums: every pixel
must agree to 1e-4 of its value (conftest.assert_image_parity).
"""
import numpy as np
import pytest
import torch

from conftest import assert_image_parity, build_golden_scene, golden_cases, load_golden
import oracle

pytestmark = pytest.mark.gpu

REL = 1e-4


def product_scene(wl, ltc=None):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, ltc)


@pytest.mark.parametrize("case", golden_cases())
def test_forward_matches_oracle(case, ltc_table):
    meta, _ = load_golden(case)
    wl = build_golden_scene(meta)
    W, H = wl.resolution
    sc = product_scene(wl, ltc_table)
    img = sc.forward(W, H, wl.spp, wl.max_bounces, meta["seed"]).cpu().numpy()
    ref = oracle.oracle_render(wl, meta["seed"], rng_mode=oracle.PHILOX, ltc_table=ltc_table)["image"]
    assert_image_parity(img, ref)


def test_forward_larger_image_matches_oracle():
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(seed=0, resolution=(96, 80), spp=8)
    sc = product_scene(wl)
    img = sc.forward(96, 80, 8, 1, 42).cpu().numpy()
    ref = oracle.oracle_render(wl, 42, rng_mode=oracle.PHILOX)["image"]
    assert_image_parity(img, ref)


def test_hit_ids_match_oracle():
    """Closest-hit triangle ids agree with the oracle's BVH on random rays."""
    import scenes
    wl = scenes.heightfield_small(seed=1, grid=40)
    rng = np.random.default_rng(0)
    n = 20000
    # rays from above aimed at the surface, plus random directions (misses, grazing hits)
    o = rng.uniform([-6, 2, -6], [6, 8, 6], (n, 3))
    target = np.stack([rng.uniform(-5, 5, n), rng.uniform(-0.5, 0.5, n), rng.uniform(-5, 5, n)], 1)
    d = target - o
    d[n // 2:] = rng.normal(size=(n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    sc = product_scene(wl)
    tri, t = sc.trace(torch.from_numpy(rays))
    tri, t = tri.cpu().numpy(), t.cpu().numpy()
    sh, lt, tr = oracle.trace(wl, rays)
    # oracle ids are (shape, local triangle); product ids are global
    offs = np.cumsum([0] + [s.indices.shape[0] for s in wl.shapes])
    gid = np.where(sh >= 0, offs[np.maximum(sh, 0)] + lt, -1)
    hits = (gid >= 0).sum()
    assert hits > n // 2
    same = gid == tri
    # a mismatch is only allowed as a tie: same distance to float round-off
    tie = np.isclose(t, tr, rtol=1e-5, atol=1e-6) & ~same
    assert (same | tie).all(), f"{(~(same | tie)).sum()} rays hit different triangles"
    assert same.mean() > 0.999


def test_hit_ids_match_oracle_linear_scan():
    """Scenes of at most 16 triangles are traced by testing every triangle:
    the soft-shadow scene's 8 triangles against the oracle's BVH."""
    from delta_ray_b200 import workloads
    from scenes import scene_rays
    wl = workloads.soft_shadow(seed=3, resolution=(32, 32), spp=1, max_bounces=1)
    rays = scene_rays(wl, 20000, seed=0)
    sc = product_scene(wl)
    tri, t = sc.trace(torch.from_numpy(rays))
    tri, t = tri.cpu().numpy(), t.cpu().numpy()
    sh, lt, tr = oracle.trace(wl, rays)
    offs = np.cumsum([0] + [s.indices.shape[0] for s in wl.shapes])
    gid = np.where(sh >= 0, offs[np.maximum(sh, 0)] + lt, -1)
    assert (gid >= 0).mean() > 0.15
    same = gid == tri
    tie = np.isclose(t, tr, rtol=1e-5, atol=1e-6) & ~same
    assert (same | tie).all(), f"{(~(same | tie)).sum()} rays hit different triangles"
    assert same.mean() > 0.999


def test_hit_ids_match_oracle_on_the_glossy_heightfield_mesh():
    """The deep LBVH of the glossy heightfield configuration's mesh (130,054
    triangles): 40,000 rays, half aimed at the surface from above, half
    grazing it from just above, against the oracle's own BVH.  A different
    id is only allowed where both hits lie at the same distance (a tie
    between triangles sharing an edge, where each BVH keeps the lower id of
    the candidates it reached)."""
    from delta_ray_b200 import workloads
    wl = workloads.heightfield(seed=0, resolution=(32, 24), spp=1)
    rng = np.random.default_rng(7)
    n = 20000
    o = rng.uniform([-6, 2, -6], [6, 8, 6], (n, 3))
    target = np.stack([rng.uniform(-5, 5, n), rng.uniform(-0.5, 0.5, n), rng.uniform(-5, 5, n)], 1)
    d = target - o
    og = np.stack([rng.uniform(-5, 5, n), rng.uniform(0.3, 0.8, n), rng.uniform(-5, 5, n)], 1)
    dg = np.stack([rng.normal(size=n), rng.uniform(-0.15, -0.02, n), rng.normal(size=n)], 1)
    o, d = np.concatenate([o, og]), np.concatenate([d, dg])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    sc = product_scene(wl)
    tri, t = sc.trace(torch.from_numpy(rays))
    tri, t = tri.cpu().numpy(), t.cpu().numpy()
    sh, lt, tr = oracle.trace(wl, rays)
    offs = np.cumsum([0] + [s.indices.shape[0] for s in wl.shapes])
    gid = np.where(sh >= 0, offs[np.maximum(sh, 0)] + lt, -1)
    assert (gid >= 0).mean() > 0.5
    same = gid == tri
    tie = (t == tr) & (gid >= 0) & (tri >= 0) & ~same
    assert (same | tie).all(), f"{(~(same | tie)).sum()} rays hit different triangles"
    assert same.mean() > 0.999
    assert np.array_equal(t[same & (gid >= 0)], tr[same & (gid >= 0)])
