"""Deep paths in the checkpointed form (the path procedure's kernel logic,
compiled for the CPU).

With per-bounce records the trace keeps 32 B per bounce for the replay and
stops at 64 bounces.  The checkpointed form keeps the trace's state at the
start of every segment of bounces and traces a segment again, from the same
streams, when the suffix sweep and the replay need its records.  It must give
the same bits as the records (image, every gradient entry, the point and edge
counts) and, beyond the records' 64 bounces, the same bits for any segment
length.
"""
import numpy as np
import pytest

from native import harness


def _render(wl, seed, d_image, ckpt, ltc):
    harness.set_checkpoints(ckpt)
    try:
        return harness.render(wl, seed, d_image, ltc_table=ltc)
    finally:
        harness.set_checkpoints(0)


@pytest.mark.parametrize("name,bounces", [("glossy_shadow", 12), ("mirror_shadow", 9), ("mirror_hall", 12),
                                          ("icosphere_room", 10)])
def test_checkpointed_paths_give_the_records_bits(name, bounces, ltc_table):
    import scenes
    wl = scenes.SCENES[name](seed=4, resolution=(20, 16), spp=2, max_bounces=bounces)
    W, H = wl.resolution
    d_image = np.random.default_rng(1).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    ref = _render(wl, 17, d_image, 0, ltc_table)
    for k in (4, 16):
        got = _render(wl, 17, d_image, k, ltc_table)
        assert np.array_equal(got["image"], ref["image"]), (name, k)
        assert np.array_equal(got["grad"], ref["grad"]), (name, k)
        assert np.array_equal(got["stats"], ref["stats"]), (name, k)


def test_checkpointed_paths_go_beyond_64_bounces(ltc_table):
    """A closed room of 0.95-albedo walls: with roulette from bounce 5 (survival
    at most 0.95 per bounce) some of its paths outlive 64 bounces.  At
    max_bounces 100 the two segment lengths (8 and 16 bounces) give the same
    bits, and differ from the per-bounce records, which stop at 64.  (The
    oracle is no check here: its tape rounds every division of a path by the
    reciprocal, the kernels only where the rounding decides which edges a point
    sees, and on paths this long some roulette decision always parts.)"""
    import scenes
    wl = scenes.SCENES["icosphere_room"](seed=2, resolution=(12, 10), spp=8, max_bounces=100)
    for m in wl.materials:
        m.diffuse_reflectance = m.diffuse_reflectance * 0 + 0.95
    W, H = wl.resolution
    d_image = np.random.default_rng(3).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    a = _render(wl, 23, d_image, 8, ltc_table)
    b = _render(wl, 23, d_image, 16, ltc_table)
    assert np.array_equal(a["image"], b["image"]) and np.array_equal(a["grad"], b["grad"])
    assert np.array_equal(a["stats"], b["stats"])
    rec = _render(wl, 23, d_image, 0, ltc_table)
    assert not np.array_equal(a["image"], rec["image"])
    assert a["image"].sum() > rec["image"].sum()  # the bounces beyond 64 add light


@pytest.mark.gpu
def test_checkpointed_kernel_beyond_64_bounces_matches_the_cpu_build(ltc_table):
    """max_bounces 100 on the GPU (k_backward_paths in the checkpointed form)
    against the same per-sample logic built for the CPU: equal counts, every
    pixel and gradient entry within the parity bounds."""
    import scenes
    import torch
    from conftest import assert_grad_parity, assert_image_parity
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    wl = scenes.SCENES["icosphere_room"](seed=2, resolution=(12, 10), spp=8, max_bounces=100)
    for m in wl.materials:
        m.diffuse_reflectance = m.diffuse_reflectance * 0 + 0.95
    W, H = wl.resolution
    d_image = np.random.default_rng(3).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    cpu = _render(wl, 23, d_image, 16, ltc_table)
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sc = Scene(cam, mats, shps, lts, 0, torch.from_numpy(ltc_table))
    try:
        g, img = sc.backward(W, H, wl.spp, wl.max_bounces, 23, torch.from_numpy(d_image).cuda(), want_image=True)
        assert tuple(sc.last_counts()) == tuple(cpu["stats"])
        assert_image_parity(img.cpu().numpy(), cpu["image"])
        assert_grad_parity(g.cpu().numpy(), cpu["grad"])
    finally:
        sc.close()
