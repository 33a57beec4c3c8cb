"""The LBVH's 4-wide form (dr_trace.cuh: widen_node, trace_before_wide), which
the ray stage's occlusion walks take, against the binary walk on the CPU
build: the same answer for every ray, whatever the bound (ta, ida) --
before, at and beyond the ray's closest hit, ties by triangle id included."""
import numpy as np

from native import harness


def test_wide_walk_answers_as_the_binary_walk():
    import scenes
    wl = scenes.heightfield_small(seed=1, grid=40)
    rng = np.random.default_rng(3)
    n = 6000
    o = rng.uniform([-6, 2, -6], [6, 8, 6], (n, 3))
    target = np.stack([rng.uniform(-5, 5, n), rng.uniform(-0.5, 0.5, n), rng.uniform(-5, 5, n)], 1)
    d = target - o
    d[n // 3:] = rng.normal(size=(n - n // 3, 3))  # random directions: misses and grazing hits
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    tri, t, _ = harness.trace(wl, rays)
    hit = tri >= 0
    assert hit.mean() > 0.3
    # bounds: at the closest hit with its own id, with ids around it, and a little before and after it
    ta = np.where(hit, t, rng.uniform(1, 20, n)).astype(np.float32)
    scale = rng.choice([1.0, 0.999, 1.001, 0.5], n).astype(np.float32)
    ta = ta * scale
    ida = np.where(hit, tri + rng.integers(-1, 2, n), rng.integers(0, 1000, n)).astype(np.int32)
    out = harness.trace_before(wl, rays, ta, ida)
    assert np.array_equal(out[:, 0], out[:, 1]), int((out[:, 0] != out[:, 1]).sum())
    assert 0.05 < out[:, 0].mean() < 0.95  # both answers occur
