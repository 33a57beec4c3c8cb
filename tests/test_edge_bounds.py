"""The edge-tree node tests of the traversal, compiled for the CPU.

The silhouette test of a node (dr_edges.cuh: contains_silhouette) first runs a
filter in sine space and leaves only close cases to the float evaluation with
the reproducible atan and acos.  The filter must never change an answer: here
it is checked against the float evaluation alone on random nodes and points,
and on (node, point) pairs built at offsets of 1e-8 to 1e-3 rad from the
decision boundary |pi/2 - acos(c)| = angle + atan(vt), where the filter has to
step aside.
"""
import numpy as np

from native import harness


def _nodes(rng, n, max_angle):
    c = rng.uniform(-5, 5, (n, 3))
    ext = np.exp(rng.uniform(np.log(1e-3), np.log(3), (n, 3)))
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    angle = np.where(rng.random(n) < 0.2, 0.0, rng.uniform(0, max_angle, n))
    return c - ext, c + ext, axis, angle


def test_silhouette_filter_agrees_on_random_pairs():
    rng = np.random.default_rng(1)
    n = 400_000
    lo, hi, axis, angle = _nodes(rng, n, np.pi)
    p = rng.uniform(-20, 20, (n, 3))
    fast, exact = harness.silhouette(lo, hi, axis, angle, p)
    assert np.array_equal(fast, exact)
    assert 0.05 < exact.mean() < 0.95  # both answers occur


def test_silhouette_filter_agrees_at_the_boundary():
    rng = np.random.default_rng(2)
    n = 400_000
    lo, hi, axis, angle = _nodes(rng, n, 1.2)
    lo = lo.astype(np.float32).astype(np.float64)
    hi = hi.astype(np.float32).astype(np.float64)
    centre = (lo + hi) / 2
    r = np.linalg.norm(hi - centre, axis=1)
    dist = r / rng.uniform(0.05, 0.95, n)  # vt = r / dist < 1
    rng_ = angle.astype(np.float32).astype(np.float64) + np.arctan(r / dist)
    off = np.exp(rng.uniform(np.log(1e-8), np.log(1e-3), n)) * rng.choice([-1, 1], n)
    target = np.clip(rng_ + off, 0, np.pi / 2) * rng.choice([-1, 1], n)  # asin(c) on either side
    cval = np.sin(target)
    perp = rng.normal(size=(n, 3))
    perp -= (perp * axis).sum(1, keepdims=True) * axis
    perp /= np.linalg.norm(perp, axis=1, keepdims=True)
    u = cval[:, None] * axis + np.sqrt(1 - cval ** 2)[:, None] * perp  # unit, cos(axis, u) = c
    p = centre - dist[:, None] * u
    fast, exact = harness.silhouette(lo, hi, axis, angle, p)
    assert np.array_equal(fast, exact)
    assert 0.2 < exact.mean() < 0.8
