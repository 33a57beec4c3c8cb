"""Shared test setup: the `gpu` marker, import paths and golden-case helpers."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
LTC_PATH = os.path.join(ROOT, "oracle", "_ref", "ltc_tabM.f32")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


def build_golden_scene(meta):
    from golden.make_golden import build_case
    return build_case(meta["builder"], meta["kwargs"])


@pytest.fixture(scope="session")
def ltc_table():
    if not os.path.exists(LTC_PATH):
        pytest.skip("reference LTC table not built (make -C oracle ref)")
    return np.fromfile(LTC_PATH, np.float32)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(1e-30, np.abs(b).max()))


# GPU-vs-oracle gradient parity: both sides draw the same Philox samples and
# evaluate the same float operations in the same order (no FMA contraction,
# the same reproducible transcendental functions), so every branch agrees and
# only the order of the float atomic sums into each gradient entry differs.
# Each entry must agree to GRAD_REL of its own size; GRAD_FLOOR (relative to
# the largest entry) covers entries that are sums of large terms of both signs
# cancelling to nearly zero, where a reordered sum moves the last bits of the
# big terms.
GRAD_REL = 1e-4
GRAD_FLOOR = 1e-5


def assert_grad_parity(g, o, rel=GRAD_REL, floor=GRAD_FLOOR, what="gradient"):
    g = np.asarray(g, np.float64)
    o = np.asarray(o, np.float64)
    assert g.shape == o.shape and np.isfinite(g).all()
    m = float(np.abs(o).max())
    tol = rel * np.abs(o) + floor * m
    bad = np.abs(g - o) > tol
    if bad.any():
        idx = np.flatnonzero(bad)[:5]
        raise AssertionError(f"{what}: {int(bad.sum())} of {g.size} entries differ beyond {rel} relative "
                             f"(+{floor} of max {m:.4g}); first: " +
                             ", ".join(f"[{i}] {g[i]:.7g} vs {o[i]:.7g}" for i in idx))


# GPU-vs-oracle image parity: each pixel to 1e-4 of its value (plus 1e-6 of
# the image's peak for near-black pixels).
IMG_REL = 1e-4


def assert_image_parity(img, ref, rel=IMG_REL):
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    assert img.shape == ref.shape and np.isfinite(img).all()
    tol = rel * np.abs(ref) + 1e-6 * float(np.abs(ref).max()) + 1e-9
    over = np.abs(img - ref) - tol
    bad = (over > 0).any(-1)
    if bad.any():
        y, x, c = np.unravel_index(np.argmax(over), over.shape)
        raise AssertionError(f"{int(bad.sum())} of {bad.size} pixels differ beyond {rel} relative; worst at "
                             f"({x}, {y}) channel {c}: {img[y, x, c]:.9g} vs {ref[y, x, c]:.9g} "
                             f"(image peak {float(np.abs(ref).max()):.6g})")
