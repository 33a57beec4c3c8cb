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
