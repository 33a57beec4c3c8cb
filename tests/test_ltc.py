"""The LTC fitter (delta_ray_b200/ltc_fit.cpp) and the committed fitted tables."""
import math

import numpy as np
import pytest

IDENT = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)


@pytest.mark.parametrize("model", [0, 1])
def test_committed_tables_fit_their_lobes(model):
    from delta_ray_b200 import ltc
    t = ltc.default_table(model).reshape(128 * 128, 9)
    assert np.isfinite(t).all()
    assert (t[:, 0] > 0).all() and (t[:, 4] > 0).all()
    for ir, it in [(127, 0), (64, 32), (32, 64), (16, 96), (8, 16)]:
        r, th = ir / 127, it / 127 * math.pi / 2
        fit = ltc.fit_l1(model, r, th, t[ir + it * 128], 48)
        ident = ltc.fit_l1(model, r, th, IDENT, 48)
        assert fit < 0.5 * ident + 0.02, (ir, it, fit, ident)
        if model == 1:
            assert fit < 0.1, (ir, it, fit)


def test_fitter_runs_on_a_small_table():
    from delta_ray_b200 import ltc
    m, err = ltc.fit_table(1, n=6, strata=12, iters=80, threads=2)
    assert np.isfinite(m).all() and np.isfinite(err).all()
    m = m.reshape(36, 9)
    # entry (roughness 1, normal view): close to the plain cosine
    assert ltc.fit_l1(1, 1.0, 0.0, m[5], 32) < 0.1
