"""The learned edge proposal on the GPU: network inference inside the
backward pass, the defensive-mixture traversal, and online training.

Unbiasedness is checked statistically: over independent seeds, the
secondary-edge gradient with the proposal has the mean of the plain
edge-tree sampling (the reference's estimator)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _scene():
    import scenes
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    wl = scenes.SCENES["heightfield_small"](seed=8, resolution=(64, 48), spp=4, max_bounces=1)
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return wl, Scene(cam, mats, shps, lts, 0, None)


def _grads(sc, wl, seeds, learned):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import RenderOptions
    W, H = wl.resolution
    opts = RenderOptions(dp_mode=_abi.DR_DP_SUM, learned_proposal=learned)
    d = torch.ones((H, W, 3), device="cuda")
    return np.stack([sc.backward(W, H, wl.spp, wl.max_bounces, s, d, opts)[0].cpu().numpy() for s in seeds])


def _zscores(a, b):
    K = a.shape[0]
    se = np.hypot(a.std(0, ddof=1), b.std(0, ddof=1)) / np.sqrt(K)
    m = se > 1e-3 * se.max()
    return (a.mean(0) - b.mean(0))[m] / se[m]


def test_untrained_proposal_is_unbiased():
    wl, sc = _scene()
    sc.set_proposal(train=False, mix=0.8)
    plain = _grads(sc, wl, range(100, 132), False)
    learned = _grads(sc, wl, range(200, 232), True)
    z = _zscores(learned, plain)
    assert z.size > 50
    assert np.sqrt((z ** 2).mean()) < 1.4 and (np.abs(z) < 3).mean() >= 0.95
    sc.close()


def test_online_training_lowers_the_loss_and_stays_unbiased():
    from delta_ray_b200 import proposal
    wl, sc = _scene()
    sc.set_proposal(train=True, mix=0.8, learning_rate=3e-3, train_points=4096,
                    params=proposal.init_params(seed=1))
    losses = []
    for s in range(40):
        _grads(sc, wl, [300 + s], True)
        losses.append(sc.proposal_state()[1])
    p, _, steps = sc.proposal_state()
    assert steps == 40 and torch.isfinite(p).all()
    assert np.mean(losses[-5:]) < 0.9 * np.mean(losses[:5]), losses
    sc.set_proposal(train=False, mix=0.8)
    plain = _grads(sc, wl, range(400, 432), False)
    learned = _grads(sc, wl, range(500, 532), True)
    z = _zscores(learned, plain)
    assert np.sqrt((z ** 2).mean()) < 1.4 and (np.abs(z) < 3).mean() >= 0.95
    sc.close()
