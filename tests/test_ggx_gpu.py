"""GGX lobes on the GPU: parity with the oracle's GGX restatement (the
reference has no GGX) and gradients of the GGX parameters against central
finite differences (common random numbers, sub-pixel samples over the whole
pixel, every sampled edge's position derivative summed, the BSDF sampling pdf
held constant: DR_FLAG_DETACHED_PDF)."""
import numpy as np
import pytest
import torch

from conftest import assert_grad_parity, assert_image_parity, rel_err
import oracle

pytestmark = pytest.mark.gpu


def _scene(wl, ltc, ggx):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, None if ltc is None else torch.from_numpy(ltc), torch.from_numpy(ggx))


@pytest.mark.parametrize("builder", ["ggx_shadow", "ggx_textured"])
def test_ggx_matches_oracle(builder, ltc_table):
    import scenes
    from delta_ray_b200 import ltc
    ggx = ltc.default_table(ltc.GGX)
    wl = scenes.SCENES[builder](seed=9, resolution=(40, 32), spp=4, max_bounces=2)
    W, H = wl.resolution
    d_image = np.random.default_rng(4).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = _scene(wl, ltc_table, ggx)
    img = sc.forward(W, H, wl.spp, wl.max_bounces, 31).cpu().numpy()
    grad, _ = sc.backward(W, H, wl.spp, wl.max_bounces, 31, torch.from_numpy(d_image).cuda())
    o = oracle.oracle_render(wl, 31, d_image, rng_mode=oracle.PHILOX, ltc_table=ltc_table, ltc_table_ggx=ggx)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    # the forward against the oracle's forward: the oracle's backward values
    # divide through the reciprocal (autodiff.h:161-180), and a GGX peak at
    # low roughness (k = z^2 (A - 1) + 1 near 0) turns that rounding into
    # ~1e-3 on a sample
    of = oracle.oracle_render(wl, 31, None, rng_mode=oracle.PHILOX, ltc_table=ltc_table, ltc_table_ggx=ggx)
    assert_image_parity(img, of["image"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()


@pytest.mark.parametrize("seed", [31, 32])
def test_ggx_heightfield_matches_oracle(seed, ltc_table):
    """A GGX heightfield (10 x 10 vertices, 4 patches, roughness 0.05-0.5).
    Its shading points sample ~50 edges each among many nearly coplanar
    triangles, where a single edge-tree choice decided differently would
    move the gradient of a vertex by a lot; counts and every gradient entry
    against the oracle."""
    import scenes
    from delta_ray_b200 import ltc
    ggx = ltc.default_table(ltc.GGX)
    wl = scenes.SCENES["ggx_heightfield"](seed=9, resolution=(40, 32), spp=4, max_bounces=2)
    W, H = wl.resolution
    d_image = np.random.default_rng(4).uniform(0.5, 1.5, (H, W, 3)).astype(np.float32)
    sc = _scene(wl, ltc_table, ggx)
    grad, _ = sc.backward(W, H, wl.spp, wl.max_bounces, seed, torch.from_numpy(d_image).cuda())
    o = oracle.oracle_render(wl, seed, d_image, rng_mode=oracle.PHILOX, ltc_table=ltc_table, ltc_table_ggx=ggx)
    assert tuple(sc.last_counts()) == tuple(o["stats"])
    assert_grad_parity(grad.cpu().numpy(), o["grad"])
    sc.close()


def _ggx_ground(roughness=0.3):
    from delta_ray_b200 import workloads
    wl = workloads.soft_shadow(2, (96, 96), 32, 1)
    m = wl.materials[0]
    m.microfacet = 1
    m.specular_reflectance = torch.tensor([0.4, 0.4, 0.4])
    m.roughness = torch.tensor([roughness])
    return wl


def _jitter(wl, seed, ggx, d_image=None, spp=None):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import RenderOptions
    sc = _scene(wl, None, ggx)
    W, H = wl.resolution
    opts = RenderOptions(dp_mode=_abi.DR_DP_SUM, full_pixel_jitter=True, detached_pdf=True)
    try:
        if d_image is None:
            return float(sc.forward(W, H, spp or wl.spp, wl.max_bounces, seed, opts).double().sum())
        g, _ = sc.backward(W, H, wl.spp, wl.max_bounces, seed, torch.as_tensor(d_image, device="cuda"), opts)
        return g.cpu().numpy()
    finally:
        sc.close()


@pytest.mark.parametrize("param", ["roughness", "specular"])
def test_ggx_parameter_gradients_match_finite_differences(param):
    """The ground's GGX roughness and specular reflectance (summed over the
    three channels) enter the image through the lobe's value and its sampling
    pdf; the gradient and the central difference of the image sum agree."""
    import copy
    from delta_ray_b200 import ltc
    from stats_util import _grad_blocks
    ggx = ltc.default_table(ltc.GGX)
    wl = _ggx_ground()
    W, H = wl.resolution
    blocks, _ = _grad_blocks(wl)
    o, n = blocks[(param, 0)]
    base = getattr(wl.materials[0], "roughness" if param == "roughness" else "specular_reflectance").clone()
    h = 1e-2
    g, fd = [], []
    for k in range(6):
        seed = 300 + k
        g.append(_jitter(wl, seed, ggx, np.ones((H, W, 3), np.float32))[o:o + n].sum())
        vals = []
        for sgn in (1, -1):
            w2 = copy.deepcopy(wl)
            setattr(w2.materials[0], "roughness" if param == "roughness" else "specular_reflectance",
                    base + sgn * h)
            vals.append(_jitter(w2, seed, ggx, spp=wl.spp))
        fd.append((vals[0] - vals[1]) / (2 * h))
    g, fd = np.array(g), np.array(fd)
    se = np.sqrt(g.var(ddof=1) / len(g) + fd.var(ddof=1) / len(fd))
    print(param, g.mean(), fd.mean(), se)
    assert abs(g.mean() - fd.mean()) < 4 * se + 0.05 * abs(fd.mean()), (g.mean(), fd.mean(), se)
