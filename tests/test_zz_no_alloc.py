"""dr_render_backward_noalloc: the backward pass with its work queues in the
library's fixed per-device scratch array, called through the C ABI and
compared with dr_render_backward on the same scene, seed and adjoint.

The file name sorts last so that the test also runs after every other GPU
test in the same process, and it passes alone in a fresh process as well
(scene creation loads the module that holds the scratch array and every
kernel a backward call launches)."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_err

TOL = 1e-4  # float atomics reorder the gradient sums; the parity bound of the backward tests
DR_ERR_INVALID_ARGUMENT = 1


def _bind(L):
    from delta_ray_b200 import _abi
    L.dr_render_backward_noalloc.argtypes = [C.c_void_p, C.POINTER(_abi.dr_render_desc), C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
    L.dr_render_backward_noalloc.restype = C.c_int
    return L


def _scene(res, spp, B, seed=2):
    from delta_ray_b200 import workloads
    from delta_ray_b200.render_pytorch import Scene, unpack_args
    wl = workloads.soft_shadow(seed, res, spp, B)
    cam, mats, shps, lts, _, _, _, _ = unpack_args(wl.serialize())
    return Scene(cam, mats, shps, lts, 0, None)


def _call(L, sc, W, H, spp, B, seed, d_image, grad, img):
    """The C-ABI call alone, then a device synchronize (no torch kernel)."""
    from delta_ray_b200 import _abi
    rd = _abi.render_desc(W, H, spp, B, seed)
    st = L.dr_render_backward_noalloc(sc.handle, C.byref(rd), C.c_void_p(d_image.data_ptr()),
                                      C.c_void_p(grad.data_ptr()), C.c_void_p(img.data_ptr()), None)
    torch.cuda.synchronize()
    return st


def _noalloc(L, sc, W, H, spp, B, seed, d_image, grad=None, img=None):
    if grad is None:
        grad = torch.empty((sc.grad_total,), dtype=torch.float32, device="cuda")
    grad.fill_(float("nan"))  # the call must overwrite every entry
    if img is None:
        img = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    return _call(L, sc, W, H, spp, B, seed, d_image, grad, img), grad, img


@pytest.mark.gpu
@pytest.mark.parametrize("res,spp,B", [((32, 32), 4, 1), ((40, 24), 8, 3)])
def test_noalloc_backward_matches_backward_twice(res, spp, B):
    from delta_ray_b200 import _lib
    L = _bind(_lib.lib())
    W, H = res
    sc = _scene(res, spp, B)
    seed = 11
    gen = torch.Generator().manual_seed(5)
    d_image = torch.rand((H, W, 3), generator=gen).cuda()
    ref_grad, ref_img = sc.backward(W, H, spp, B, seed, d_image, want_image=True)
    ref_grad = ref_grad.cpu().numpy()
    assert np.abs(ref_grad).max() > 0
    grad_buf = torch.empty((sc.grad_total,), dtype=torch.float32, device="cuda")
    img_buf = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    for k in range(2):  # two calls in a row reuse the same scratch
        grad_buf.fill_(float("nan"))  # the call must overwrite every entry
        img_buf.fill_(float("nan"))
        torch.cuda.synchronize()
        # only the library's call between the two readings: a torch kernel's
        # first launch in a fresh process loads its code, which takes memory
        free_before = torch.cuda.mem_get_info()[0]
        st = _call(L, sc, W, H, spp, B, seed, d_image, grad_buf, img_buf)
        free_after = torch.cuda.mem_get_info()[0]
        assert st == 0, _lib.last_error()
        # the call takes no device memory: the free memory the driver reports is unchanged
        assert free_after == free_before, (k, free_before, free_after)
        grad, img = grad_buf, img_buf
        g = grad.cpu().numpy()
        assert np.isfinite(g).all()
        assert rel_err(g, ref_grad) < TOL
        assert np.allclose(img.cpu().numpy(), ref_img.cpu().numpy(), rtol=1e-6, atol=1e-7)
    sc.close()


@pytest.mark.gpu
def test_noalloc_backward_specular_chains():
    """Specular chains (several shading points per pixel sample) fit the
    scratch's point queue and match dr_render_backward."""
    import scenes
    from delta_ray_b200 import _abi, _lib
    from delta_ray_b200.render_pytorch import Scene, unpack_args
    L = _bind(_lib.lib())
    wl = scenes.mirror_hall(seed=4, resolution=(40, 32), spp=2, max_bounces=5)
    W, H = wl.resolution
    cam, mats, shps, lts, _, _, _, _ = unpack_args(wl.serialize())
    sc = Scene(cam, mats, shps, lts, 0, None)
    d_image = torch.rand((H, W, 3), generator=torch.Generator().manual_seed(6)).cuda()
    ref_grad, _ = sc.backward(W, H, 2, 5, 9, d_image)
    st, grad, _ = _noalloc(L, sc, W, H, 2, 5, 9, d_image)
    assert st == 0, _lib.last_error()
    assert rel_err(grad.cpu().numpy(), ref_grad.cpu().numpy()) < TOL
    sc.close()


@pytest.mark.gpu
def test_noalloc_backward_rejects_oversize_calls():
    from delta_ray_b200 import _lib
    L = _bind(_lib.lib())
    sc = _scene((32, 32), 4, 1)
    W, H, spp = 128, 128, 8  # 131072 pixel samples > 65536
    d_image = torch.ones((H, W, 3), dtype=torch.float32, device="cuda")
    st, _, _ = _noalloc(L, sc, W, H, spp, 1, 3, d_image)
    assert st == DR_ERR_INVALID_ARGUMENT
    assert "65536" in _lib.last_error()
    sc.close()


@pytest.mark.gpu
def test_noalloc_backward_streams_large_edge_stages():
    """A glossy heightfield whose shading points sample about 2,000 edges each:
    the items outgrow the fixed scratch, so the no-alloc call evaluates them in
    several passes over the points; the result must match the regular call
    (whose item queue grows instead)."""
    from delta_ray_b200 import _lib, workloads
    from delta_ray_b200.render_pytorch import Scene, unpack_args
    L = _bind(_lib.lib())
    W, H, spp, B = 32, 24, 4, 2
    wl = workloads.heightfield(0, (W, H), spp, B)  # 130,054 triangles
    cam, mats, shps, lts, _, _, _, _ = unpack_args(wl.serialize())
    sc = Scene(cam, mats, shps, lts, 0, None)
    d_image = torch.ones((H, W, 3), dtype=torch.float32, device="cuda")
    ref_grad, _ = sc.backward(W, H, spp, B, 21, d_image)
    _, ref_items = sc.last_counts()
    st, grad, _ = _noalloc(L, sc, W, H, spp, B, 21, d_image)
    assert st == 0, _lib.last_error()
    _, items = sc.last_counts()
    assert items == ref_items and items > 900_000  # more than the scratch holds at once
    assert rel_err(grad.cpu().numpy(), ref_grad.cpu().numpy()) < TOL
    sc.close()
