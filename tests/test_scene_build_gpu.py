"""The GPU build of a large scene's edge data (dr_scene_build.cu) against the
host build of the same rules (dr_host_scene.h, compiled for the CPU by the
test harness): unique edges, the kept / silhouette / normal split, both edge
trees and the primary-edge sampler, compared byte for byte.

Scenes of more than 8,192 triangles build on the GPU.  Trees of more than
16,384 edges follow the product's split rule (a stable sort on the split
coordinate, exact fixed-point cone axes, total-order boxes), smaller ones the
reference's std::nth_element rule on the host; both paths are covered.  A
scene update with moved vertices reuses the edge topology and must equal a
fresh host build of the moved scene."""
import ctypes as C

import numpy as np
import pytest
import torch

from native import harness

pytestmark = pytest.mark.gpu

ARRAYS = ("sil_nodes", "sil_edges", "nrm_nodes", "nrm_edges", "prim_edges", "prim_cdf", "prim_func",
          "prim_func_int")


def _scene(wl):
    from delta_ray_b200 import _abi
    from delta_ray_b200.render_pytorch import Scene
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return Scene(cam, mats, shps, lts, 0, None)


def device_edges(sc, what):
    from delta_ray_b200 import _lib
    L = _lib.lib()
    code, elem = harness.EDGE_DATA[what]
    n = C.c_int64()
    ms = C.c_float()
    _lib.check(L.dr_scene_edge_data(sc.handle, code, None, 0, C.byref(n), C.byref(ms)))
    buf = np.zeros(max(1, n.value * elem), np.uint8)
    _lib.check(L.dr_scene_edge_data(sc.handle, code, C.c_void_p(buf.ctypes.data), buf.size, C.byref(n), None))
    return buf[:n.value * elem].tobytes(), ms.value


# float fields of each element (32-bit words), the rest are integers
_FLOAT_WORDS = {"sil_nodes": set(range(10)) | {12}, "nrm_nodes": set(range(10)) | {12}, "prim_cdf": {0},
                "prim_func": {0}, "prim_func_int": {0}}


def _same(what, dev, host):
    """Equal bit for bit, except that any two NaNs are equal (the silhouette
    tree's cone axes are NaN by construction, normalize(0), and the CPU and
    the GPU encode a NaN differently)."""
    if len(dev) != len(host):
        return False, -1
    elem_words = harness.EDGE_DATA[what][1] // 4
    a = np.frombuffer(dev, np.uint32).reshape(-1, elem_words)
    b = np.frombuffer(host, np.uint32).reshape(-1, elem_words)
    eq = a == b
    for w in _FLOAT_WORDS.get(what, ()):
        fa, fb = a[:, w].view(np.float32), b[:, w].view(np.float32)
        eq[:, w] |= np.isnan(fa) & np.isnan(fb)
    bad = ~eq.all(1)
    return not bad.any(), int(np.flatnonzero(bad)[0]) if bad.any() else -1


def assert_same_edge_data(sc, wl):
    sizes = {}
    for what in ARRAYS:
        dev, _ = device_edges(sc, what)
        host = harness.scene_edges(wl, what)
        elem = harness.EDGE_DATA[what][1]
        sizes[what] = len(host) // elem
        ok, first = _same(what, dev, host)
        if not ok:
            raise AssertionError(f"{what}: {len(dev) // elem} vs {len(host) // elem} elements, first difference at "
                                 f"element {first}")
    return sizes


def _moved(wl, seed):
    """The same scene with every vertex moved a little (same triangles)."""
    import copy
    w2 = copy.deepcopy(wl)
    rng = np.random.default_rng(seed)
    for s in w2.shapes:
        s.vertices = s.vertices + torch.from_numpy(rng.normal(0, 1e-3, tuple(s.vertices.shape)).astype(np.float32))
    return w2


def test_glossy_heightfield_mesh_edge_data():
    """The glossy heightfield configuration's mesh: 64 patches without shading
    normals, so ~195,000 edges form one silhouette tree (the product's rule
    on the GPU); then an update with moved vertices."""
    from delta_ray_b200 import _abi, workloads
    wl = workloads.heightfield(seed=0, resolution=(64, 48), spp=1)
    sc = _scene(wl)
    sizes = assert_same_edge_data(sc, wl)
    assert sizes["sil_edges"] > 100_000 and sizes["nrm_edges"] == 0 and sizes["prim_edges"] > 0
    _, ms = device_edges(sc, "sil_nodes")
    assert ms > 0
    w2 = _moved(wl, 1)
    cam, mats, shps, lts = _abi.scene_dicts(w2.camera, w2.materials, w2.shapes, w2.lights)
    sc.update(cam, mats, shps, lts)
    assert_same_edge_data(sc, w2)
    sc.close()


@pytest.mark.parametrize("subdiv", [(3, 3), (2, 3)])
def test_icosphere_room_edge_data(subdiv):
    """Icospheres with shading normals: a normal tree of tens of thousands of
    edges (the product's rule on the GPU, with cone axes from the fixed-point
    normal sums) beside a small silhouette tree (the room's boundary edges,
    the reference's rule on the host)."""
    import scenes
    wl = scenes.icosphere_room(seed=3, n_spheres=30, subdiv=subdiv, resolution=(48, 40), spp=1, max_bounces=1)
    assert sum(s.indices.shape[0] for s in wl.shapes) > 8192
    sc = _scene(wl)
    sizes = assert_same_edge_data(sc, wl)
    assert sizes["nrm_edges"] > 16384
    sc.close()


def test_mid_size_scene_trees_follow_the_reference_rule():
    """A scene just above the GPU-build size whose trees stay below 16,384
    edges: the GPU extracts and splits the edges, the host builds both trees
    with the reference's rule, the GPU the primary-edge sampler."""
    from delta_ray_b200 import workloads
    wl = workloads.heightfield(seed=2, resolution=(48, 32), spp=1, grid=70, patch=16)  # 9,526 triangles
    ntri = sum(s.indices.shape[0] for s in wl.shapes)
    assert 8192 < ntri
    sc = _scene(wl)
    sizes = assert_same_edge_data(sc, wl)
    assert 0 < sizes["sil_edges"] <= 16384
    sc.close()
