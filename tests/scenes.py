"""Small scenes for the parity tests (beyond the benchmark workloads).

Each builder returns a ``delta_ray_b200.workloads.Workload`` that exercises a
feature of the reference path: the Blinn-Phong lobe and its LTC edge sampling
(material.h:257-489), textures with uv scaling (material.h:108-239), two-sided
materials (pathtrace.h:116-133, material.h:264-268), shading normals and the
directional edge tree (intersect.h:128-141, edge_tree.cpp:219-250), and the
fisheye camera (camera.h:51-71).
"""
import numpy as np
import torch

from delta_ray_b200 import workloads
from delta_ray_b200.light import Light
from delta_ray_b200.material import Material
from delta_ray_b200.shape import Shape

_t = workloads._t


def glossy_shadow(seed=0, resolution=(48, 40), spp=2, max_bounces=2):
    wl = workloads.soft_shadow(seed, resolution, spp, max_bounces)
    rng = np.random.default_rng(seed + 100)
    for m in wl.materials[:2]:
        m.specular_reflectance = _t(rng.uniform(0.2, 0.6, 3))
        m.roughness = _t([rng.uniform(0.05, 0.4)])
    wl.materials[0].two_sided = True
    wl.name = "glossy_shadow"
    return wl


def textured(seed=0, resolution=(40, 40), spp=2, max_bounces=2):
    wl = workloads.soft_shadow(seed, resolution, spp, max_bounces)
    rng = np.random.default_rng(seed + 200)
    ground = wl.shapes[0]
    v = ground.vertices.numpy()
    uv = ((v[:, [0, 2]] + 5.0) / 10.0).astype(np.float32)
    ground.uvs = _t(uv)
    m = wl.materials[0]
    m.diffuse_reflectance = _t(rng.uniform(0.2, 0.9, (8, 8, 3)))
    m.specular_reflectance = _t(rng.uniform(0.0, 0.3, (4, 4, 3)))
    m.roughness = _t(rng.uniform(0.1, 0.6, (4, 4, 1)))
    m.diffuse_uv_scale = _t([1.5, 2.0])
    m.specular_uv_scale = m.diffuse_uv_scale
    m.roughness_uv_scale = m.diffuse_uv_scale
    wl.name = "textured"
    return wl


def _icosphere(subdiv):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t],
         [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
         [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
         [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    v = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    for _ in range(subdiv):
        cache, nf = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = nf
    return np.array(v, np.float32), np.array(f, np.int32)


def smooth_sphere(seed=0, resolution=(40, 40), spp=2, max_bounces=1, subdiv=1):
    """An icosphere with per-vertex shading normals on a ground plane."""
    wl = workloads.soft_shadow(seed, resolution, spp, max_bounces)
    v, f = _icosphere(subdiv)
    center = np.array([0.3, 1.2, 0.2], np.float32)
    verts = (v * 1.0 + center).astype(np.float32)
    wl.shapes[1] = Shape(_t(verts), _t(f, np.int32), None, _t(v), 1)
    wl.materials[1].specular_reflectance = _t([0.3, 0.3, 0.3])
    wl.materials[1].roughness = _t([0.2])
    wl.name = "smooth_sphere"
    return wl


def fisheye(seed=0, resolution=(32, 32), spp=2, max_bounces=1):
    wl = workloads.soft_shadow(seed, resolution, spp, max_bounces)
    res = wl.resolution
    wl.camera = workloads._camera([0, 6, -6], [0, 0, 0], [0, 1, 0], 45.0, res, fisheye=True)
    wl.name = "fisheye"
    return wl


def heightfield_small(seed=0, resolution=(40, 32), spp=2, max_bounces=2, grid=10):
    wl = workloads.heightfield(seed, resolution, spp, max_bounces, grid=grid, patch=grid)
    wl.name = "heightfield_small"
    return wl


def mirror_shadow(seed=0, resolution=(48, 40), spp=2, max_bounces=3):
    """soft_shadow over a near-mirror ground (roughness 0.005: the reference's
    "specular" samples, material.h:410) under a two-sided near-mirror blocker,
    with a diffuse back wall carrying vertex normals.  Paths run camera ->
    ground -> blocker / wall through chains of specular vertices, which are
    secondary-edge shading points (pathtrace.h:218-227)."""
    wl = workloads.soft_shadow(seed, resolution, spp, max_bounces)
    g = wl.materials[0]
    g.diffuse_reflectance = _t([0.15, 0.15, 0.15])
    g.specular_reflectance = _t([0.7, 0.7, 0.7])
    g.roughness = _t([0.005])
    b = wl.materials[1]
    b.diffuse_reflectance = _t([0.2, 0.1, 0.1])
    b.specular_reflectance = _t([0.6, 0.6, 0.5])
    b.roughness = _t([0.008])
    b.two_sided = True
    wl.materials.append(Material(diffuse_reflectance=_t([0.6, 0.5, 0.4])))
    wv, wi = workloads._quad([0, 4, 4], 5.0, 4.0, [1, 0, 0], [0, 1, 0], normal=[0, 0, -1])
    rng = np.random.default_rng(seed + 300)
    wn = np.tile([0.0, 0.0, -1.0], (4, 1)) + rng.uniform(-0.2, 0.2, (4, 3))
    wn = (wn / np.linalg.norm(wn, axis=1, keepdims=True)).astype(np.float32)
    wl.shapes.append(Shape(_t(wv), _t(wi, np.int32), None, _t(wn), len(wl.materials) - 1))
    wl.name = "mirror_shadow"
    return wl


def mirror_hall(seed=0, resolution=(32, 24), spp=2, max_bounces=5):
    """Two facing mirrors (no diffuse lobe, roughness 0.003: every sample is
    "specular", material.h:353-412) over a diffuse ground with a blocker and
    an overhead light.  Camera paths bounce between the mirrors, so a pixel
    sample has up to max_bounces shading points (pathtrace.h:218-227)."""
    rng = np.random.default_rng(seed)
    res = [int(resolution[0]), int(resolution[1])]
    cam = workloads._camera([0, 2, -5], [2, 1.8, -3.5], [0, 1, 0], 60.0, res)
    mats = [Material(diffuse_reflectance=_t(rng.uniform(0.3, 0.8, 3))),
            Material(diffuse_reflectance=_t([0.0, 0.0, 0.0]), specular_reflectance=_t([0.85, 0.9, 0.8]),
                     roughness=_t([0.003])),
            Material(diffuse_reflectance=_t(rng.uniform(0.3, 0.8, 3))),
            Material(diffuse_reflectance=_t([0.0, 0.0, 0.0]))]
    gv, gi = workloads._quad([0, 0, 0], 5.0, 6.0, [1, 0, 0], [0, 0, 1], normal=[0, 1, 0])
    m0v, m0i = workloads._quad([-2, 2, 0], 6.0, 2.0, [0, 0, 1], [0, 1, 0], normal=[1, 0, 0])
    m1v, m1i = workloads._quad([2, 2, 0], 6.0, 2.0, [0, 0, 1], [0, 1, 0], normal=[-1, 0, 0])
    bv = np.array([[-0.6, 1.2, -0.6], [0.6, 1.2, -0.6], [0.6, 1.2, 0.6], [-0.6, 1.2, 0.6], [0.0, 1.2, 0.0]])
    bv = (bv + rng.uniform(-0.2, 0.2, size=bv.shape)).astype(np.float32)
    bi = np.array([[4, 1, 0], [4, 2, 1], [4, 3, 2], [4, 0, 3]], np.int32)
    lv, li = workloads._quad([0, 4.5, 0.5], 1.0, 1.0, [1, 0, 0], [0, 0, 1], normal=[0, -1, 0])
    shapes = [Shape(_t(gv), _t(gi, np.int32), None, None, 0),
              Shape(_t(m0v), _t(m0i, np.int32), None, None, 1),
              Shape(_t(m1v), _t(m1i, np.int32), None, None, 1),
              Shape(_t(bv), _t(bi, np.int32), None, None, 2),
              Shape(_t(lv), _t(li, np.int32), None, None, 3)]
    lights = [Light(4, _t([20.0, 20.0, 20.0]))]
    return workloads.Workload("mirror_hall", cam, mats, shapes, lights, res, int(spp), int(max_bounces),
                              {"seed": seed})


def ggx_shadow(seed=0, resolution=(48, 40), spp=2, max_bounces=2):
    """glossy_shadow with GGX lobes (no counterpart in the reference)."""
    wl = glossy_shadow(seed, resolution, spp, max_bounces)
    for m in wl.materials[:2]:
        m.microfacet = 1
    wl.name = "ggx_shadow"
    return wl


def ggx_textured(seed=0, resolution=(40, 40), spp=2, max_bounces=2):
    """textured with a GGX lobe: textured roughness and specular reflectance."""
    wl = textured(seed, resolution, spp, max_bounces)
    wl.materials[0].microfacet = 1
    wl.name = "ggx_textured"
    return wl


def ggx_heightfield(seed=0, resolution=(40, 32), spp=2, max_bounces=2):
    """A 10 x 10-vertex heightfield in 4 patches with GGX lobes."""
    wl = workloads.heightfield(seed=seed, resolution=resolution, spp=spp, max_bounces=max_bounces, grid=10,
                               patch=5, microfacet="ggx")
    wl.name = "ggx_heightfield"
    return wl


def icosphere_room(seed=0, resolution=(48, 40), spp=2, max_bounces=2, n_spheres=12, subdiv=(1, 2)):
    """A closed box room (12 triangles, 10 units a side, facing inwards) with
    a ceiling light and seeded icospheres (subdivision levels in `subdiv`,
    radii U(0.3, 1.2), shading normals): a reduced stand-in for the batched
    multi-view configuration (200 spheres of levels 3-5, about 1M triangles)."""
    rng = np.random.default_rng(seed)
    res = [int(resolution[0]), int(resolution[1])]
    cam = workloads._camera([0, 5, -4.5], [0, 3, 0], [0, 1, 0], 60.0, res)
    mats = [Material(diffuse_reflectance=_t([0.6, 0.6, 0.55])), Material(diffuse_reflectance=_t([0.0, 0.0, 0.0]))]
    shapes = []
    h = 5.0
    walls = [([0, 0, 0], [1, 0, 0], [0, 0, 1], [0, 1, 0]), ([0, 2 * h, 0], [1, 0, 0], [0, 0, 1], [0, -1, 0]),
             ([-h, h, 0], [0, 0, 1], [0, 1, 0], [1, 0, 0]), ([h, h, 0], [0, 0, 1], [0, 1, 0], [-1, 0, 0]),
             ([0, h, -h], [1, 0, 0], [0, 1, 0], [0, 0, 1]), ([0, h, h], [1, 0, 0], [0, 1, 0], [0, 0, -1])]
    for c, ax, ay, nrm in walls:
        v, f = workloads._quad(c, h, h, ax, ay, normal=nrm)
        shapes.append(Shape(_t(v), _t(f, np.int32), None, None, 0))
    lv, lf = workloads._quad([0, 2 * h - 0.01, 0], 1.5, 1.5, [1, 0, 0], [0, 0, 1], normal=[0, -1, 0])
    shapes.append(Shape(_t(lv), _t(lf, np.int32), None, None, 1))
    lights = [Light(len(shapes) - 1, _t([12.0, 12.0, 12.0]))]
    for k in range(n_spheres):
        mats.append(Material(diffuse_reflectance=_t(rng.uniform(0.2, 0.9, 3)),
                             specular_reflectance=_t(rng.uniform(0.0, 0.4, 3)), roughness=_t([rng.uniform(0.1, 0.5)])))
        v, f = _icosphere(int(rng.integers(subdiv[0], subdiv[1] + 1)))
        r = rng.uniform(0.3, 1.2)
        c = np.array([rng.uniform(-3.5, 3.5), rng.uniform(r, 4.0), rng.uniform(-3.5, 3.5)], np.float32)
        shapes.append(Shape(_t((v * r + c).astype(np.float32)), _t(f, np.int32), None, _t(v), len(mats) - 1))
    return workloads.Workload("icosphere_room", cam, mats, shapes, lights, res, int(spp), int(max_bounces),
                              {"seed": seed})


SCENES = {"glossy_shadow": glossy_shadow, "textured": textured, "smooth_sphere": smooth_sphere,
          "fisheye": fisheye, "heightfield_small": heightfield_small, "mirror_shadow": mirror_shadow,
          "mirror_hall": mirror_hall, "icosphere_room": icosphere_room, "ggx_shadow": ggx_shadow,
          "ggx_textured": ggx_textured, "ggx_heightfield": ggx_heightfield}


def scene_rays(wl, n, seed=0):
    """n rays [n, 6] (float32): origins in a box twice the scene's size, half of
    them aimed at random points of the scene's bounding box, half in random
    directions (misses and grazing hits)."""
    v = np.concatenate([np.asarray(sh.vertices, np.float64).reshape(-1, 3) for sh in wl.shapes])
    lo, hi = v.min(0), v.max(0)
    c, e = (lo + hi) / 2, np.maximum(hi - lo, 1e-3)
    rng = np.random.default_rng(seed)
    o = rng.uniform(c - e, c + e, (n, 3))
    d = rng.uniform(lo, hi, (n, 3)) - o
    d[n // 2:] = rng.normal(size=(n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)
