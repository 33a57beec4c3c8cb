"""Seeded synthetic scenes used by the benchmark and the parity tests.

Each builder returns a ``Workload`` holding package scene objects (camera,
materials, shapes, lights) plus resolution, spp and max_bounces, ready for
``RenderFunction.serialize_scene``.  Geometry follows the reference's demo
scenes (test/test_single_triangle.py, test/test_shadow.py, the heightfield
topology of heightfield_gan.py:18-33); all randomness comes from
``numpy.random.default_rng(seed)``.

* ``single_triangle``: one diffuse triangle (-1.7,1,0),(1,1,0),(-0.5,-1,0)
  with N(0, 0.05) jitter, albedo 0.5, a 1x1 emissive quad at z=+5 facing -z
  (radiance 20), pinhole camera at (0,0,-5) looking at the origin, fov 45.
  Defaults 256x256, 4 spp, max_bounces 1.
* ``soft_shadow``: 10x10 ground quad at y=0, 4-triangle blocker around y=1.5
  with U(-0.3, 0.3) offsets, albedos U(0.3, 0.8), 2x2 light quad at y=5
  (radiance 15), camera at (0,6,-6).  Defaults 512x512, 16 spp, max_bounces 1.
* ``heightfield``: 256x256-vertex grid over [-5,5]^2 (130,050 triangles), six
  seeded sinusoidal octaves of amplitude 0.3*2^-k, one Blinn-Phong material per
  32x32 patch (64 materials, roughness U(0.05, 0.5), specular 0.04-0.9) and two
  light quads (radiance 10 and 5).  Defaults 640x480, 64 spp, max_bounces 3.
"""
from dataclasses import dataclass, field

import numpy as np
import torch

from .camera import Camera
from .light import Light
from .material import Material
from .shape import Shape


@dataclass
class Workload:
    name: str
    camera: Camera
    materials: list
    shapes: list
    lights: list
    resolution: list
    spp: int
    max_bounces: int
    meta: dict = field(default_factory=dict)

    def serialize(self):
        from .render_pytorch import RenderFunction
        return RenderFunction.serialize_scene(self.camera, self.materials, self.shapes,
                                              self.lights, self.resolution, self.spp,
                                              self.max_bounces)

    @property
    def num_triangles(self):
        return int(sum(s.indices.shape[0] for s in self.shapes))


def _t(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=dtype)))


def _camera(pos, look, up, fov, resolution, fisheye=False):
    return Camera(position=_t(pos), look_at=_t(look), up=_t(up), cam_to_world=None,
                  fov=_t([fov]), clip_near=_t([0.01]), clip_far=_t([10000.0]),
                  resolution=resolution, fisheye=fisheye)


def _quad(center, half_x, half_y, axis_x, axis_y, normal):
    """Two triangles of a rectangle whose geometric normal is ``normal``."""
    c = np.asarray(center, np.float64)
    ax = np.asarray(axis_x, np.float64) * half_x
    ay = np.asarray(axis_y, np.float64) * half_y
    v = np.stack([c - ax - ay, c + ax - ay, c - ax + ay, c + ax + ay]).astype(np.float32)
    idx = np.array([[0, 1, 2], [1, 3, 2]], np.int32)
    n = np.cross(v[idx[0, 1]] - v[idx[0, 0]], v[idx[0, 2]] - v[idx[0, 0]])
    if np.dot(n, normal) < 0:
        idx = idx[:, [0, 2, 1]].copy()
    return v, idx


def single_triangle(seed=0, resolution=(256, 256), spp=4, max_bounces=1):
    rng = np.random.default_rng(seed)
    res = [int(resolution[0]), int(resolution[1])]
    cam = _camera([0, 0, -5], [0, 0, 0], [0, 1, 0], 45.0, res)
    tri = np.array([[-1.7, 1.0, 0.0], [1.0, 1.0, 0.0], [-0.5, -1.0, 0.0]])
    tri = (tri + rng.normal(0.0, 0.05, size=tri.shape)).astype(np.float32)
    mat = Material(diffuse_reflectance=_t([0.5, 0.5, 0.5]))
    lv, li = _quad([0, 0, 5], 0.5, 0.5, [1, 0, 0], [0, 1, 0], normal=[0, 0, -1])
    shapes = [Shape(_t(tri), _t([[0, 1, 2]], np.int32), None, None, 0),
              Shape(_t(lv), _t(li, np.int32), None, None, 0)]
    lights = [Light(1, _t([20.0, 20.0, 20.0]))]
    return Workload("single_triangle", cam, [mat], shapes, lights, res, int(spp),
                    int(max_bounces), {"seed": seed})


def soft_shadow(seed=0, resolution=(512, 512), spp=16, max_bounces=1):
    rng = np.random.default_rng(seed)
    res = [int(resolution[0]), int(resolution[1])]
    cam = _camera([0, 6, -6], [0, 0, 0], [0, 1, 0], 45.0, res)
    mats = [Material(diffuse_reflectance=_t(rng.uniform(0.3, 0.8, 3))),
            Material(diffuse_reflectance=_t(rng.uniform(0.3, 0.8, 3))),
            Material(diffuse_reflectance=_t([0.0, 0.0, 0.0]))]
    gv, gi = _quad([0, 0, 0], 5.0, 5.0, [1, 0, 0], [0, 0, 1], normal=[0, 1, 0])
    # 4-triangle fan around a centre vertex, lifted to y = 1.5 and jittered.
    bv = np.array([[-1.0, 1.5, -1.0], [1.0, 1.5, -1.0], [1.0, 1.5, 1.0],
                   [-1.0, 1.5, 1.0], [0.0, 1.5, 0.0]])
    bv = (bv + rng.uniform(-0.3, 0.3, size=bv.shape)).astype(np.float32)
    bi = np.array([[4, 1, 0], [4, 2, 1], [4, 3, 2], [4, 0, 3]], np.int32)
    lv, li = _quad([0, 5, 0], 1.0, 1.0, [1, 0, 0], [0, 0, 1], normal=[0, -1, 0])
    shapes = [Shape(_t(gv), _t(gi, np.int32), None, None, 0),
              Shape(_t(bv), _t(bi, np.int32), None, None, 1),
              Shape(_t(lv), _t(li, np.int32), None, None, 2)]
    lights = [Light(2, _t([15.0, 15.0, 15.0]))]
    return Workload("soft_shadow", cam, mats, shapes, lights, res, int(spp),
                    int(max_bounces), {"seed": seed})


def heightfield(seed=0, resolution=(640, 480), spp=64, max_bounces=3, grid=256,
                patch=32, microfacet="blinn_phong"):
    """Glossy heightfield; one shape (and material) per ``patch`` x ``patch`` block.

    ``microfacet`` picks the patches' specular lobe: "blinn_phong" (the
    reference's material model) or "ggx"."""
    rng = np.random.default_rng(seed)
    res = [int(resolution[0]), int(resolution[1])]
    cam = _camera([0, 7, -9], [0, 0, 0], [0, 1, 0], 45.0, res)
    xs = np.linspace(-5.0, 5.0, grid)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    H = np.zeros_like(X)
    for k in range(6):
        amp = 0.3 * 2.0 ** (-k)
        freq = rng.uniform(0.5, 1.5, 2) * (2.0 ** k)
        phase = rng.uniform(0, 2 * np.pi, 2)
        H += amp * np.sin(freq[0] * X + phase[0]) * np.sin(freq[1] * Z + phase[1])
    npatch = (grid - 1 + patch - 1) // patch
    mats, shapes = [], []
    gidx = np.arange(grid * grid).reshape(grid, grid)
    patch_grid_index = []  # per patch shape: the grid index of each of its vertices
    for pj in range(npatch):
        for pi in range(npatch):
            i0, i1 = pi * patch, min((pi + 1) * patch, grid - 1)
            j0, j1 = pj * patch, min((pj + 1) * patch, grid - 1)
            sub = np.stack([X[j0:j1 + 1, i0:i1 + 1], H[j0:j1 + 1, i0:i1 + 1],
                            Z[j0:j1 + 1, i0:i1 + 1]], -1).reshape(-1, 3)
            patch_grid_index.append(gidx[j0:j1 + 1, i0:i1 + 1].reshape(-1))
            w = i1 - i0 + 1
            idx = []
            for j in range(j1 - j0):
                for i in range(i1 - i0):
                    a = j * w + i
                    idx.append([a, a + w, a + 1])
                    idx.append([a + 1, a + w, a + w + 1])
            spec = rng.uniform(0.04, 0.9)
            mats.append(Material(diffuse_reflectance=_t(rng.uniform(0.2, 0.7, 3)),
                                 specular_reflectance=_t([spec, spec, spec]),
                                 roughness=_t([rng.uniform(0.05, 0.5)]), microfacet=microfacet))
            shapes.append(Shape(_t(sub), _t(np.array(idx, np.int32), np.int32), None, None,
                                len(mats) - 1))
    mats.append(Material(diffuse_reflectance=_t([0.0, 0.0, 0.0])))
    black = len(mats) - 1
    l0v, l0i = _quad([-2.5, 6.0, 0.0], 1.0, 1.0, [1, 0, 0], [0, 0, 1], normal=[0, -1, 0])
    l1v, l1i = _quad([3.0, 5.0, 2.0], 0.75, 0.75, [1, 0, 0], [0, 0, 1], normal=[0, -1, 0])
    shapes.append(Shape(_t(l0v), _t(l0i, np.int32), None, None, black))
    shapes.append(Shape(_t(l1v), _t(l1i, np.int32), None, None, black))
    lights = [Light(len(shapes) - 2, _t([10.0, 10.0, 10.0])),
              Light(len(shapes) - 1, _t([5.0, 5.0, 5.0]))]
    # meta: the height grid and how the patches' vertices map onto it (the
    # inverse-rendering loop optimises the grid's heights)
    return Workload("heightfield", cam, mats, shapes, lights, res, int(spp),
                    int(max_bounces), {"seed": seed, "grid": grid, "patch": patch,
                                       "heights": H.astype(np.float32), "patch_grid_index": patch_grid_index})


BUILDERS = {"single_triangle": single_triangle, "soft_shadow": soft_shadow,
            "heightfield": heightfield}
