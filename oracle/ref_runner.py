"""Test infrastructure: drive the compiled reference renderer (oracle/_ref).

``render_reference(workload, seed, d_image=None)`` builds the reference's own
pybind11 objects from a package ``Workload`` exactly as the reference's
RenderFunction.forward does (render_pytorch.py:137-193) and calls
``delta_ray.render`` (delta_ray.cpp:1017).  ``d_image=None`` is the forward
pass (0-d adjoint, delta_ray.cpp:1029); an [H, W, 3] adjoint runs the backward
pass, which re-renders the image and returns every gradient.

Only tests, the fixture generator and bench.py's reference arm import this.
"""
import glob
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


_MODULES = {}


def load_reference(strict=False):
    """Import the compiled reference, or raise ImportError.

    strict=False: the reference's own flags (-O3 -ffast-math), used as the
    CPU baseline.  strict=True: the same sources built with IEEE arithmetic,
    used for sample-exact comparisons (fast-math flips rare branches).
    """
    if strict in _MODULES:
        return _MODULES[strict]
    d = os.path.join(REF_DIR, "strict") if strict else REF_DIR
    cands = glob.glob(os.path.join(d, "delta_ray*.so"))
    if not cands:
        raise ImportError("reference build missing: run `make -C oracle ref`")
    spec = importlib.util.spec_from_file_location("delta_ray", cands[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _MODULES[strict] = mod
    return mod


def reference_available(strict=False):
    d = os.path.join(REF_DIR, "strict") if strict else REF_DIR
    return bool(glob.glob(os.path.join(d, "delta_ray*.so")))


def _np(t):
    return np.ascontiguousarray(t.detach().cpu().numpy())


def render_reference(wl, seed, d_image=None, print_progress=False, strict=False):
    """Returns a dict with 'image' and (backward only) the gradients."""
    dr = load_reference(strict)
    cam = wl.camera
    keep = []  # the pybind objects hold numpy views: keep the arrays alive
    camera = dr.Camera(_np(cam.cam_to_world), _np(cam.world_to_cam), _np(cam.sample_to_cam),
                       _np(cam.cam_to_sample), float(cam.fov_factor.item()),
                       float(cam.aspect_ratio), float(cam.clip_near.item()), bool(cam.fisheye))
    materials = []
    for m in wl.materials:
        arrs = [_np(m.diffuse_reflectance), _np(m.specular_reflectance), _np(m.roughness),
                _np(m.diffuse_uv_scale), _np(m.specular_uv_scale), _np(m.roughness_uv_scale)]
        keep.append(arrs)
        materials.append(dr.Material(*arrs, bool(m.two_sided)))
    shapes = []
    for s in wl.shapes:
        v = _np(s.vertices)
        i = np.ascontiguousarray(_np(s.indices).astype(np.int32))
        uv = None if s.uvs is None else _np(s.uvs)
        n = None if s.normals is None else _np(s.normals)
        keep.append((v, i, uv, n))
        shapes.append(dr.Shape(v, i, uv, n, materials[s.mat_id], None))
    lights = []
    for l in wl.lights:
        inten = _np(l.intensity)
        keep.append(inten)
        light = dr.Light(shapes[l.shape_id], inten)
        shapes[l.shape_id].light = light
        lights.append(light)
    W, H = wl.resolution
    if d_image is None:
        d_img = np.array(0.0, dtype=np.float32)
    else:
        d_img = np.ascontiguousarray(np.asarray(d_image, dtype=np.float32).reshape(H, W, 3))
    res = dr.render(camera, shapes, materials, lights, (W, H), d_img, int(wl.spp),
                    int(wl.max_bounces), int(seed), bool(print_progress))
    out = {"image": np.array(res.image)}
    if d_image is not None:
        out["d_cam_to_world"] = np.array(res.d_camera.d_cam_to_world)
        out["d_world_to_cam"] = np.array(res.d_camera.d_world_to_cam)
        out["d_sample_to_cam"] = np.array(res.d_camera.d_sample_to_cam)
        out["d_cam_to_sample"] = np.array(res.d_camera.d_cam_to_sample)
        out["d_vertices"] = [np.array(d.vertices) for d in res.d_shapes]
        out["d_normals"] = [np.array(d.normals) for d in res.d_shapes]
        out["d_diffuse"] = [np.array(d.diffuse_reflectance) for d in res.d_materials]
        out["d_specular"] = [np.array(d.specular_reflectance) for d in res.d_materials]
        out["d_roughness"] = [np.array(d.roughness) for d in res.d_materials]
        out["d_intensity"] = [np.array(d.intensity) for d in res.d_lights]
        out["dx_image"] = np.array(res.dx_image)
    return out
