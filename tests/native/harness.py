"""Test infrastructure: ctypes front end of tests/native/host_harness.cpp.

The harness runs the renderer's per-sample kernel logic on the CPU; the
library is built by ``build()`` into tests/_build/libhost_harness.so.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "tests", "_build", "libhost_harness.so")
_lib = None


def build():
    src = os.path.join(HERE, "host_harness.cpp")
    csrc = os.path.join(ROOT, "delta_ray_b200", "csrc")
    deps = [src] + [os.path.join(csrc, f) for f in os.listdir(csrc)]
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-DDR_HOST_BUILD", "-o", LIB,
                    src],
                   check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        from delta_ray_b200 import _abi
        build()
        L = C.CDLL(LIB)
        L.hh_render.argtypes = [C.POINTER(_abi.dr_scene_desc), C.POINTER(_abi.dr_render_desc), C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.hh_trace.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.hh_trace.restype = C.c_longlong
        L.hh_set_proposal.argtypes = [C.c_int, C.c_float]
        L.hh_set_split.argtypes = [C.c_int]
        L.hh_set_checkpoints.argtypes = [C.c_int]
        L.hh_math.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]
        L.hh_scene_edges.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_int, C.c_void_p, C.c_longlong]
        L.hh_scene_edges.restype = C.c_longlong
        L.hh_silhouette.argtypes = [C.c_void_p] * 5 + [C.c_longlong, C.c_void_p]
        L.hh_trace_pairs.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_void_p, C.c_int, C.c_void_p]
        L.hh_trace_before.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_void_p]
        _lib = L
    return _lib


def render(wl, seed, d_image=None, parts=7, ltc_table=None, dp_mode=0, primary_edge_samples=0, flags=0,
           ltc_table_ggx=None):
    from delta_ray_b200 import _abi
    L = load()
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"), ltc_table, ltc_table_ggx)
    W, H = wl.resolution
    rd = _abi.render_desc(W, H, wl.spp, wl.max_bounces, seed, primary_edge_samples, dp_mode, flags)
    image = np.zeros((H, W, 3), np.float32)
    grad = np.zeros(sd.grad_total, np.float32)
    stats = np.zeros(2, np.int64)
    dimg = None if d_image is None else np.ascontiguousarray(np.asarray(d_image, np.float32))
    L.hh_render(C.byref(sd.desc), C.byref(rd), None if dimg is None else dimg.ctypes.data, image.ctypes.data,
                grad.ctypes.data, int(parts), stats.ctypes.data)
    return {"image": image, "grad": grad, "stats": stats, "sd": sd}


def trace(wl, rays):
    from delta_ray_b200 import _abi
    L = load()
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"))
    rays = np.ascontiguousarray(np.asarray(rays, np.float32).reshape(-1, 6))
    tri = np.zeros(len(rays), np.int32)
    t = np.zeros(len(rays), np.float32)
    visits = L.hh_trace(C.byref(sd.desc), rays.ctypes.data, len(rays), tri.ctypes.data, t.ctypes.data)
    return tri, t, visits


def set_proposal(seed, alpha):
    """Synthetic learned proposal of later renders (seed 0: none)."""
    load().hh_set_proposal(int(seed), float(alpha))


def set_checkpoints(k):
    """Later renders trace paths in the checkpointed form (segments of k = 4,
    8 or 16 bounces, up to 16 segments; 0: per-bounce records, up to 64)."""
    load().hh_set_checkpoints(int(k))


def set_split(on):
    """Walk large traversals in two stages (subtrees handed on at depth 4)."""
    load().hh_set_split(int(bool(on)))


MATH_FUNCS = {"sin": 0, "cos": 1, "atan": 2, "atan2": 3, "acos": 4, "exp": 5, "log": 6, "pow": 7}


def math_eval(name, x, y=None):
    """The reproducible transcendental functions (csrc/dr_math.h) on the CPU."""
    L = load()
    x = np.ascontiguousarray(x, np.float32)
    yy = None if y is None else np.ascontiguousarray(np.broadcast_to(np.asarray(y, np.float32), x.shape))
    out = np.empty_like(x)
    L.hh_math(MATH_FUNCS[name], x.ctypes.data, None if yy is None else yy.ctypes.data, out.ctypes.data, x.size)
    return out


EDGE_DATA = {"sil_nodes": (0, 56), "sil_edges": (1, 20), "nrm_nodes": (2, 56), "nrm_edges": (3, 20),
             "prim_edges": (4, 20), "prim_cdf": (5, 4), "prim_func": (6, 4), "prim_func_int": (7, 4)}


def scene_edges(wl, what):
    """One array of the scene's edge data as the host build makes it, as bytes."""
    from delta_ray_b200 import _abi
    L = load()
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"))
    code, elem = EDGE_DATA[what]
    n = L.hh_scene_edges(C.byref(sd.desc), code, None, 0)
    buf = np.zeros(max(1, n * elem), np.uint8)
    L.hh_scene_edges(C.byref(sd.desc), code, buf.ctypes.data, buf.size)
    return buf[:n * elem].tobytes()


def trace_pairs(wl, rays):
    """[n, 9] ray pairs -> [n, 4] hit ids: the paired walk's two, then two single walks'."""
    from delta_ray_b200 import _abi
    L = load()
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"))
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.zeros((rays.shape[0], 4), np.int32)
    L.hh_trace_pairs(C.byref(sd.desc), rays.ctypes.data, rays.shape[0], out.ctypes.data)
    return out


def trace_before(wl, rays, ta, ida):
    """Whether a triangle hits ahead of (ta, ida) for rays [n, 6], through the
    binary LBVH walk and through the 4-wide walk: [n, 2] int."""
    from delta_ray_b200 import _abi
    L = load()
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    sd = _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"))
    rays = np.ascontiguousarray(rays, np.float32)
    ta = np.ascontiguousarray(ta, np.float32)
    ida = np.ascontiguousarray(ida, np.int32)
    out = np.zeros((rays.shape[0], 2), np.int32)
    L.hh_trace_before(C.byref(sd.desc), rays.ctypes.data, ta.ctypes.data, ida.ctypes.data, rays.shape[0],
                      out.ctypes.data)
    return out


def silhouette(lo, hi, axis, angle, p):
    """contains_silhouette per (node, point): (filtered, float evaluation alone)."""
    L = load()
    arrs = [np.ascontiguousarray(np.asarray(a, np.float32)) for a in (lo, hi, axis, angle, p)]
    n = arrs[3].shape[0]
    out = np.zeros((n, 2), np.int32)
    L.hh_silhouette(*[a.ctypes.data for a in arrs], n, out.ctypes.data)
    return out[:, 0].astype(bool), out[:, 1].astype(bool)
