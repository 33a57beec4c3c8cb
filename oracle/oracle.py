"""Test infrastructure: Python front end of the C++ restatement (dr_oracle.cpp).

``oracle_render(workload, seed, d_image=None, rng_mode=...)`` renders a package
``Workload`` with the restated reference algorithm and returns the same dict
keys as ``ref_runner.render_reference`` plus the flat gradient.

rng_mode REFERENCE (0) draws random numbers exactly as the compiled reference
does (std::mt19937 per 8x8 tile and per edge thread); PHILOX (1) draws them
from the counter-based streams that the GPU product uses, so the product can be
compared sample for sample.

Only tests, smoke() and bench.py's CPU-baseline leg import this module.
"""
import ctypes as C
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from delta_ray_b200 import _abi  # noqa: E402

REFERENCE = 0
PHILOX = 1
PHILOX_LIBM = 2  # Philox streams, host libm transcendentals (the product's are reproducible ones)
LIB_PATH = os.path.join(HERE, "_build", "libdr_oracle.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("oracle not built: run `make -C oracle port`")
        lib = C.CDLL(LIB_PATH)
        lib.dro_render.argtypes = [C.POINTER(_abi.dr_scene_desc), C.POINTER(_abi.dr_render_desc),
                                   C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_void_p]
        lib.dro_render.restype = C.c_int
        lib.dro_render_parts.argtypes = list(lib.dro_render.argtypes) + [C.c_int]
        lib.dro_render_parts.restype = C.c_int
        lib.dro_trace.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_void_p, C.c_longlong,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
        lib.dro_philox.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int,
                                   C.c_void_p]
        lib.dro_scene_info.argtypes = [C.POINTER(_abi.dr_scene_desc), C.c_void_p]
        lib.dro_philox_raw.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def scene_desc(wl, ltc_table=None, ltc_table_ggx=None):
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    return _abi.SceneDesc.from_scene(cam, mats, shps, lts, torch.device("cpu"), ltc_table, ltc_table_ggx)


def oracle_render(wl, seed, d_image=None, rng_mode=REFERENCE, cores=8, ltc_table=None,
                  dp_mode=_abi.DR_DP_REFERENCE_LAST, primary_edge_samples=0, threads=0,
                  shape_rank=None, parts=7, flags=0, ltc_table_ggx=None):
    """shape_rank: sort key per shape for the edge order (see dr_oracle.cpp Scene).
    parts: backward terms to include (1 continuous, 2 secondary edges, 4 primary edges)."""
    lib = load()
    sd = scene_desc(wl, ltc_table, ltc_table_ggx)
    W, H = wl.resolution
    rd = _abi.render_desc(W, H, wl.spp, wl.max_bounces, seed, primary_edge_samples, dp_mode, flags)
    image = np.zeros((H, W, 3), np.float32)
    grad = np.zeros(sd.grad_total, np.float32)
    stats = np.zeros(2, np.int64)
    dimg = None
    if d_image is not None:
        dimg = np.ascontiguousarray(np.asarray(d_image, np.float32).reshape(H, W, 3))
    rank = None
    if shape_rank is not None:
        rank = np.ascontiguousarray(np.asarray(shape_rank, np.int32))
    lib.dro_render_parts(C.byref(sd.desc), C.byref(rd), int(rng_mode), int(cores),
                         None if dimg is None else dimg.ctypes.data, image.ctypes.data,
                         grad.ctypes.data, stats.ctypes.data, int(threads),
                         None if rank is None else rank.ctypes.data, int(parts))
    out = {"image": image, "grad": grad, "stats": stats}
    if d_image is not None:
        cam, mats, shps, _ = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
        parts = sd.split_grad(torch.from_numpy(grad), mats, shps)
        for k, v in parts.items():
            if isinstance(v, list):
                out[k] = [None if x is None else x.numpy() for x in v]
            else:
                out[k] = v.numpy()
    return out


def trace(wl, rays):
    """Closest-hit (shape, triangle, t) per ray under the shared hit rule."""
    lib = load()
    sd = scene_desc(wl)
    rays = np.ascontiguousarray(np.asarray(rays, np.float32).reshape(-1, 6))
    n = rays.shape[0]
    sh = np.zeros(n, np.int32)
    tr = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    lib.dro_trace(C.byref(sd.desc), rays.ctypes.data, n, sh.ctypes.data, tr.ctypes.data,
                  t.ctypes.data)
    return sh, tr, t


def philox(seed, kind, ident, sub, n):
    lib = load()
    out = np.zeros(n, np.float32)
    lib.dro_philox(int(seed), int(kind), int(ident), int(sub), int(n), out.ctypes.data)
    return out


def philox_raw(ctr, key):
    lib = load()
    c = np.ascontiguousarray(np.asarray(ctr, np.uint32))
    k = np.ascontiguousarray(np.asarray(key, np.uint32))
    out = np.zeros(4, np.uint32)
    lib.dro_philox_raw(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def scene_info(wl):
    lib = load()
    sd = scene_desc(wl)
    out = np.zeros(6, np.int32)
    lib.dro_scene_info(C.byref(sd.desc), out.ctypes.data)
    keys = ["primary_edges", "silhouette_edges", "silhouette_nodes", "normal_edges",
            "normal_nodes", "triangles"]
    return dict(zip(keys, out.tolist()))


def _rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(1e-30, np.abs(b).max()))


def match_reference_order(wl, ref_out, seed, d_image=None, cores=8, ltc_table=None):
    """Finds the shape order the reference used for one call.

    The compiled reference orders edges by Shape* address, which varies from
    call to call.  Returns (rank, oracle_out, err) for the permutation whose
    oracle render is closest to ``ref_out`` (image and flat gradient).
    """
    import itertools
    n = len(wl.shapes)
    perms = list(itertools.permutations(range(n))) if n <= 5 else [tuple(range(n)),
                                                                    tuple(range(n))[::-1]]
    best = None
    ref_flat = None
    for perm in perms:
        rank = np.empty(n, np.int32)
        rank[list(perm)] = np.arange(n)
        out = oracle_render(wl, seed, d_image, REFERENCE, cores, ltc_table, shape_rank=rank)
        err = _rel_err(out["image"], ref_out["image"])
        if d_image is not None:
            if ref_flat is None:
                ref_flat = flat_from_parts(wl, ref_out)
            err = max(err, _rel_err(out["grad"], ref_flat))
        if best is None or err < best[2]:
            best = (rank, out, err)
        if err < 1e-5:
            break
    return best


def flat_from_parts(wl, out):
    """Flat gradient (product layout) assembled from per-parameter arrays."""
    parts = [out["d_cam_to_world"].ravel(), out["d_world_to_cam"].ravel(),
             out["d_sample_to_cam"].ravel(), out["d_cam_to_sample"].ravel()]
    for i in range(len(wl.materials)):
        parts += [np.asarray(out["d_diffuse"][i]).ravel(), np.asarray(out["d_specular"][i]).ravel(),
                  np.asarray(out["d_roughness"][i]).ravel()]
    for i, s in enumerate(wl.shapes):
        parts.append(np.asarray(out["d_vertices"][i]).ravel())
        if s.normals is not None:
            parts.append(np.asarray(out["d_normals"][i]).ravel())
    for i in range(len(wl.lights)):
        parts.append(np.asarray(out["d_intensity"][i]).ravel())
    return np.concatenate(parts).astype(np.float32)
