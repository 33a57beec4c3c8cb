"""LTC tables for edge sampling: the fitting tool and the fitted defaults.

The renderer importance-samples a point on a silhouette edge with a linearly
transformed cosine fitted to the shading point's specular lobe (material.h:
464-489 in the reference, which ships one Blinn-Phong table, ltc.inc).  This
module fits such tables for the renderer's own lobes with the project's
fitter (ltc_fit.cpp: Heitz et al. 2016 with Nelder-Mead):

    python -m delta_ray_b200.ltc        # refits data/ltc_blinn_phong.f32 and data/ltc_ggx.f32

``default_table(model)`` returns the committed fit: model 0 is the
renderer's Blinn-Phong lobe (exponent 2 / roughness, the reference's rational
Smith term), model 1 is GGX (alpha = roughness^2).  Each table is
128 x 128 entries (roughness x view angle) of a row-major 3x3 matrix, the
layout of ``dr_scene_desc.ltc_table`` / ``ltc_table_ggx``.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ltc_fit.cpp")
LIB = os.path.join(HERE, "libltc_fit.so")
DATA = os.path.join(HERE, "data")
N = 128
FILES = {0: "ltc_blinn_phong.f32", 1: "ltc_ggx.f32"}
BLINN_PHONG, GGX = 0, 1


def build():
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    subprocess.run(["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-pthread", "-fvisibility=hidden", "-o", LIB,
                    SRC], check=True)
    return LIB


def _lib():
    L = C.CDLL(build())
    L.ltc_fit_table.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    L.ltc_fit_table.restype = C.c_int
    L.ltc_fit_l1.argtypes = [C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int]
    L.ltc_fit_l1.restype = C.c_double
    return L


def fit_table(model, n=N, strata=24, iters=300, threads=None):
    """([n * n * 9] float32 table, [n * n] final fit errors)."""
    L = _lib()
    m = np.zeros(n * n * 9, np.float32)
    err = np.zeros(n * n, np.float32)
    if L.ltc_fit_table(int(model), int(n), int(strata), int(iters), m.ctypes.data, err.ctypes.data,
                       int(threads or os.cpu_count() or 1)) != 0:
        raise ValueError("ltc_fit_table failed")
    return m, err


def fit_l1(model, roughness, theta, m9, strata=64):
    """Integral of |LTC density - normalised lobe| for one table entry (0 = exact, 2 = disjoint)."""
    m9 = np.ascontiguousarray(np.asarray(m9, np.float32).reshape(9))
    return float(_lib().ltc_fit_l1(int(model), float(roughness), float(theta), m9.ctypes.data, int(strata)))


def default_table(model):
    """The committed fitted table of `model` as [128 * 128 * 9] float32."""
    path = os.path.join(DATA, FILES[model])
    t = np.fromfile(path, np.float32)
    if t.size != N * N * 9:
        raise ValueError(f"{path}: expected {N * N * 9} floats, found {t.size}")
    return t


def main():
    os.makedirs(DATA, exist_ok=True)
    for model, name in FILES.items():
        m, err = fit_table(model)
        m.tofile(os.path.join(DATA, name))
        print(f"{name}: max fit error {err.max():.3g}, mean {err.mean():.3g}")


if __name__ == "__main__":
    sys.exit(main())
