"""Material description (mirrors the reference material.py:5-19).

A material is Lambertian diffuse plus a specular lobe: Blinn-Phong, as in the
reference, or GGX (``microfacet="ggx"``; alpha = roughness^2, no counterpart in
the reference).  Each of
``diffuse_reflectance`` ([3] or [h, w, 3]), ``specular_reflectance`` ([3] or
[h, w, 3]) and ``roughness`` ([1] or [h, w, 1]) is either a constant or a
texture looked up bilinearly with wrap-around.

Compatibility note: the reference constructor stores ``diffuse_uv_scale`` in
all three uv-scale slots (material.py:17-19 of the reference), ignoring the
specular and roughness scales it is given.  ``Material`` keeps that behaviour so
that scenes render identically; pass ``exact_uv_scales=True`` to keep the three
scales that were given.
"""
import torch


def _f32(values):
    return torch.tensor(values, dtype=torch.float32)


class Material:
    def __init__(self, diffuse_reflectance, specular_reflectance=None,
                 roughness=None, diffuse_uv_scale=None, specular_uv_scale=None,
                 roughness_uv_scale=None, two_sided=False, exact_uv_scales=False,
                 microfacet="blinn_phong"):
        if specular_reflectance is None:
            specular_reflectance = _f32([0.0, 0.0, 0.0])
        if roughness is None:
            roughness = _f32([1.0])
        if diffuse_uv_scale is None:
            diffuse_uv_scale = _f32([1.0, 1.0])
        if specular_uv_scale is None:
            specular_uv_scale = _f32([1.0, 1.0])
        if roughness_uv_scale is None:
            roughness_uv_scale = _f32([1.0, 1.0])
        self.diffuse_reflectance = diffuse_reflectance
        self.specular_reflectance = specular_reflectance
        self.roughness = roughness
        self.diffuse_uv_scale = diffuse_uv_scale
        if exact_uv_scales:
            self.specular_uv_scale = specular_uv_scale
            self.roughness_uv_scale = roughness_uv_scale
        else:
            self.specular_uv_scale = diffuse_uv_scale
            self.roughness_uv_scale = diffuse_uv_scale
        self.two_sided = two_sided
        models = {"blinn_phong": 0, "ggx": 1}
        if microfacet not in models:
            raise ValueError(f"microfacet must be one of {sorted(models)}")
        self.microfacet = models[microfacet]
