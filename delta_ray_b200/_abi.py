"""ctypes mirror of include/delta_ray_b200.h and scene-descriptor marshalling.

``SceneDesc.from_scene(cam, materials, shapes, lights, device)`` turns the
package's scene objects (the reference's RenderFunction inputs,
render_pytorch.py:13-55) into a ``dr_scene_desc`` whose pointers reference
contiguous float32/int32 copies held by the returned object.  ``device`` is a
torch.device: ``cpu`` keeps host copies (the library uploads them), a CUDA
device keeps device copies, None leaves each array on its own tensor's device
(converted to the descriptor's dtype where needed).
"""
import ctypes as C

import numpy as np
import torch

c_float_p = C.POINTER(C.c_float)
c_int_p = C.POINTER(C.c_int)
c_size_p = C.POINTER(C.c_size_t)


class dr_camera_desc(C.Structure):
    _fields_ = [("cam_to_world", c_float_p), ("world_to_cam", c_float_p),
                ("sample_to_cam", c_float_p), ("cam_to_sample", c_float_p),
                ("fov_factor", C.c_float), ("aspect_ratio", C.c_float),
                ("clip_near", C.c_float), ("fisheye", C.c_int)]


class dr_material_desc(C.Structure):
    _fields_ = [("diffuse", c_float_p), ("diffuse_w", C.c_int), ("diffuse_h", C.c_int),
                ("specular", c_float_p), ("specular_w", C.c_int), ("specular_h", C.c_int),
                ("roughness", c_float_p), ("roughness_w", C.c_int), ("roughness_h", C.c_int),
                ("diffuse_uv_scale", c_float_p), ("specular_uv_scale", c_float_p),
                ("roughness_uv_scale", c_float_p), ("two_sided", C.c_int), ("microfacet", C.c_int)]


class dr_shape_desc(C.Structure):
    _fields_ = [("vertices", c_float_p), ("num_vertices", C.c_int),
                ("indices", c_int_p), ("num_triangles", C.c_int),
                ("uvs", c_float_p), ("normals", c_float_p), ("material_id", C.c_int)]


class dr_light_desc(C.Structure):
    _fields_ = [("shape_id", C.c_int), ("intensity", c_float_p)]


class dr_scene_desc(C.Structure):
    _fields_ = [("camera", dr_camera_desc),
                ("materials", C.POINTER(dr_material_desc)), ("num_materials", C.c_int),
                ("shapes", C.POINTER(dr_shape_desc)), ("num_shapes", C.c_int),
                ("lights", C.POINTER(dr_light_desc)), ("num_lights", C.c_int),
                ("ltc_table", c_float_p), ("ltc_table_ggx", c_float_p)]


class dr_render_desc(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("spp", C.c_int),
                ("max_bounces", C.c_int), ("seed", C.c_uint64),
                ("primary_edge_samples", C.c_int64), ("dp_mode", C.c_int),
                ("flags", C.c_int), ("reserved", C.c_int * 7)]


class dr_grad_layout(C.Structure):
    _fields_ = [("total", C.c_size_t), ("camera", C.c_size_t),
                ("material", c_size_p), ("shape_vertices", c_size_p),
                ("shape_normals", c_size_p), ("light", c_size_p)]


DR_DP_REFERENCE_LAST = 0
DR_DP_SUM = 1
DR_FLAG_FULL_PIXEL_JITTER = 1
DR_FLAG_DETACHED_PDF = 2
DR_FLAG_EDGE_LOBE_MIS = 4
DR_FLAG_LEARNED_PROPOSAL = 8


def camera_desc(cam, keep):
    """dr_camera_desc of a camera dict (scene_dicts' layout); the float32
    host copies of the matrices are appended to `keep`."""
    cd = dr_camera_desc()
    for name in ("cam_to_world", "world_to_cam", "sample_to_cam", "cam_to_sample"):
        t = torch.as_tensor(cam[name], dtype=torch.float32).detach().cpu().contiguous()
        keep.append(t)
        setattr(cd, name, C.cast(t.data_ptr(), c_float_p))
    cd.fov_factor = float(cam["fov_factor"])
    cd.aspect_ratio = float(cam["aspect_ratio"])
    cd.clip_near = float(cam["clip_near"])
    cd.fisheye = int(bool(cam["fisheye"]))
    return cd


class dr_view_desc(C.Structure):
    _fields_ = [("camera", dr_camera_desc), ("render", dr_render_desc), ("d_image", C.c_void_p),
                ("image", C.c_void_p)]


class dr_tuning(C.Structure):
    _fields_ = [("hand_steps", C.c_int32), ("task_rounds", C.c_int32), ("queue_items", C.c_int64),
                ("depth_first", C.c_int32), ("reserved", C.c_int32)]


class dr_tune_report(C.Structure):
    _fields_ = [("best", dr_tuning), ("best_ms", C.c_float), ("start_ms", C.c_float), ("trials", C.c_int32)]


class dr_proposal_desc(C.Structure):
    _fields_ = [("train", C.c_int), ("mix", C.c_float), ("learning_rate", C.c_float), ("train_points", C.c_int64),
                ("params", C.c_void_p)]


def render_desc(width, height, spp, max_bounces, seed, primary_edge_samples=0,
                dp_mode=DR_DP_REFERENCE_LAST, flags=0):
    rd = dr_render_desc()
    rd.width, rd.height, rd.spp, rd.max_bounces = int(width), int(height), int(spp), int(max_bounces)
    rd.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    rd.primary_edge_samples = int(primary_edge_samples)
    rd.dp_mode = int(dp_mode)
    rd.flags = int(flags)
    return rd


def _tex_dims(t, channels):
    """(w, h) of a texture tensor, (0, 0) for a constant ([channels])."""
    if t.dim() == 1:
        if t.shape[0] != channels:
            raise ValueError(f"constant material channel must have {channels} entries")
        return 0, 0
    if t.dim() != 3 or t.shape[2] != channels:
        raise ValueError(f"texture must be [h, w, {channels}]")
    return int(t.shape[1]), int(t.shape[0])


class SceneDesc:
    """Owns contiguous copies of the scene arrays and the ctypes descriptor."""

    def __init__(self):
        self.keep = []
        self.desc = dr_scene_desc()
        self.grad_sizes = []  # (kind, index, numel) in flat-layout order

    def _ptr(self, t, dtype, device):
        """Pointer to t as a contiguous `dtype` array on `device` (None: on the
        tensor's own device; the library reads host and device memory)."""
        if t is None:
            return None
        if not torch.is_tensor(t):
            t = torch.as_tensor(np.asarray(t))
        t = t.detach().to(device=t.device if device is None else device, dtype=dtype).contiguous()
        self.keep.append(t)
        ctype = C.c_float if dtype == torch.float32 else C.c_int
        return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ctype))

    @classmethod
    def from_scene(cls, cam, materials, shapes, lights, device=torch.device("cpu"),
                   ltc_table=None, ltc_table_ggx=None):
        self = cls()
        f32 = torch.float32
        d = self.desc
        cd = d.camera
        cd.cam_to_world = self._ptr(cam["cam_to_world"], f32, device)
        cd.world_to_cam = self._ptr(cam["world_to_cam"], f32, device)
        cd.sample_to_cam = self._ptr(cam["sample_to_cam"], f32, device)
        cd.cam_to_sample = self._ptr(cam["cam_to_sample"], f32, device)
        cd.fov_factor = float(cam["fov_factor"])
        cd.aspect_ratio = float(cam["aspect_ratio"])
        cd.clip_near = float(cam["clip_near"])
        cd.fisheye = int(bool(cam["fisheye"]))
        mats = (dr_material_desc * max(1, len(materials)))()
        for i, m in enumerate(materials):
            md = mats[i]
            diffuse = torch.as_tensor(m["diffuse"])
            specular = torch.as_tensor(m["specular"])
            roughness = torch.as_tensor(m["roughness"])
            md.diffuse_w, md.diffuse_h = _tex_dims(diffuse, 3)
            md.specular_w, md.specular_h = _tex_dims(specular, 3)
            md.roughness_w, md.roughness_h = _tex_dims(roughness, 1)
            md.diffuse = self._ptr(diffuse, f32, device)
            md.specular = self._ptr(specular, f32, device)
            md.roughness = self._ptr(roughness, f32, device)
            md.diffuse_uv_scale = self._ptr(m["diffuse_uv_scale"], f32, device)
            md.specular_uv_scale = self._ptr(m["specular_uv_scale"], f32, device)
            md.roughness_uv_scale = self._ptr(m["roughness_uv_scale"], f32, device)
            md.two_sided = int(bool(m["two_sided"]))
            md.microfacet = int(m.get("microfacet", 0))
        shps = (dr_shape_desc * max(1, len(shapes)))()
        for i, s in enumerate(shapes):
            sd = shps[i]
            v = torch.as_tensor(s["vertices"])
            idx = torch.as_tensor(s["indices"])
            if v.dim() != 2 or v.shape[1] != 3 or idx.dim() != 2 or idx.shape[1] != 3:
                raise ValueError("vertices must be [V, 3] and indices [F, 3]")
            sd.vertices = self._ptr(v, f32, device)
            sd.num_vertices = int(v.shape[0])
            sd.indices = self._ptr(idx, torch.int32, device)
            sd.num_triangles = int(idx.shape[0])
            sd.uvs = self._ptr(s.get("uvs"), f32, device)
            sd.normals = self._ptr(s.get("normals"), f32, device)
            sd.material_id = int(s["material_id"])
        lts = (dr_light_desc * max(1, len(lights)))()
        for i, l in enumerate(lights):
            lts[i].shape_id = int(l["shape_id"])
            lts[i].intensity = self._ptr(l["intensity"], f32, device)
        self.keep += [mats, shps, lts]
        d.materials, d.num_materials = mats, len(materials)
        d.shapes, d.num_shapes = shps, len(shapes)
        d.lights, d.num_lights = lts, len(lights)
        d.ltc_table = self._ptr(ltc_table, f32, device) if ltc_table is not None else None
        d.ltc_table_ggx = self._ptr(ltc_table_ggx, f32, device) if ltc_table_ggx is not None else None
        # flat gradient layout (include/delta_ray_b200.h)
        sizes = [("camera", 0, 64)]
        for i, m in enumerate(materials):
            md = mats[i]
            sizes.append(("diffuse", i, 3 if md.diffuse_w == 0 else md.diffuse_w * md.diffuse_h * 3))
            sizes.append(("specular", i, 3 if md.specular_w == 0 else md.specular_w * md.specular_h * 3))
            sizes.append(("roughness", i, 1 if md.roughness_w == 0 else md.roughness_w * md.roughness_h))
        for i, s in enumerate(shapes):
            sizes.append(("vertices", i, 3 * shps[i].num_vertices))
            if s.get("normals") is not None:
                sizes.append(("normals", i, 3 * shps[i].num_vertices))
        for i, _ in enumerate(lights):
            sizes.append(("intensity", i, 3))
        self.grad_sizes = sizes
        return self

    @property
    def grad_total(self):
        return sum(n for _, _, n in self.grad_sizes)

    def split_grad(self, flat, materials, shapes):
        """Slices a flat gradient into a dict of per-parameter views shaped like the inputs."""
        out = {"d_vertices": [None] * len(shapes), "d_normals": [None] * len(shapes),
               "d_diffuse": [], "d_specular": [], "d_roughness": [], "d_intensity": []}
        o = 0
        for kind, i, n in self.grad_sizes:
            seg = flat[o:o + n]
            o += n
            if kind == "camera":
                out["d_cam_to_world"] = seg[0:16].reshape(4, 4)
                out["d_world_to_cam"] = seg[16:32].reshape(4, 4)
                out["d_sample_to_cam"] = seg[32:48].reshape(4, 4)
                out["d_cam_to_sample"] = seg[48:64].reshape(4, 4)
            elif kind in ("diffuse", "specular", "roughness"):
                shape = tuple(torch.as_tensor(materials[i][kind]).shape)
                out["d_" + kind].append(seg.reshape(shape))
            elif kind == "vertices":
                out["d_vertices"][i] = seg.reshape(-1, 3)
            elif kind == "normals":
                out["d_normals"][i] = seg.reshape(-1, 3)
            elif kind == "intensity":
                out["d_intensity"].append(seg)
        return out


def scene_dicts(cam, materials, shapes, lights):
    """Package scene objects -> the plain dicts SceneDesc.from_scene consumes."""
    camd = dict(cam_to_world=cam.cam_to_world, world_to_cam=cam.world_to_cam,
                sample_to_cam=cam.sample_to_cam, cam_to_sample=cam.cam_to_sample,
                fov_factor=float(torch.as_tensor(cam.fov_factor).reshape(-1)[0]),
                aspect_ratio=float(cam.aspect_ratio),
                clip_near=float(torch.as_tensor(cam.clip_near).reshape(-1)[0]),
                fisheye=bool(cam.fisheye))
    mats = [dict(diffuse=m.diffuse_reflectance, specular=m.specular_reflectance,
                 roughness=m.roughness, diffuse_uv_scale=m.diffuse_uv_scale,
                 specular_uv_scale=m.specular_uv_scale, roughness_uv_scale=m.roughness_uv_scale,
                 two_sided=m.two_sided, microfacet=getattr(m, "microfacet", 0)) for m in materials]
    shps = [dict(vertices=s.vertices, indices=s.indices, uvs=s.uvs, normals=s.normals,
                 material_id=s.mat_id) for s in shapes]
    lts = [dict(shape_id=l.shape_id, intensity=l.intensity) for l in lights]
    return camd, mats, shps, lts
