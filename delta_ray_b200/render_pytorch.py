"""Drop-in replacement of the reference's render_pytorch.RenderFunction.

``RenderFunction.serialize_scene(cam, materials, shapes, lights, resolution,
num_samples, max_bounces)`` returns the same flat argument list as the
reference (render_pytorch.py:13-55), and ``RenderFunction.apply(seed, *args)``
renders it (render_pytorch.py:58-233); ``loss.backward()`` returns one
gradient per argument (render_pytorch.py:236-333).  Differences:

* rendering runs on the GPU through libdr_b200.so; inputs may be CPU or CUDA
  tensors, the image is a CUDA tensor (``RenderOptions.output_device``
  changes that) and gradients come back on each input's own device;
* the scene is built once in forward and reused by backward (the reference
  rebuilds it in both passes);
* a ``RenderOptions`` object may be appended after ``max_bounces``;
* uv-scale gradients are None: the reference computes them but never
  accumulates them (delta_ray.cpp:853-859, :1127-1128).
"""
import ctypes as C

import torch

from . import _abi, _lib


def set_item_queue_limit(items=0):
    """Upper bound on the edge items a backward call holds on the device at
    once (dr_set_item_queue_limit; 0: the default, 8 GiB worth).  Calls whose
    points sample more edges run their edge stage in chunks of points."""
    _lib.check(_lib.lib().dr_set_item_queue_limit(int(items)))


class RenderOptions:
    """Optional trailing argument of RenderFunction.apply.

    primary_edge_samples: number of primary-edge samples in backward
        (0 = spp * width * height, the reference's total).
    dp_mode: _abi.DR_DP_REFERENCE_LAST (the reference's behaviour) or
        _abi.DR_DP_SUM (sum every sampled edge's position derivative).
    ltc_table, ltc_table_ggx: [128*128*9] float32 LTC tables for edge sampling
        of Blinn-Phong and GGX lobes; "fitted" (default) selects the tables
        fitted to this renderer's lobes (delta_ray_b200.ltc), None identity
        matrices (the cosine lobe); pass the reference's table (ltc.inc) to
        sample edges as the reference does.
    output_device: device of the returned image (default: the render device).
    device: CUDA device index to render on (default: current device).
    full_pixel_jitter: spread each pixel's samples over the whole pixel (a box
        filter, the image whose derivative the edge terms estimate) instead of
        the reference's [0, 1/spp) sub-pixel offsets (delta_ray.cpp:1236-1237).
    detached_pdf: hold the BSDF sampling pdf constant in the backward pass
        (unbiased gradients of roughness and lobe weights) instead of
        differentiating it at a fixed sampled direction as the reference does.
    learned_proposal: draw secondary edges with the scene's learned proposal
        (Scene.set_proposal) and, in its training mode, train it on this call.
    edge_lobe_mis: divide a secondary-edge sample by the two lobes' mixture
        density at the sampled point (balance heuristic).  The reference
        divides by the picked lobe's pick probability times its line pdf,
        which doubles the edge term on materials with both a diffuse and a
        specular lobe (delta_ray.cpp:88-105, 318-330).
    """

    def __init__(self, primary_edge_samples=0, dp_mode=_abi.DR_DP_REFERENCE_LAST, ltc_table="fitted",
                 output_device=None, device=None, full_pixel_jitter=False, ltc_table_ggx="fitted",
                 detached_pdf=False, edge_lobe_mis=False, learned_proposal=False):
        self.primary_edge_samples = int(primary_edge_samples)
        self.dp_mode = int(dp_mode)
        self.flags = (_abi.DR_FLAG_FULL_PIXEL_JITTER if full_pixel_jitter else 0) | \
            (_abi.DR_FLAG_DETACHED_PDF if detached_pdf else 0) | \
            (_abi.DR_FLAG_EDGE_LOBE_MIS if edge_lobe_mis else 0) | \
            (_abi.DR_FLAG_LEARNED_PROPOSAL if learned_proposal else 0)
        self.ltc_table = ltc_table
        self.ltc_table_ggx = ltc_table_ggx
        self.output_device = output_device
        self.device = device


_FITTED = {}  # model -> the committed fitted LTC table (read once; the library copies it)


def _table(t, model):
    """An LTC table argument: "fitted" -> the committed fit of `model`, None -> None."""
    if isinstance(t, str):
        if t != "fitted":
            raise ValueError(f"unknown LTC table {t!r}")
        if model not in _FITTED:
            from . import ltc
            _FITTED[model] = torch.from_numpy(ltc.default_table(model))
        return _FITTED[model]
    return t


class Scene:
    """A device scene (dr_scene) built from unpacked RenderFunction arguments."""

    def __init__(self, cam, materials, shapes, lights, device_index, ltc_table="fitted", ltc_table_ggx="fitted"):
        L = _lib.lib()
        ltc_table, ltc_table_ggx = _table(ltc_table, 0), _table(ltc_table_ggx, 1)
        self._tables = (ltc_table, ltc_table_ggx)
        self.device_index = int(device_index)
        self.device = torch.device("cuda", self.device_index)
        self.materials = materials
        self.shapes = shapes
        # the description is read where it lies (host or device); the library
        # keeps its own copies, so no tensor is moved for it
        self.sd = _abi.SceneDesc.from_scene(cam, materials, shapes, lights, None, ltc_table, ltc_table_ggx)
        handle = C.c_void_p()
        with torch.cuda.device(self.device_index):
            torch.cuda.current_stream().synchronize()
            _lib.check(L.dr_scene_create(C.byref(self.sd.desc), self.device_index, C.byref(handle)))
        self.handle = handle
        lay = _abi.dr_grad_layout()
        _lib.check(L.dr_scene_grad_layout(self.handle, C.byref(lay)))
        self.grad_total = int(lay.total)
        if self.grad_total != self.sd.grad_total:
            raise RuntimeError("gradient layout mismatch between library and binding")

    def update(self, cam, materials, shapes, lights, ltc_table="keep", ltc_table_ggx="keep"):
        """New parameters for the same meshes (dr_scene_update): positions,
        normals, materials, lights and camera may change; the edge topology
        and the LBVH's tree are kept when the triangle indices are unchanged.
        The LTC tables stay those of the scene unless given."""
        t0 = self._tables[0] if isinstance(ltc_table, str) and ltc_table == "keep" else _table(ltc_table, 0)
        t1 = self._tables[1] if isinstance(ltc_table_ggx, str) and ltc_table_ggx == "keep" else _table(ltc_table_ggx, 1)
        self._tables = (t0, t1)
        sd = _abi.SceneDesc.from_scene(cam, materials, shapes, lights, None, t0, t1)
        with torch.cuda.device(self.device_index):
            torch.cuda.current_stream().synchronize()
            _lib.check(_lib.lib().dr_scene_update(self.handle, C.byref(sd.desc)))
        self.sd, self.materials, self.shapes = sd, materials, shapes

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, width, height, spp, max_bounces, seed, opts=None):
        opts = opts or RenderOptions()
        img = torch.empty((height, width, 3), dtype=torch.float32, device=self.device)
        rd = _abi.render_desc(width, height, spp, max_bounces, seed, opts.primary_edge_samples, opts.dp_mode,
                              opts.flags)
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.lib().dr_render_forward(self.handle, C.byref(rd), C.c_void_p(img.data_ptr()),
                                                    self._stream()))
        return img

    def backward(self, width, height, spp, max_bounces, seed, d_image, opts=None, want_image=False):
        opts = opts or RenderOptions()
        d_image = d_image.detach().to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(d_image.shape) != (height, width, 3):
            raise ValueError(f"d_image must be [{height}, {width}, 3]")
        grad = torch.empty(self.grad_total, dtype=torch.float32, device=self.device)
        img = torch.empty((height, width, 3), dtype=torch.float32, device=self.device) if want_image else None
        rd = _abi.render_desc(width, height, spp, max_bounces, seed, opts.primary_edge_samples, opts.dp_mode,
                              opts.flags)
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.lib().dr_render_backward(
                self.handle, C.byref(rd), C.c_void_p(d_image.data_ptr()), C.c_void_p(grad.data_ptr()),
                C.c_void_p(img.data_ptr()) if img is not None else None, self._stream()))
        return grad, img

    def tuning(self):
        """The scene's queue settings (dr_scene_get_tuning): hand_steps,
        task_rounds, queue_items, depth_first."""
        t = _abi.dr_tuning()
        _lib.check(_lib.lib().dr_scene_get_tuning(self.handle, C.byref(t)))
        return {"hand_steps": t.hand_steps, "task_rounds": t.task_rounds, "queue_items": t.queue_items,
                "depth_first": t.depth_first}

    def set_tuning(self, hand_steps=64, task_rounds=3, queue_items=0, depth_first=0):
        """Sets the scene's queue settings (dr_scene_set_tuning); the
        defaults are the library's."""
        t = _abi.dr_tuning(int(hand_steps), int(task_rounds), int(queue_items), int(depth_first), 0)
        _lib.check(_lib.lib().dr_scene_set_tuning(self.handle, C.byref(t)))

    def autotune(self, width, height, spp, max_bounces, seed, d_image, opts=None, max_trials=16):
        """Times backward calls of this render under several queue settings
        and keeps the fastest on the scene (dr_scene_autotune).  Returns the
        chosen setting with best_ms, start_ms and trials."""
        opts = opts or RenderOptions()
        d_image = d_image.detach().to(device=self.device, dtype=torch.float32).contiguous()
        if tuple(d_image.shape) != (height, width, 3):
            raise ValueError(f"d_image must be [{height}, {width}, 3]")
        grad = torch.empty(self.grad_total, dtype=torch.float32, device=self.device)
        rd = _abi.render_desc(width, height, spp, max_bounces, seed, opts.primary_edge_samples, opts.dp_mode,
                              opts.flags)
        rep = _abi.dr_tune_report()
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.lib().dr_scene_autotune(self.handle, C.byref(rd), C.c_void_p(d_image.data_ptr()),
                                                    C.c_void_p(grad.data_ptr()), int(max_trials), C.byref(rep),
                                                    self._stream()))
        b = rep.best
        return {"hand_steps": b.hand_steps, "task_rounds": b.task_rounds, "queue_items": b.queue_items,
                "depth_first": b.depth_first, "best_ms": rep.best_ms, "start_ms": rep.start_ms,
                "trials": rep.trials}

    def backward_views(self, views, opts=None):
        """Backward render of several views in one call.  views: a list of
        dicts with keys camera (a Camera or a scene_dicts camera dict),
        width, height, spp, max_bounces, seed, d_image ([H, W, 3]).  Returns
        (flat gradient summed over the views, with a zero camera block;
        camera gradients [n_views, 64], one block per view)."""
        opts = opts or RenderOptions()
        keep, descs = [], (_abi.dr_view_desc * max(1, len(views)))()
        for k, v in enumerate(views):
            cam = v["camera"]
            if not isinstance(cam, dict):
                cam = _abi.scene_dicts(cam, [], [], [])[0]
            d = torch.as_tensor(v["d_image"]).detach().to(device=self.device, dtype=torch.float32).contiguous()
            if tuple(d.shape) != (v["height"], v["width"], 3):
                raise ValueError(f"view {k}: d_image must be [{v['height']}, {v['width']}, 3]")
            keep.append(d)
            descs[k].camera = _abi.camera_desc(cam, keep)
            descs[k].render = _abi.render_desc(v["width"], v["height"], v["spp"], v["max_bounces"], v["seed"],
                                               opts.primary_edge_samples, opts.dp_mode, opts.flags)
            descs[k].d_image = d.data_ptr()
            descs[k].image = None
        grad = torch.empty(self.grad_total, dtype=torch.float32, device=self.device)
        cam_grads = torch.empty((max(1, len(views)), 64), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.lib().dr_render_backward_views(self.handle, len(views), descs,
                                                           C.c_void_p(grad.data_ptr()),
                                                           C.c_void_p(cam_grads.data_ptr()), self._stream()))
        return grad, cam_grads[:len(views)]

    def trace(self, rays):
        """Closest hit (global triangle id, t) of rays [n, 6] on the device."""
        rays = rays.detach().to(device=self.device, dtype=torch.float32).contiguous().reshape(-1, 6)
        n = rays.shape[0]
        tri = torch.empty(n, dtype=torch.int32, device=self.device)
        t = torch.empty(n, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device_index):
            _lib.check(_lib.lib().dr_trace_rays(self.handle, C.c_void_p(rays.data_ptr()), n,
                                                C.c_void_p(tri.data_ptr()), C.c_void_p(t.data_ptr()),
                                                self._stream()))
        return tri, t

    def set_proposal(self, train=True, mix=0.5, learning_rate=1e-3, train_points=32768, params=None):
        """Attach (or reconfigure) the scene's learned edge proposal, used by
        backward calls with RenderOptions(learned_proposal=True).  params:
        a flat tensor of proposal.param_count() floats (None keeps the
        current ones; a fixed initialisation the first time)."""
        p = None if params is None else torch.as_tensor(params, dtype=torch.float32).contiguous()
        d = _abi.dr_proposal_desc(int(bool(train)), float(mix), float(learning_rate), int(train_points),
                                  None if p is None else p.data_ptr())
        _lib.check(_lib.lib().dr_scene_set_proposal(self.handle, C.byref(d)))

    def proposal_state(self):
        """(parameters [CPU tensor], last training loss, training steps taken)."""
        from . import proposal
        p = torch.empty(proposal.param_count(), dtype=torch.float32)
        loss, steps = C.c_float(), C.c_int64()
        _lib.check(_lib.lib().dr_scene_proposal_state(self.handle, C.c_void_p(p.data_ptr()), C.byref(loss),
                                                      C.byref(steps)))
        return p, float(loss.value), int(steps.value)

    def split_grad(self, flat):
        return self.sd.split_grad(flat, self.materials, self.shapes)

    def set_profiling(self, on=True):
        _lib.check(_lib.lib().dr_scene_set_profiling(self.handle, int(bool(on))))

    def last_timings(self):
        """[(stage name, ms)] of the last render call (profiling must be on)."""
        out = []
        name = C.create_string_buffer(64)
        ms = C.c_float()
        i = 0
        while _lib.lib().dr_scene_last_timings(self.handle, i, name, len(name), C.byref(ms)) == 0:
            out.append((name.value.decode(), ms.value))
            i += 1
        return out

    def last_work(self):
        """Work counts of the last backward call (dr_scene_last_work): points,
        items, line samples passed to the ray stage (for large meshes: those
        whose rays hit one of the edge's faces), shaded samples, subtree tasks,
        first-stage items,
        node visits of the point walks and of the subtree walks, candidates of
        the ray stage (samples that passed its connectivity test), subtrees
        walked depth first after a full level queue."""
        w = (C.c_int64 * 10)()
        _lib.check(_lib.lib().dr_scene_last_work(self.handle, w, 10))
        keys = ("points", "items", "survivors", "shaded", "tasks", "items_first_stage", "visits_walk",
                "visits_tasks", "candidates", "spilled")
        return dict(zip(keys, (int(x) for x in w)))

    def last_counts(self):
        p, it = C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().dr_scene_last_counts(self.handle, C.byref(p), C.byref(it)))
        return p.value, it.value

    def launch_count(self):
        n = C.c_int()
        _lib.check(_lib.lib().dr_scene_last_launch_count(self.handle, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().dr_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def unpack_args(args):
    """Splits the flat argument list (render_pytorch.py:61-135 of the reference)."""
    i = 0

    def take():
        nonlocal i
        v = args[i]
        i += 1
        return v
    nm, ns, nl = take(), take(), take()
    cam = dict(cam_to_world=take(), world_to_cam=take(), sample_to_cam=take(), cam_to_sample=take(),
               fov_factor=float(take()), aspect_ratio=float(take()), clip_near=float(take()),
               fisheye=bool(take()))
    mats = []
    for _ in range(nm):
        m = dict(diffuse=take(), specular=take(), roughness=take(), diffuse_uv_scale=take(),
                 specular_uv_scale=take(), roughness_uv_scale=take())
        ts = take()
        # a GGX material serializes its two_sided slot as (two_sided, microfacet)
        m["two_sided"], m["microfacet"] = (bool(ts[0]), int(ts[1])) if isinstance(ts, tuple) else (bool(ts), 0)
        mats.append(m)
    shps = []
    for _ in range(ns):
        shps.append(dict(vertices=take(), indices=take(), uvs=take(), normals=take(),
                         material_id=int(take())))
    lts = []
    for _ in range(nl):
        lts.append(dict(shape_id=int(take()), intensity=take()))
    resolution = take()
    spp = int(take())
    max_bounces = int(take())
    opts = None
    if i < len(args) and isinstance(args[i], RenderOptions):
        opts = take()
    if i != len(args):
        raise ValueError("unexpected trailing arguments to RenderFunction")
    return cam, mats, shps, lts, (int(resolution[0]), int(resolution[1])), spp, max_bounces, opts


class RenderFunction(torch.autograd.Function):
    """Differentiable render of a serialized scene (see module docstring)."""

    @staticmethod
    def serialize_scene(cam, materials, shapes, lights, resolution, num_samples, max_bounces):
        args = [len(materials), len(shapes), len(lights), cam.cam_to_world, cam.world_to_cam,
                cam.sample_to_cam, cam.cam_to_sample,
                float(torch.as_tensor(cam.fov_factor).reshape(-1)[0]), cam.aspect_ratio,
                float(torch.as_tensor(cam.clip_near).reshape(-1)[0]), cam.fisheye]
        for m in materials:
            model = getattr(m, "microfacet", 0)
            args += [m.diffuse_reflectance, m.specular_reflectance, m.roughness, m.diffuse_uv_scale,
                     m.specular_uv_scale, m.roughness_uv_scale, (m.two_sided, model) if model else m.two_sided]
        for s in shapes:
            args += [s.vertices, s.indices, s.uvs, s.normals, s.mat_id]
        for l in lights:
            args += [l.shape_id, l.intensity]
        args += [resolution, num_samples, max_bounces]
        return args

    @staticmethod
    def forward(ctx, seed, *args):
        cam, mats, shps, lts, (W, H), spp, B, opts = unpack_args(args)
        opts = opts or RenderOptions()
        dev = opts.device if opts.device is not None else torch.cuda.current_device()
        scene = Scene(cam, mats, shps, lts, dev, opts.ltc_table, opts.ltc_table_ggx)
        img = scene.forward(W, H, spp, B, seed, opts)
        ctx.scene = scene
        ctx.render = (W, H, spp, B, int(seed), opts)
        ctx.arg_devices = [a.device if torch.is_tensor(a) else None for a in args]
        ctx.nargs = len(args)
        ctx.counts = (len(mats), len(shps), len(lts))
        ctx.has_normals = [s["normals"] is not None for s in shps]
        if opts.output_device is not None:
            img = img.to(opts.output_device)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        W, H, spp, B, seed, opts = ctx.render
        scene = ctx.scene
        flat, _ = scene.backward(W, H, spp, B, seed, grad_img, opts)
        # inputs all on one device (the host, typically): one copy of the flat
        # gradient there, then views of it
        devs = {d for d in ctx.arg_devices if d is not None}
        if len(devs) == 1:
            flat = flat.to(devs.pop())
        g = scene.split_grad(flat)
        nm, ns, nl = ctx.counts
        out = [None, None, None, None]  # seed, num_materials, num_shapes, num_lights
        out += [g["d_cam_to_world"], g["d_world_to_cam"], g["d_sample_to_cam"], g["d_cam_to_sample"]]
        out += [None, None, None, None]  # fov_factor, aspect_ratio, clip_near, fisheye
        for i in range(nm):
            out += [g["d_diffuse"][i], g["d_specular"][i], g["d_roughness"][i], None, None, None, None]
        for i in range(ns):
            out += [g["d_vertices"][i], None, None, g["d_normals"][i] if ctx.has_normals[i] else None, None]
        for i in range(nl):
            out += [None, g["d_intensity"][i]]
        out += [None, None, None]
        while len(out) < ctx.nargs + 1:
            out.append(None)  # RenderOptions
        # gradients live on each input's device
        res = [None]
        for grad, dev in zip(out[1:], ctx.arg_devices):
            if grad is not None and dev is not None:
                grad = grad.to(dev)
            res.append(grad)
        ctx.scene = None
        return tuple(res)
