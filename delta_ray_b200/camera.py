"""Pinhole / fisheye camera description (mirrors the reference camera.py:7-47).

The renderer only consumes the four 4x4 matrices, ``fov_factor`` (tan of half
the field of view), ``aspect_ratio`` (width / height), ``clip_near`` and the
``fisheye`` flag; this class builds them from a look-at description exactly as
the reference does so that existing scripts keep working.
"""
import numpy as np
import torch

from . import transform


class Camera:
    def __init__(self, position, look_at, up, cam_to_world, fov, clip_near,
                 clip_far, resolution, fisheye=False):
        self.resolution = resolution
        self.num_pixels = resolution[0] * resolution[1]
        if cam_to_world is None:
            self.position = position
            self.look_at = look_at
            self.up = up
            self.cam_to_world = transform.gen_look_at_matrix(position, look_at, up)
        else:
            self.cam_to_world = cam_to_world
        self.world_to_cam = torch.inverse(self.cam_to_world)
        aspect_ratio = resolution[0] / resolution[1]
        s = torch.tensor([-0.5, -0.5 * aspect_ratio, 1.0], dtype=torch.float32)
        t = torch.tensor([-1.0, -1.0 / aspect_ratio, 0.0], dtype=torch.float32)
        s = transform.gen_scale_matrix(s)
        t = transform.gen_translate_matrix(t)
        p = transform.gen_perspective_matrix(fov, clip_near, clip_far)
        self.cam_to_sample = s @ t @ p
        self.sample_to_cam = torch.inverse(self.cam_to_sample)
        self.fov = fov
        self.fov_factor = torch.tan(transform.radians(0.5 * fov))
        self.aspect_ratio = aspect_ratio
        self.clip_near = clip_near
        self.clip_far = clip_far
        self.fisheye = fisheye
