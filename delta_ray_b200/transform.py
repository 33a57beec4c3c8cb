"""Camera transforms: look-at, scale, translate and perspective 4x4 matrices.

Mirrors the reference helpers transform.py:6-47 (radians, normalize,
gen_look_at_matrix, gen_scale_matrix, gen_translate_matrix,
gen_perspective_matrix) so that scenes built with this package produce the same
matrices as scenes built with the reference.  All functions take and return
torch tensors and stay differentiable.
"""
import math

import torch


def radians(deg):
    return (math.pi / 180.0) * deg


def normalize(v):
    return v / torch.norm(v)


def gen_look_at_matrix(pos, look, up):
    """Camera-to-world matrix whose columns are (left, up, forward, position).

    Same construction as transform.py:12-22 of the reference: forward is
    normalize(look - pos), left = normalize(cross(up, forward)) and the
    recomputed up = normalize(cross(forward, left)).
    """
    fwd = normalize(look - pos)
    left = normalize(torch.cross(normalize(up), fwd, dim=0))
    new_up = normalize(torch.cross(fwd, left, dim=0))
    zero = torch.zeros(1, dtype=torch.float32)
    one = torch.ones(1, dtype=torch.float32)
    cols = [torch.cat([left, zero]), torch.cat([new_up, zero]),
            torch.cat([fwd, zero]), torch.cat([pos, one])]
    return torch.stack(cols, dim=1)


def gen_scale_matrix(scale):
    return torch.diag(torch.cat([scale, torch.ones(1, dtype=torch.float32)]))


def gen_translate_matrix(translate):
    m = torch.eye(4, dtype=torch.float32)
    m = m.clone()
    m[0:3, 3] = translate
    return m


def gen_perspective_matrix(fov, clip_near, clip_far):
    """Perspective projection as in transform.py:32-41 of the reference."""
    clip_dist = clip_far - clip_near
    cot = 1.0 / torch.tan(radians(fov / 2.0))
    z = torch.zeros(1, dtype=torch.float32)
    o = torch.ones(1, dtype=torch.float32)
    return torch.stack([torch.cat([cot, z, z, z]),
                        torch.cat([z, cot, z, z]),
                        torch.cat([z, z, 1 / clip_dist, -clip_near / clip_dist]),
                        torch.cat([z, z, o, z])])
