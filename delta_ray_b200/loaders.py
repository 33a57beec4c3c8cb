"""Scene loaders: Mitsuba 0.5 XML scenes, Mitsuba ``.serialized`` meshes and
Wavefront OBJ files, producing this package's Camera / Material / Shape /
Light objects (the inputs of ``RenderFunction.serialize_scene``).

They follow the reference's loaders:

* ``load_mitsuba``    load_mitsuba.py:1-287: ``sensor`` (fov, ``toWorld``
  look-at or transform chain, film size), ``bsdf`` of type ``diffuse`` (rgb
  or texture ``reflectance`` / ``specular``, ``roughness``) and ``twosided``,
  ``shape`` of type ``serialized``, ``obj`` and ``rectangle`` with an
  optional ``area`` emitter.  As in the reference, a shape without a bsdf
  reference takes the last material (its material id is -1), and normals are
  transformed by the inverse transpose without renormalising.
* ``load_serialized`` load_serialized.cpp:1-277: the Mitsuba mesh format
  (versions 3 and 4: a 2-byte magic, 2-byte version, then a zlib stream with
  flags, name (v4), vertex and triangle counts, positions, optional normals,
  texture coordinates and colors in single or double precision, and 32-bit
  indices; a file holding several meshes ends with their byte offsets and
  their count).
* ``load_obj``        load_obj.py:6-83: one output vertex per distinct
  (position, uv, normal) index triple, quads split into two triangles.
  Negative (relative) indices count back from the end of the position,
  texture-coordinate and normal lists as the OBJ format defines; the
  reference offsets them by its own output arrays instead.

Textures are read from ``.npy`` files (the reference reads images through
OpenEXR / scikit-image, which this package does not depend on).
"""
import os
import struct
import xml.etree.ElementTree as etree
import zlib

import numpy as np
import torch

from . import transform
from .camera import Camera
from .light import Light
from .material import Material
from .shape import Shape

_HAS_NORMALS = 0x0001
_HAS_TEXCOORDS = 0x0002
_HAS_COLORS = 0x0008
_DOUBLE_PRECISION = 0x2000
_MAGIC = 0x041C


def _f32(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float32)))


# ---------------------------------------------------------------------------
# Mitsuba .serialized
# ---------------------------------------------------------------------------
def load_serialized(filename, shape_index=0):
    """(indices [F, 3] int32, vertices [V, 3] float32, uvs [V, 2] or [0, 2],
    normals [V, 3] or [0, 3]) of mesh ``shape_index`` of a .serialized file."""
    with open(filename, "rb") as f:
        data = f.read()
    if len(data) < 8:
        raise ValueError(f"{filename}: too short for a serialized mesh")
    magic, version = struct.unpack_from("<HH", data, 0)
    if magic != _MAGIC or version not in (3, 4):
        raise ValueError(f"{filename}: not a Mitsuba serialized mesh (magic {magic:#x}, version {version})")
    start = 4
    if shape_index > 0:
        (count,) = struct.unpack_from("<I", data, len(data) - 4)
        if shape_index >= count:
            raise ValueError(f"{filename}: mesh {shape_index} requested, the file holds {count}")
        if version == 4:
            (offset,) = struct.unpack_from("<Q", data, len(data) - 4 - 8 * (count - shape_index))
        else:
            (offset,) = struct.unpack_from("<I", data, len(data) - 4 * (count - shape_index + 1))
        start = offset + 4  # skip that mesh's magic and version
    z = zlib.decompressobj()
    raw = z.decompress(data[start:])
    pos = 0

    def take(fmt, n=1):
        nonlocal pos
        size = np.dtype(fmt).itemsize * n
        if pos + size > len(raw):
            raise ValueError(f"{filename}: mesh data ends early")
        out = np.frombuffer(raw, dtype=np.dtype(fmt), count=n, offset=pos)
        pos += size
        return out

    flags = int(take("<u4")[0])
    if version == 4:
        end = raw.index(b"\0", pos)
        pos = end + 1  # mesh name
    nv = int(take("<u8")[0])
    nt = int(take("<u8")[0])
    real = "<f8" if flags & _DOUBLE_PRECISION else "<f4"
    vertices = take(real, 3 * nv).astype(np.float32).reshape(nv, 3)
    normals = np.zeros((0, 3), np.float32)
    uvs = np.zeros((0, 2), np.float32)
    if flags & _HAS_NORMALS:
        normals = take(real, 3 * nv).astype(np.float32).reshape(nv, 3)
    if flags & _HAS_TEXCOORDS:
        uvs = take(real, 2 * nv).astype(np.float32).reshape(nv, 2)
    if flags & _HAS_COLORS:
        take(real, 3 * nv)  # vertex colors: not used by the renderer
    indices = take("<u4", 3 * nt).astype(np.int32).reshape(nt, 3)
    return indices, vertices, uvs, normals


def write_serialized(filename, meshes, version=4, double_precision=False):
    """Writes meshes [(indices, vertices, uvs or None, normals or None, name)]
    as a Mitsuba .serialized file (the inverse of load_serialized)."""
    real = "<f8" if double_precision else "<f4"
    blobs = []
    for indices, vertices, uvs, normals, name in meshes:
        flags = (_DOUBLE_PRECISION if double_precision else 0x1000)
        flags |= _HAS_NORMALS if normals is not None else 0
        flags |= _HAS_TEXCOORDS if uvs is not None else 0
        body = struct.pack("<I", flags)
        if version == 4:
            body += name.encode() + b"\0"
        v = np.asarray(vertices)
        body += struct.pack("<QQ", v.shape[0], np.asarray(indices).shape[0])
        body += v.astype(real).tobytes()
        if normals is not None:
            body += np.asarray(normals).astype(real).tobytes()
        if uvs is not None:
            body += np.asarray(uvs).astype(real).tobytes()
        body += np.asarray(indices).astype("<u4").tobytes()
        blobs.append(struct.pack("<HH", _MAGIC, version) + zlib.compress(body))
    offsets, out = [], b""
    for b in blobs:
        offsets.append(len(out))
        out += b
    fmt = "<Q" if version == 4 else "<I"
    out += b"".join(struct.pack(fmt, o) for o in offsets) + struct.pack("<I", len(blobs))
    with open(filename, "wb") as f:
        f.write(out)


# ---------------------------------------------------------------------------
# Wavefront OBJ
# ---------------------------------------------------------------------------
def load_obj(filename):
    """(indices [F, 3] int32, vertices [V, 3] float32, uvs [V, 2] or None,
    normals [V, 3] or None)."""
    pos_pool, uv_pool, n_pool = [], [], []
    vertices, uvs, normals, indices = [], [], [], []
    vmap = {}

    def resolve(s, pool_len):
        i = int(s)
        return i - 1 if i > 0 else pool_len + i

    def vertex_id(token):
        parts = token.split("/")
        pi = resolve(parts[0], len(pos_pool))
        ti = resolve(parts[1], len(uv_pool)) if len(parts) > 1 and parts[1] != "" else None
        ni = resolve(parts[2], len(n_pool)) if len(parts) > 2 and parts[2] != "" else None
        key = (pi, ti, ni)
        vid = vmap.get(key)
        if vid is None:
            vid = len(vertices)
            vmap[key] = vid
            vertices.append(pos_pool[pi])
            if ti is not None:
                uvs.append(uv_pool[ti])
            if ni is not None:
                normals.append(n_pool[ni])
        return vid

    with open(filename, "r") as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "v":
                pos_pool.append([float(x) for x in tok[1:4]])
            elif tok[0] == "vt":
                uv_pool.append([float(x) for x in tok[1:3]])
            elif tok[0] == "vn":
                n_pool.append([float(x) for x in tok[1:4]])
            elif tok[0] == "f":
                if len(tok) > 5:
                    raise ValueError(f"{filename}: faces with more than 4 vertices are not supported")
                ids = [vertex_id(t) for t in tok[1:]]
                indices.append([ids[0], ids[1], ids[2]])
                if len(ids) == 4:
                    indices.append([ids[0], ids[2], ids[3]])
    out_uv = np.array(uvs, np.float32) if uvs else None
    out_n = np.array(normals, np.float32) if normals else None
    return np.array(indices, np.int32).reshape(-1, 3), np.array(vertices, np.float32).reshape(-1, 3), out_uv, out_n


# ---------------------------------------------------------------------------
# Mitsuba XML
# ---------------------------------------------------------------------------
def _vector(s):
    v = np.array([float(x) for x in s.replace(",", " ").split()], np.float32)
    return v


def _transform(node):
    m = np.identity(4, dtype=np.float32)
    for c in node:
        if c.tag == "matrix":
            t = np.array([float(x) for x in c.attrib["value"].split()], np.float32).reshape(4, 4)
        elif c.tag == "translate":
            t = transform.gen_translate_matrix(
                _f32([float(c.attrib.get(k, 0.0)) for k in "xyz"])).numpy()
        elif c.tag == "scale":
            t = transform.gen_scale_matrix(_f32([float(c.attrib.get(k, 1.0)) for k in "xyz"])).numpy()
        else:
            continue
        m = t @ m
    return m


def _texture(node):
    tex, us, vs = None, 1.0, 1.0
    for c in node:
        name = c.attrib.get("name")
        if name == "filename":
            path = c.attrib["value"]
            if not path.endswith(".npy"):
                raise ValueError(f"texture {path}: only .npy textures are supported")
            tex = _f32(np.load(path))
        elif name == "uscale":
            us = float(c.attrib["value"])
        elif name == "vscale":
            vs = float(c.attrib["value"])
    return tex, _f32([us, vs])


def _camera(node):
    fov = _f32([45.0])
    to_world = np.identity(4, dtype=np.float32)
    look = None
    resolution = [256, 256]
    for c in node:
        name = c.attrib.get("name")
        if name == "fov":
            fov = _f32([float(c.attrib["value"])])
        elif name == "toWorld":
            la = [g for g in c if g.tag == "lookat"]
            if la:
                g = la[0]
                look = (_f32(_vector(g.attrib["origin"])), _f32(_vector(g.attrib["target"])),
                        _f32(_vector(g.attrib["up"])))
            else:
                to_world = _transform(c)
        if c.tag == "film":
            for g in c:
                if g.attrib.get("name") == "width":
                    resolution[0] = int(g.attrib["value"])
                elif g.attrib.get("name") == "height":
                    resolution[1] = int(g.attrib["value"])
    clip_near, clip_far = _f32([0.01]), _f32([10000.0])
    if look is not None:
        cam = Camera(look[0], look[1], look[2], None, fov, clip_near, clip_far, resolution)
    else:
        cam = Camera(None, None, None, _f32(to_world), fov, clip_near, clip_far, resolution)
    return cam, resolution


def _material(node, two_sided=False):
    node_id = node.attrib.get("id")
    kind = node.attrib["type"]
    if kind == "twosided":
        return node_id, _material(node[0], True)[1]
    if kind != "diffuse":
        raise ValueError(f"bsdf type {kind!r} is not supported (diffuse and twosided are)")
    kd, kd_uv = _f32([0.5, 0.5, 0.5]), _f32([1.0, 1.0])
    ks, ks_uv = _f32([0.0, 0.0, 0.0]), _f32([1.0, 1.0])
    rough = _f32([1.0])
    for c in node:
        name = c.attrib.get("name")
        if name == "reflectance":
            if c.tag == "texture":
                kd, kd_uv = _texture(c)
            elif c.tag == "rgb":
                kd = _f32(_vector(c.attrib["value"]))
        elif name == "specular":
            if c.tag == "texture":
                ks, ks_uv = _texture(c)
            elif c.tag == "rgb":
                ks = _f32(_vector(c.attrib["value"]))
        elif name == "roughness":
            rough = _f32([float(c.attrib["value"])])
    return node_id, Material(kd, specular_reflectance=ks, roughness=rough, diffuse_uv_scale=kd_uv,
                             specular_uv_scale=ks_uv, two_sided=two_sided)


def _radiance(emitter):
    for g in emitter:
        if g.attrib.get("name") == "radiance":
            v = _vector(g.attrib["value"])
            return _f32(np.repeat(v, 3) if v.shape[0] == 1 else v)
    return None


def _shape(node, material_ids, shape_id, base_dir):
    kind = node.attrib["type"]
    to_world = np.identity(4, dtype=np.float32)
    mesh_index, mat_id, radiance, filename = 0, -1, None, ""
    for c in node:
        name = c.attrib.get("name")
        if name == "filename":
            filename = os.path.join(base_dir, c.attrib["value"])
        elif name == "toWorld":
            to_world = _transform(c)
        elif name == "shapeIndex":
            mesh_index = int(c.attrib["value"])
        if c.tag == "ref":
            mat_id = material_ids[c.attrib["id"]]
        elif c.tag == "emitter":
            radiance = _radiance(c)
    if kind == "serialized":
        indices, vertices, uvs, normals = load_serialized(filename, mesh_index)
        uvs = uvs if uvs.shape[0] else None
        normals = normals if normals.shape[0] else None
    elif kind == "obj":
        indices, vertices, uvs, normals = load_obj(filename)
    elif kind == "rectangle":
        indices = np.array([[0, 2, 1], [1, 2, 3]], np.int32)
        vertices = np.array([[-1, -1, 0], [-1, 1, 0], [1, -1, 0], [1, 1, 0]], np.float32)
        uvs = normals = None
    else:
        raise ValueError(f"shape type {kind!r} is not supported (serialized, obj and rectangle are)")
    hom = np.concatenate([vertices, np.ones((vertices.shape[0], 1), np.float32)], 1) @ to_world.T
    vertices = (hom[:, :3] / hom[:, 3:4]).astype(np.float32)
    if normals is not None:
        normals = (normals @ np.linalg.inv(to_world.T)[:3, :3]).astype(np.float32)
    light = Light(shape_id, radiance) if radiance is not None else None
    shape = Shape(_f32(vertices), torch.from_numpy(np.ascontiguousarray(indices, np.int32)),
                  None if uvs is None else _f32(uvs), None if normals is None else _f32(normals), mat_id)
    return shape, light


def load_mitsuba(filename):
    """(camera, materials, shapes, lights, resolution) of a Mitsuba XML scene;
    file names inside it are relative to the scene's directory."""
    root = etree.parse(filename).getroot()
    base_dir = os.path.dirname(os.path.abspath(filename))
    cam, resolution = None, None
    materials, material_ids, shapes, lights = [], {}, [], []
    for c in root:
        if c.tag == "sensor":
            cam, resolution = _camera(c)
        elif c.tag == "bsdf":
            node_id, m = _material(c)
            if node_id is not None:
                material_ids[node_id] = len(materials)
                materials.append(m)
        elif c.tag == "shape":
            s, l = _shape(c, material_ids, len(shapes), base_dir)
            shapes.append(s)
            if l is not None:
                lights.append(l)
    for s in shapes:  # material id -1 (no bsdf reference) indexes the last material, as in the reference
        if s.mat_id < 0:
            s.mat_id = len(materials) + s.mat_id
    return cam, materials, shapes, lights, resolution
