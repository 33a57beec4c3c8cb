"""Triangle mesh description (mirrors the reference shape.py:1-6).

``vertices`` [V, 3] float32, ``indices`` [F, 3] int32, optional ``uvs`` [V, 2]
and optional per-vertex shading ``normals`` [V, 3]; ``mat_id`` indexes the
material list passed to the renderer.
"""


class Shape:
    def __init__(self, vertices, indices, uvs, normals, mat_id):
        self.vertices = vertices
        self.indices = indices
        self.uvs = uvs
        self.normals = normals
        self.mat_id = mat_id
