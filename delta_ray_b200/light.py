"""Area light description (mirrors the reference light.py:1-3).

A light turns every triangle of shape ``shape_id`` into a one-sided emitter of
radiance ``intensity`` [3] (emitting on the side of the geometric normal).
"""


class Light:
    def __init__(self, shape_id, intensity):
        self.shape_id = shape_id
        self.intensity = intensity
