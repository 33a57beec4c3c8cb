"""delta_ray_b200: a B200-native differentiable edge-sampling path tracer.

Drop-in for the reference's ``render_pytorch.RenderFunction`` API.  The CUDA
library (libdr_b200.so) is loaded lazily on first render; there is no CPU
fallback.
"""
from .camera import Camera
from .light import Light
from .material import Material
from .render_pytorch import RenderFunction, RenderOptions, Scene
from .shape import Shape

__all__ = ["Camera", "Light", "Material", "RenderFunction", "RenderOptions", "Scene", "Shape"]
