"""powerfoam_b200: the Power Foam rendering hot path (tile rasterizer, cell-walk
ray tracer and their adjoints) as hand-written sm_100a CUDA behind a C ABI
(libpfoam.so, include/pfoam.h), with drop-in Python classes mirroring
powerfoam/rasterize.py and powerfoam/raytrace.py."""

from .camera import TorchCamera, look_at
from .rasterize import TILE_WIDTH, Rasterizer, RasterGradFn, VisOptions
from .raytrace import RayTracer

__all__ = ["TorchCamera", "look_at", "Rasterizer", "RasterGradFn", "VisOptions", "RayTracer", "TILE_WIDTH"]
