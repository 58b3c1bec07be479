"""B200-native path-tracing frame (raygen, wide-BVH traversal, Disney BSDF +
next-event estimation, ReSTIR DI/GI, SVGF, TAA) behind a C ABI that mirrors the
reference renderer's NodeRenderer / PathTracerGpu interface."""
from . import presets, scenes
from .renderer import PathTracer, RendererError

__all__ = ["PathTracer", "RendererError", "presets", "scenes"]
