"""B200-native differentiable vector-graphics rasteriser: the diffvg-rs scene API
(``Scene``, ``ShapeGroup``, ``Shape``, ``Path``, paints, ``Renderer``) over the
C ABI of libdvg_b200.so."""
from .scene import (BackwardOptions, Circle, Color, Ellipse, Filter, FilterType, FillRule, GradientStop,
                    LinearGradient, Mat3, Path, PathGeometry, PathSegment, RadialGradient, Rect, RenderOptions, Rng,
                    Scene, Shape, ShapeGroup, StrokeCap, StrokeJoin)
from .abi import GradBuffers, SceneGrad, pack_scene
from .renderer import (Batch, DeviceGrads, Image, RenderError, Renderer, SdfImage, UploadedScene, device_view,
                       load_library)

__all__ = [
    "BackwardOptions", "Circle", "Color", "Ellipse", "Filter", "FilterType", "FillRule", "GradientStop",
    "LinearGradient", "Mat3", "Path", "PathGeometry", "PathSegment", "RadialGradient", "Rect", "RenderOptions",
    "Rng", "Scene", "Shape", "ShapeGroup", "StrokeCap", "StrokeJoin", "GradBuffers", "SceneGrad", "pack_scene",
    "Batch", "DeviceGrads", "Image", "device_view", "RenderError", "Renderer", "UploadedScene", "load_library", "SdfImage",
]
