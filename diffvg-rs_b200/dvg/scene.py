"""Scene model mirroring the diffvg-rs crate's public types.

Same names, fields and defaults as the crate so that code written against the
crate reads the same here:

* ``FilterType``, ``Filter``, ``FillRule``, ``StrokeJoin``, ``StrokeCap``,
  ``GradientStop``, ``LinearGradient``, ``RadialGradient``, ``Paint``,
  ``Circle`` / ``Ellipse`` / ``Rect`` / ``PathGeometry`` (``ShapeGeometry``),
  ``Shape``, ``ShapeGroup``, ``Scene``                  (src/scene.rs:5-291)
* ``Path``, ``PathSegment`` and ``Path.from_segments``   (src/geometry.rs:58-204)
* ``Color``                                              (src/color.rs:5-63)
* ``Mat3``                                               (src/math.rs:142-291)

``FilterType.GAUSSIAN`` is an addition of this library (the crate has none).
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

Vec2 = Tuple[float, float]


class Mat3:
    """3x3 row-major affine transform (src/math.rs:142-291)."""

    __slots__ = ("m",)

    def __init__(self, m=None):
        self.m = np.eye(3, dtype=np.float32) if m is None else np.asarray(m, dtype=np.float32).reshape(3, 3).copy()

    @staticmethod
    def identity() -> "Mat3":
        return Mat3()

    @staticmethod
    def translate(tx: float, ty: float) -> "Mat3":
        return Mat3([[1, 0, tx], [0, 1, ty], [0, 0, 1]])

    @staticmethod
    def scale(sx: float, sy: float) -> "Mat3":
        return Mat3([[sx, 0, 0], [0, sy, 0], [0, 0, 1]])

    @staticmethod
    def rotate(radians: float) -> "Mat3":
        s = np.float32(math.sin(radians))
        c = np.float32(math.cos(radians))
        return Mat3([[c, -s, 0], [s, c, 0], [0, 0, 1]])

    def mul(self, other: "Mat3") -> "Mat3":
        """self * other, evaluated in f32 as the crate does (src/math.rs:185-195)."""
        a, b = self.m, other.m
        out = np.zeros((3, 3), dtype=np.float32)
        for r in range(3):
            for c in range(3):
                out[r, c] = (a[r, 0] * b[0, c] + a[r, 1] * b[1, c]) + a[r, 2] * b[2, c]
        return Mat3(out)

    def inverse(self) -> Optional["Mat3"]:
        """Affine inverse in f32, None when |det| < 1e-6 (src/math.rs:269-290)."""
        f = np.float32
        a, b, c, d = f(self.m[0, 0]), f(self.m[0, 1]), f(self.m[1, 0]), f(self.m[1, 1])
        tx, ty = f(self.m[0, 2]), f(self.m[1, 2])
        det = f(a * d - b * c)
        if abs(det) < f(1.0e-6):
            return None
        inv_det = f(1.0) / det
        m00, m01, m10, m11 = d * inv_det, -b * inv_det, -c * inv_det, a * inv_det
        m02 = -(m00 * tx + m01 * ty)
        m12 = -(m10 * tx + m11 * ty)
        return Mat3([[m00, m01, m02], [m10, m11, m12], [0, 0, 1]])

    def transform_point(self, v: Vec2) -> Vec2:
        f = np.float32
        x = (self.m[0, 0] * f(v[0]) + self.m[0, 1] * f(v[1])) + self.m[0, 2]
        y = (self.m[1, 0] * f(v[0]) + self.m[1, 1] * f(v[1])) + self.m[1, 2]
        return (float(x), float(y))

    def flat(self) -> np.ndarray:
        return self.m.reshape(9)

    def __repr__(self) -> str:
        return f"Mat3({self.m.tolist()})"


@dataclass
class Color:
    """Linear, non-premultiplied RGBA (src/color.rs:5-63)."""

    r: float = 0.0
    g: float = 0.0
    b: float = 0.0
    a: float = 0.0

    @staticmethod
    def opaque(r: float, g: float, b: float) -> "Color":
        return Color(r, g, b, 1.0)

    def with_alpha(self, a: float) -> "Color":
        return Color(self.r, self.g, self.b, a)

    def to_tuple(self) -> Tuple[float, float, float, float]:
        return (self.r, self.g, self.b, self.a)


Color.TRANSPARENT = Color(0.0, 0.0, 0.0, 0.0)


class FilterType(enum.IntEnum):
    BOX = 0
    TENT = 1
    RADIAL_PARABOLIC = 2
    HANN = 3
    GAUSSIAN = 4  # addition of this library


@dataclass
class Filter:
    filter_type: FilterType = FilterType.BOX
    radius: float = 0.5


class FillRule(enum.IntEnum):
    NON_ZERO = 0
    EVEN_ODD = 1


class StrokeJoin(enum.IntEnum):
    MITER = 0
    BEVEL = 1
    ROUND = 2


class StrokeCap(enum.IntEnum):
    BUTT = 0
    SQUARE = 1
    ROUND = 2


@dataclass
class GradientStop:
    offset: float
    color: Color


@dataclass
class LinearGradient:
    start: Vec2
    end: Vec2
    stops: List[GradientStop] = field(default_factory=list)


@dataclass
class RadialGradient:
    center: Vec2
    radius: Vec2
    stops: List[GradientStop] = field(default_factory=list)


Paint = Union[Color, LinearGradient, RadialGradient]  # Paint::Solid is a Color


class PathSegment:
    """High-level path commands (src/geometry.rs:58-71)."""

    @dataclass
    class MoveTo:
        p: Vec2

    @dataclass
    class LineTo:
        p: Vec2

    @dataclass
    class QuadTo:
        c: Vec2
        p: Vec2

    @dataclass
    class CubicTo:
        c1: Vec2
        c2: Vec2
        p: Vec2

    @dataclass
    class Close:
        pass


@dataclass
class Path:
    """diffvg path encoding (src/geometry.rs:78-104)."""

    num_control_points: List[int] = field(default_factory=list)
    points: List[Vec2] = field(default_factory=list)
    thickness: Optional[List[float]] = None
    is_closed: bool = False
    use_distance_approx: bool = False

    @staticmethod
    def from_segments(segments: Sequence[object]) -> "Path":
        """Single-subpath conversion with the crate's rules (src/geometry.rs:110-169)."""
        points: List[Vec2] = []
        ncp: List[int] = []
        has_current = False
        is_closed = False
        for seg in segments:
            if isinstance(seg, PathSegment.MoveTo):
                if not has_current:
                    points.append(tuple(seg.p))
                    has_current = True
            elif isinstance(seg, PathSegment.LineTo):
                if has_current:
                    ncp.append(0)
                    points.append(tuple(seg.p))
                else:
                    points.append(tuple(seg.p))
                    has_current = True
            elif isinstance(seg, PathSegment.QuadTo):
                if has_current:
                    ncp.append(1)
                    points += [tuple(seg.c), tuple(seg.p)]
                else:
                    points.append(tuple(seg.p))
                    has_current = True
            elif isinstance(seg, PathSegment.CubicTo):
                if has_current:
                    ncp.append(2)
                    points += [tuple(seg.c1), tuple(seg.c2), tuple(seg.p)]
                else:
                    points.append(tuple(seg.p))
                    has_current = True
            elif isinstance(seg, PathSegment.Close):
                if has_current:
                    is_closed = True
        return Path(ncp, points, None, is_closed, False)

    def with_thickness(self, thickness: Sequence[float]) -> "Path":
        self.thickness = list(thickness)
        return self

    def with_closed(self, is_closed: bool) -> "Path":
        self.is_closed = is_closed
        return self

    def with_distance_approx(self, flag: bool) -> "Path":
        self.use_distance_approx = flag
        return self

    def is_empty(self) -> bool:
        return len(self.num_control_points) == 0 or len(self.points) == 0


@dataclass
class Circle:
    center: Vec2
    radius: float


@dataclass
class Ellipse:
    center: Vec2
    radius: Vec2


@dataclass
class Rect:
    min: Vec2
    max: Vec2


@dataclass
class PathGeometry:
    path: Path


ShapeGeometry = Union[Circle, Ellipse, Rect, PathGeometry]


@dataclass
class Shape:
    """Shape with local transform and stroke settings (src/scene.rs:184-211)."""

    geometry: ShapeGeometry
    transform: Mat3 = field(default_factory=Mat3.identity)
    stroke_width: float = 0.0
    stroke_join: StrokeJoin = StrokeJoin.ROUND
    stroke_cap: StrokeCap = StrokeCap.ROUND
    stroke_miter_limit: float = 4.0


@dataclass
class ShapeGroup:
    """Shapes sharing paints and a transform (src/scene.rs:215-257)."""

    shape_indices: List[int]
    fill: Optional[Paint] = None
    stroke: Optional[Paint] = None
    opacity: float = 1.0
    fill_rule: FillRule = FillRule.NON_ZERO
    shape_to_canvas: Mat3 = field(default_factory=Mat3.identity)
    canvas_to_shape: Mat3 = field(default_factory=Mat3.identity)

    def set_shape_to_canvas(self, m: Mat3) -> None:
        self.shape_to_canvas = m
        inv = m.inverse()
        self.canvas_to_shape = inv if inv is not None else Mat3.identity()

    def set_canvas_to_shape(self, m: Mat3) -> None:
        self.canvas_to_shape = m
        inv = m.inverse()
        self.shape_to_canvas = inv if inv is not None else Mat3.identity()


@dataclass
class Scene:
    """Root scene (src/scene.rs:261-291).  Default background is transparent, box filter r=0.5."""

    width: int
    height: int
    shapes: List[Shape] = field(default_factory=list)
    groups: List[ShapeGroup] = field(default_factory=list)
    background: Color = field(default_factory=lambda: Color(0.0, 0.0, 0.0, 0.0))
    background_image: Optional[np.ndarray] = None
    filter: Filter = field(default_factory=Filter)


@dataclass
class RenderOptions:
    """src/renderer/types.rs:10-39 (same defaults)."""

    aa: float = 1.0
    path_tolerance: float = 0.5
    samples_x: int = 2
    samples_y: int = 2
    seed: int = 0
    jitter: bool = True
    use_prefiltering: bool = True


class Rng(enum.IntEnum):
    PCG32 = 0
    PHILOX = 1


@dataclass
class BackwardOptions:
    """src/backward/render.rs:19-32 plus the boundary-sampling knobs of this library."""

    compute_translation: bool = False
    boundary_samples: int = 0  # 0 = width*height*spp (the crate)
    rng: Rng = Rng.PCG32
    boundary_seed: Optional[int] = None  # None = RenderOptions.seed (the crate)
