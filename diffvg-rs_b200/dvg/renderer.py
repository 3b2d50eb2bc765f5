"""``Renderer`` over the C ABI of libdvg_b200.so (include/dvg.h).

Mirrors the crate's ``Renderer`` (src/renderer/renderer.rs:20-564):
``Renderer(device).render(scene, options) -> Image`` and
``render_backward(scene, options, backward_options, d_render_image, d_sdf_image) -> SceneGrad``.
Errors raise ``RenderError`` with the crate's kinds (``InvalidScene``,
``Launch``).  There is no CPU fallback: without the CUDA library or a device
the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .abi import (
    BackwardOptionsC,
    GradBuffers,
    GradsC,
    PackedScene,
    RenderOptionsC,
    SceneDesc,
    backward_options_c,
    pack_scene,
    render_options_c,
    unflatten_grads,
)
from .scene import BackwardOptions, RenderOptions, Scene

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libdvg_b200.so")

DVG_OK, DVG_ERR_INVALID_SCENE, DVG_ERR_LAUNCH, DVG_ERR_DEVICE_LIMIT = 0, 1, 2, 3
DVG_ERR_INVALID_ARGUMENT, DVG_ERR_OUT_OF_MEMORY, DVG_ERR_NO_DEVICE = 4, 5, 6

EXPORTED = (
    "dvg_abi_version", "dvg_last_error", "dvg_context_create", "dvg_context_destroy", "dvg_scene_upload",
    "dvg_scene_destroy", "dvg_render_host", "dvg_render_device", "dvg_render_backward_host",
    "dvg_render_backward_device", "dvg_render", "dvg_render_backward", "dvg_fwd_bwd_l2_device",
    "dvg_context_launch_count", "dvg_context_stream", "dvg_context_set_profiling", "dvg_context_profile",
    "dvg_context_profile_reset", "dvg_batch_create", "dvg_batch_destroy", "dvg_batch_buffers", "dvg_batch_step",
    "dvg_batch_losses", "dvg_render_device_noalloc", "dvg_batch_set_adam", "dvg_batch_scene_params",
    "dvg_scene_digest", "dvg_render_sdf_host", "dvg_render_sdf_device", "dvg_render_sdf",
    "dvg_eval_positions_host", "dvg_eval_positions_device", "dvg_eval_positions",
    "dvg_eval_positions_backward_host", "dvg_eval_positions_backward_device", "dvg_eval_positions_backward",
    "dvg_lbvh_build", "dvg_scene_set_tuning", "dvg_scene_get_tuning", "dvg_scene_autotune", "dvg_batch_set_tuning",
    "dvg_batch_autotune",
)


class ShardC(C.Structure):
    _fields_ = [("tile_begin", C.c_uint32), ("tile_end", C.c_uint32), ("sample_begin", C.c_uint64),
                ("sample_end", C.c_uint64)]


def _tuple(t):
    return (int(t.sample_layout), int(t.boundary_cell), int(t.fragment_slots), int(t.work_queue),
            int(t.forward_occupancy))


class TuningC(C.Structure):
    _fields_ = [("sample_layout", C.c_uint32), ("boundary_cell", C.c_uint32), ("fragment_slots", C.c_uint32),
                ("work_queue", C.c_uint32), ("forward_occupancy", C.c_uint32)]


class AdamOptionsC(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("params", C.c_uint32)]


OPT_POINTS = 1
OPT_PAINTS = 2


class RenderError(RuntimeError):
    """RenderError (src/renderer/types.rs:83-88); ``kind`` is 'InvalidScene', 'Launch', ..."""

    KINDS = {DVG_ERR_INVALID_SCENE: "InvalidScene", DVG_ERR_LAUNCH: "Launch", DVG_ERR_DEVICE_LIMIT: "DeviceLimit",
             DVG_ERR_INVALID_ARGUMENT: "InvalidArgument", DVG_ERR_OUT_OF_MEMORY: "OutOfMemory",
             DVG_ERR_NO_DEVICE: "NoDevice"}

    def __init__(self, status: int, message: str):
        self.status = status
        self.kind = self.KINDS.get(status, f"Status{status}")
        super().__init__(f"{self.kind}: {message}")


_lib: Optional[C.CDLL] = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `make -C diffvg-rs_b200` (nvcc, sm_100a)")
    L = C.CDLL(path)
    D = C.POINTER(SceneDesc)
    R = C.POINTER(RenderOptionsC)
    B = C.POINTER(BackwardOptionsC)
    Gp = C.POINTER(GradsC)
    fp = C.POINTER(C.c_float)
    vp = C.c_void_p
    L.dvg_abi_version.restype = C.c_uint32
    L.dvg_last_error.restype = C.c_char_p
    L.dvg_context_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.dvg_context_destroy.argtypes = [vp]
    L.dvg_context_destroy.restype = None
    L.dvg_scene_upload.argtypes = [vp, D, C.POINTER(vp)]
    L.dvg_scene_destroy.argtypes = [vp]
    L.dvg_scene_destroy.restype = None
    L.dvg_render_host.argtypes = [vp, vp, R, fp]
    L.dvg_render_device.argtypes = [vp, vp, R, vp]
    L.dvg_render_backward_host.argtypes = [vp, vp, R, B, fp, fp, Gp]
    L.dvg_render_backward_device.argtypes = [vp, vp, R, B, vp, vp, Gp]
    L.dvg_render.argtypes = [vp, D, R, fp]
    L.dvg_render_backward.argtypes = [vp, D, R, B, fp, fp, Gp]
    L.dvg_fwd_bwd_l2_device.argtypes = [vp, vp, R, B, vp, vp, vp, Gp]
    L.dvg_context_launch_count.argtypes = [vp]
    L.dvg_context_launch_count.restype = C.c_uint64
    L.dvg_context_stream.argtypes = [vp]
    L.dvg_context_stream.restype = vp
    L.dvg_context_set_profiling.argtypes = [vp, C.c_int]
    L.dvg_context_set_profiling.restype = C.c_int
    L.dvg_context_set_retain.argtypes = [vp, C.c_int]
    L.dvg_context_set_retain.restype = C.c_int
    Sh = C.POINTER(ShardC)
    L.dvg_scene_tile_count.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.dvg_scene_tile_groups.argtypes = [vp, C.POINTER(C.c_uint32), C.c_uint32]
    L.dvg_shard_forward.argtypes = [vp, vp, R, Sh, vp, vp]
    L.dvg_shard_resolve.argtypes = [vp, vp, vp, vp, vp]
    L.dvg_l2_device.argtypes = [vp, vp, vp, C.c_uint64, vp, vp]
    L.dvg_shard_backward.argtypes = [vp, vp, R, B, Sh, vp, vp, Gp]
    for f in ("dvg_scene_tile_count", "dvg_scene_tile_groups", "dvg_shard_forward", "dvg_shard_resolve", "dvg_l2_device",
              "dvg_shard_backward"):
        getattr(L, f).restype = C.c_int
    L.dvg_context_profile.argtypes = [vp, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                      C.c_int]
    L.dvg_context_profile.restype = C.c_int
    L.dvg_context_profile_reset.argtypes = [vp]
    L.dvg_context_profile_reset.restype = None
    L.dvg_batch_create.argtypes = [vp, C.POINTER(vp), C.c_uint32, R, B, C.POINTER(vp)]
    L.dvg_batch_destroy.argtypes = [vp]
    L.dvg_batch_destroy.restype = None
    L.dvg_batch_buffers.argtypes = [vp, C.c_uint32, C.POINTER(vp), C.POINTER(vp), Gp]
    L.dvg_batch_step.argtypes = [vp, C.c_int]
    L.dvg_batch_losses.argtypes = [vp, fp]
    L.dvg_batch_set_adam.argtypes = [vp, C.POINTER(AdamOptionsC)]
    L.dvg_scene_digest.argtypes = [vp, vp, C.POINTER(C.c_uint64)]
    L.dvg_lbvh_build.argtypes = [vp, fp, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_int32), fp]
    L.dvg_lbvh_build.restype = C.c_int
    L.dvg_scene_set_tuning.argtypes = [vp, C.POINTER(TuningC)]
    L.dvg_scene_get_tuning.argtypes = [vp, C.POINTER(TuningC)]
    L.dvg_scene_autotune.argtypes = [vp, vp, R, B, vp, C.POINTER(TuningC)]
    L.dvg_batch_set_tuning.argtypes = [vp, C.POINTER(TuningC)]
    L.dvg_batch_autotune.argtypes = [vp, C.POINTER(TuningC)]
    for name in ("dvg_scene_set_tuning", "dvg_scene_get_tuning", "dvg_scene_autotune", "dvg_batch_set_tuning",
                 "dvg_batch_autotune"):
        getattr(L, name).restype = C.c_int
    L.dvg_render_sdf_host.argtypes = [vp, vp, R, fp]
    L.dvg_render_sdf_device.argtypes = [vp, vp, R, vp]
    L.dvg_render_sdf.argtypes = [vp, D, R, fp]
    L.dvg_eval_positions_host.argtypes = [vp, vp, fp, C.c_uint64, fp]
    L.dvg_eval_positions_device.argtypes = [vp, vp, vp, C.c_uint64, vp]
    L.dvg_eval_positions.argtypes = [vp, D, fp, C.c_uint64, fp]
    L.dvg_eval_positions_backward_host.argtypes = [vp, vp, B, fp, C.c_uint64, fp, Gp]
    L.dvg_eval_positions_backward_device.argtypes = [vp, vp, B, vp, C.c_uint64, vp, Gp]
    L.dvg_eval_positions_backward.argtypes = [vp, D, B, fp, C.c_uint64, fp, Gp]
    for name in ("dvg_render_sdf_host", "dvg_render_sdf_device", "dvg_render_sdf", "dvg_eval_positions_host",
                 "dvg_eval_positions_device", "dvg_eval_positions", "dvg_eval_positions_backward_host",
                 "dvg_eval_positions_backward_device", "dvg_eval_positions_backward"):
        getattr(L, name).restype = C.c_int
    L.dvg_scene_digest.restype = C.c_int
    L.dvg_batch_scene_params.argtypes = [vp, C.c_uint32, fp, fp]
    for name in ("dvg_batch_create", "dvg_batch_buffers", "dvg_batch_step", "dvg_batch_losses", "dvg_batch_set_adam",
                 "dvg_batch_scene_params"):
        getattr(L, name).restype = C.c_int
    for name in ("dvg_context_create", "dvg_scene_upload", "dvg_render_host", "dvg_render_device",
                 "dvg_render_backward_host", "dvg_render_backward_device", "dvg_render", "dvg_render_backward",
                 "dvg_fwd_bwd_l2_device"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _check(status: int) -> None:
    if status != DVG_OK:
        msg = load_library().dvg_last_error()
        raise RenderError(status, msg.decode() if msg else "")


def _fp(a: Optional[np.ndarray]):
    if a is None:
        return C.cast(None, C.POINTER(C.c_float))
    return a.ctypes.data_as(C.POINTER(C.c_float))


@dataclass
class Image:
    """Image (src/renderer/types.rs:43-50): linear RGBA, row-major."""

    width: int
    height: int
    pixels: np.ndarray  # float32 [height, width, 4]


@dataclass
class SdfImage:
    """SdfImage (src/renderer/types.rs): per-pixel signed distance, row-major."""

    width: int
    height: int
    values: np.ndarray  # float32 [height, width]


class DeviceGrads:
    """dvg_grads pointing at caller-owned device buffers (torch tensors)."""

    def __init__(self, packed: PackedScene, torch_device, translation: bool = False):
        import torch

        d = packed.desc
        npix = int(d.width) * int(d.height)
        sizes = dict(
            d_shape_params=4 * d.num_shapes, d_shape_transform=9 * d.num_shapes,
            d_shape_stroke_width=d.num_shapes, d_points=2 * d.total_points, d_thickness=d.total_points,
            d_group_transform=9 * d.num_groups, d_paint_params=4 * d.num_paints, d_stop_offsets=d.total_stops,
            d_stop_colors=4 * d.total_stops, d_filter_radius=1, d_background=4,
            d_background_image=4 * npix if packed.desc.background_image else 0,
            d_translation=2 * npix if translation else 0,
        )
        self.tensors = {}
        self.c = GradsC()
        # one device buffer (parts at 256-byte offsets), so a single collective can sum
        # the gradients of a scene split over several processes
        offs, total = {}, 0
        for n in GradBuffers.NAMES:
            sz = int(sizes[n])
            if n in ("d_background_image", "d_translation") and sz == 0:
                continue
            offs[n] = (total, max(sz, 1))
            total += (max(sz, 1) + 63) // 64 * 64
        self.buffer = torch.zeros(max(total, 1), dtype=torch.float32, device=torch_device)
        for n in GradBuffers.NAMES:
            if n not in offs:
                setattr(self.c, n, C.cast(None, C.POINTER(C.c_float)))
                continue
            o, sz = offs[n]
            t = self.buffer[o:o + sz]
            self.tensors[n] = t
            setattr(self.c, n, C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)))

    def flat(self):
        import torch

        return torch.cat([t for t in self.tensors.values()])


class UploadedScene:
    """A scene prepared and resident in HBM (dvg_scene_upload)."""

    def __init__(self, renderer: "Renderer", scene: Scene, packed: Optional[PackedScene] = None):
        self.renderer = renderer
        self.scene = scene
        self.packed = packed if packed is not None else pack_scene(scene)
        self.handle = C.c_void_p()
        _check(renderer.lib.dvg_scene_upload(renderer.ctx, self.packed.ref(), C.byref(self.handle)))
        renderer._children.add(self)

    def close(self) -> None:
        if self.handle and self.renderer.ctx:
            self.renderer.lib.dvg_scene_destroy(self.handle)
        self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_host(self, options: RenderOptions) -> np.ndarray:
        out = np.zeros((self.scene.height, self.scene.width, 4), np.float32)
        o = render_options_c(options)
        _check(self.renderer.lib.dvg_render_host(self.renderer.ctx, self.handle, C.byref(o), _fp(out)))
        return out

    def render_device(self, options: RenderOptions, out_ptr: int) -> None:
        o = render_options_c(options)
        _check(self.renderer.lib.dvg_render_device(self.renderer.ctx, self.handle, C.byref(o), C.c_void_p(out_ptr)))

    def backward_device(self, options: RenderOptions, bopts: Optional[BackwardOptions], d_render_ptr: int,
                        grads: DeviceGrads) -> None:
        o = render_options_c(options)
        b = backward_options_c(bopts)
        _check(self.renderer.lib.dvg_render_backward_device(self.renderer.ctx, self.handle, C.byref(o), C.byref(b),
                                                            C.c_void_p(d_render_ptr), None, C.byref(grads.c)))

    def tuning(self):
        """(sample_layout, boundary_cell, fragment_slots, work_queue, forward_occupancy) used by this
        scene's launches."""
        t = TuningC()
        _check(self.renderer.lib.dvg_scene_get_tuning(self.handle, C.byref(t)))
        return _tuple(t)

    def set_tuning(self, sample_layout: int, boundary_cell: int, fragment_slots: int = 16, work_queue: int = 0,
                   forward_occupancy: int = 0) -> None:
        t = TuningC(sample_layout, boundary_cell, fragment_slots, work_queue, forward_occupancy)
        _check(self.renderer.lib.dvg_scene_set_tuning(self.handle, C.byref(t)))

    def autotune(self, options: RenderOptions, bopts: Optional[BackwardOptions], target_ptr: int):
        """dvg_scene_autotune against a device target image; returns the chosen tuning."""
        o = render_options_c(options)
        b = backward_options_c(bopts)
        t = TuningC()
        _check(self.renderer.lib.dvg_scene_autotune(self.renderer.ctx, self.handle, C.byref(o), C.byref(b),
                                                    C.c_void_p(target_ptr), C.byref(t)))
        return _tuple(t)

    def tile_count(self) -> int:
        """dvg_scene_tile_count: 16x16 tiles of the canvas (the unit of a shard's band)."""
        n = C.c_uint32()
        _check(self.renderer.lib.dvg_scene_tile_count(self.handle, C.byref(n)))
        return int(n.value)

    def tile_groups(self) -> np.ndarray:
        """dvg_scene_tile_groups: groups binned to each tile (the per-tile work estimate)."""
        n = self.tile_count()
        out = np.zeros(max(n, 1), np.uint32)
        _check(self.renderer.lib.dvg_scene_tile_groups(self.handle, out.ctypes.data_as(C.POINTER(C.c_uint32)), n))
        return out[:n]

    def shard_forward(self, options: RenderOptions, tiles, accum_ptr: int, wsum_ptr: int) -> None:
        """dvg_shard_forward over tiles [begin, end) into zeroed device accumulators."""
        o = render_options_c(options)
        sh = ShardC(int(tiles[0]), int(tiles[1]), 0, 0)
        _check(self.renderer.lib.dvg_shard_forward(self.renderer.ctx, self.handle, C.byref(o), C.byref(sh),
                                                   C.c_void_p(accum_ptr), C.c_void_p(wsum_ptr)))

    def shard_resolve(self, accum_ptr: int, wsum_ptr: int, out_ptr: int) -> None:
        _check(self.renderer.lib.dvg_shard_resolve(self.renderer.ctx, self.handle, C.c_void_p(accum_ptr),
                                                   C.c_void_p(wsum_ptr), C.c_void_p(out_ptr)))

    def shard_backward(self, options: RenderOptions, bopts: Optional[BackwardOptions], tiles, samples,
                       d_render_ptr: int, wsum_ptr: int, grads: "DeviceGrads") -> None:
        """dvg_shard_backward: tiles [begin, end), boundary samples [begin, end)."""
        o = render_options_c(options)
        b = backward_options_c(bopts)
        sh = ShardC(int(tiles[0]), int(tiles[1]), int(samples[0]), int(samples[1]))
        _check(self.renderer.lib.dvg_shard_backward(self.renderer.ctx, self.handle, C.byref(o), C.byref(b),
                                                    C.byref(sh), C.c_void_p(d_render_ptr), C.c_void_p(wsum_ptr),
                                                    C.byref(grads.c)))

    def render_sdf_device(self, options: RenderOptions, out_ptr: int) -> None:
        """dvg_render_sdf_device into width*height floats of device memory."""
        o = render_options_c(options)
        _check(self.renderer.lib.dvg_render_sdf_device(self.renderer.ctx, self.handle, C.byref(o), C.c_void_p(out_ptr)))

    def digest(self) -> int:
        """dvg_scene_digest: hash of the prepared device tables."""
        out = C.c_uint64()
        _check(self.renderer.lib.dvg_scene_digest(self.renderer.ctx, self.handle, C.byref(out)))
        return int(out.value)

    def fwd_bwd_l2_device(self, options: RenderOptions, bopts: Optional[BackwardOptions], target_ptr: int,
                          out_ptr: Optional[int], loss_ptr: Optional[int], grads: DeviceGrads) -> None:
        o = render_options_c(options)
        b = backward_options_c(bopts)
        _check(self.renderer.lib.dvg_fwd_bwd_l2_device(
            self.renderer.ctx, self.handle, C.byref(o), C.byref(b), C.c_void_p(target_ptr),
            C.c_void_p(out_ptr) if out_ptr else None, C.c_void_p(loss_ptr) if loss_ptr else None, C.byref(grads.c)))


class Renderer:
    """Renderer::new / with_device (src/renderer/renderer.rs:25-36) on a CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self._children = weakref.WeakSet()  # scenes and batches: destroyed before the context
        self.ctx = C.c_void_p()
        _check(self.lib.dvg_context_create(int(device), C.byref(self.ctx)))
        self.device = device

    def close(self) -> None:
        if self.ctx:
            for child in sorted(list(self._children), key=lambda c: 0 if isinstance(c, Batch) else 1):
                child.close()
            self.lib.dvg_context_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launch_count(self) -> int:
        return int(self.lib.dvg_context_launch_count(self.ctx))

    @property
    def stream_handle(self) -> int:
        return int(self.lib.dvg_context_stream(self.ctx) or 0)

    def l2_device(self, image_ptr: int, target_ptr: int, n: int, d_render_ptr: int, loss_ptr: int = 0) -> None:
        """dvg_l2_device: loss = sum((image - target)^2), d_render = 2 (image - target)."""
        _check(self.lib.dvg_l2_device(self.ctx, C.c_void_p(image_ptr), C.c_void_p(target_ptr), int(n),
                                      C.c_void_p(d_render_ptr), C.c_void_p(loss_ptr) if loss_ptr else None))

    def set_retain(self, enable: bool) -> None:
        """dvg_context_set_retain: keep the last render for a following render_backward."""
        _check(self.lib.dvg_context_set_retain(self.ctx, 1 if enable else 0))

    def set_profiling(self, enable: bool) -> None:
        _check(self.lib.dvg_context_set_profiling(self.ctx, 1 if enable else 0))

    def profile(self, reset: bool = True) -> dict:
        """{launcher name: (total ms, calls)} from the context's CUDA-event timing."""
        cap = 64
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        calls = (C.c_uint64 * cap)()
        n = self.lib.dvg_context_profile(self.ctx, names, ms, calls, cap)
        out = {names[i].decode(): (float(ms[i]), int(calls[i])) for i in range(min(n, cap))}
        if reset:
            self.lib.dvg_context_profile_reset(self.ctx)
        return out

    def upload(self, scene: Scene, packed: Optional[PackedScene] = None) -> UploadedScene:
        """dvg_scene_upload.  `packed`: a pack_scene(scene) result to upload instead of
        packing again (e.g. after editing its arrays in place)."""
        return UploadedScene(self, scene, packed)

    PINNED_IMAGE_BYTES = 256 << 20

    def _host_image(self, shape) -> np.ndarray:
        """An uninitialised float32 host array, page-locked up to PINNED_IMAGE_BYTES
        (torch's caching host allocator: a freed image's block is reused by the next
        one), so that the device-to-host copy of the image runs at DMA speed instead of
        through the driver's staging buffer; larger images use ordinary memory."""
        if int(np.prod(shape)) * 4 > self.PINNED_IMAGE_BYTES:
            return np.empty(shape, np.float32)
        import torch

        return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()

    def render(self, scene: Scene, options: RenderOptions = None, packed: Optional[PackedScene] = None) -> Image:
        """Renderer::render (src/renderer/renderer.rs:39-545).  `packed`: pack_scene(scene)
        made by the caller (one packing for a render and the render_backward after it)."""
        options = options or RenderOptions()
        if scene.background_image is not None:
            if np.asarray(scene.background_image).size != scene.width * scene.height * 4:
                raise RenderError(DVG_ERR_INVALID_SCENE, "background image size mismatch")
        if scene.width == 0 or scene.height == 0:
            return Image(scene.width, scene.height, np.zeros((0,), np.float32))
        packed = packed or pack_scene(scene)
        out = self._host_image((scene.height, scene.width, 4))
        o = render_options_c(options)
        _check(self.lib.dvg_render(self.ctx, packed.ref(), C.byref(o), _fp(out)))
        return Image(scene.width, scene.height, out)

    def render_backward(self, scene: Scene, options: RenderOptions = None,
                        backward_options: Optional[BackwardOptions] = None,
                        d_render_image: Optional[np.ndarray] = None, d_sdf_image: Optional[np.ndarray] = None,
                        packed: Optional[PackedScene] = None):
        """Renderer::render_backward (src/renderer/renderer.rs:548-564) -> SceneGrad."""
        options = options or RenderOptions()
        bopts = backward_options or BackwardOptions()
        npix = scene.width * scene.height
        if d_render_image is not None and np.asarray(d_render_image).size != npix * 4:
            raise RenderError(DVG_ERR_INVALID_SCENE, "d_render_image size mismatch")
        if d_sdf_image is not None and np.asarray(d_sdf_image).size != npix:
            raise RenderError(DVG_ERR_INVALID_SCENE, "d_sdf_image size mismatch")
        packed = packed or pack_scene(scene)
        has_bg = d_render_image is not None and scene.background_image is not None
        buf = GradBuffers(packed, background_image=has_bg, translation=bopts.compute_translation)
        dr = None if d_render_image is None else np.ascontiguousarray(np.asarray(d_render_image, np.float32).reshape(-1))
        ds = None if d_sdf_image is None else np.ascontiguousarray(np.asarray(d_sdf_image, np.float32).reshape(-1))
        o = render_options_c(options)
        b = backward_options_c(bopts)
        _check(self.lib.dvg_render_backward(self.ctx, packed.ref(), C.byref(o), C.byref(b), _fp(dr), _fp(ds),
                                            C.byref(buf.c)))
        return unflatten_grads(scene, packed, buf)


    def lbvh_build(self, boxes):
        """dvg_lbvh_build on [n, 4] boxes: (sorted keys [n], children [n-1, 2], bounds [2n-1, 4])."""
        b = np.ascontiguousarray(np.asarray(boxes, np.float32).reshape(-1, 4))
        n = b.shape[0]
        keys = np.zeros(n, np.uint64)
        ch = np.zeros((max(n - 1, 0), 2), np.int32)
        bounds = np.zeros((max(2 * n - 1, 0), 4), np.float32)
        _check(self.lib.dvg_lbvh_build(self.ctx, _fp(b), n, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                       ch.ctypes.data_as(C.POINTER(C.c_int32)), _fp(bounds)))
        return keys, ch, bounds

    def render_sdf(self, scene: Scene, options: RenderOptions = None) -> SdfImage:
        """Renderer::render_sdf (src/renderer/renderer.rs:586-716)."""
        options = options or RenderOptions()
        out = np.zeros((scene.height, scene.width), np.float32)
        if scene.width == 0 or scene.height == 0:
            return SdfImage(scene.width, scene.height, out.reshape(-1))
        packed = pack_scene(scene)
        o = render_options_c(options)
        _check(self.lib.dvg_render_sdf(self.ctx, packed.ref(), C.byref(o), _fp(out)))
        return SdfImage(scene.width, scene.height, out)

    def eval_positions(self, scene: Scene, positions, options: RenderOptions = None) -> np.ndarray:
        """Renderer::eval_positions (src/renderer/renderer.rs:719-848): signed distances at [n, 2] points."""
        pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1))
        out = np.zeros(pos.size // 2, np.float32)
        if out.size == 0:
            return out
        packed = pack_scene(scene)
        _check(self.lib.dvg_eval_positions(self.ctx, packed.ref(), _fp(pos), out.size, _fp(out)))
        return out

    def eval_positions_backward(self, scene: Scene, positions, options: RenderOptions = None,
                                backward_options: Optional[BackwardOptions] = None, d_sdf_values=None):
        """Renderer::eval_positions_backward (src/renderer/renderer.rs:567-583) -> SceneGrad."""
        bopts = backward_options or BackwardOptions()
        pos = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1))
        n = pos.size // 2
        if d_sdf_values is not None and np.asarray(d_sdf_values).size != n:
            raise RenderError(DVG_ERR_INVALID_SCENE, "d_sdf_image size mismatch for eval_positions")
        packed = pack_scene(scene)
        buf = GradBuffers(packed, background_image=False, translation=bopts.compute_translation)
        if d_sdf_values is not None and n:
            d = np.ascontiguousarray(np.asarray(d_sdf_values, np.float32).reshape(-1))
            b = backward_options_c(bopts)
            _check(self.lib.dvg_eval_positions_backward(self.ctx, packed.ref(), C.byref(b), _fp(pos), n, _fp(d),
                                                        C.byref(buf.c)))
        return unflatten_grads(scene, packed, buf)


def device_view(ptr: int, count: int, device=None):
    """A float32 torch tensor aliasing `count` floats of device memory at `ptr`."""
    import torch

    class _Iface:
        __cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f4", "data": (int(ptr), False),
                                    "version": 3, "strides": None}

    return torch.as_tensor(_Iface(), device=device or "cuda")


class Batch:
    """dvg_batch: many uploaded scenes stepped together (one launch per stage, CUDA graph)."""

    def __init__(self, renderer: "Renderer", scenes, options: RenderOptions,
                 backward_options: Optional[BackwardOptions] = None):
        self.renderer = renderer
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[u.handle.value for u in self.scenes])
        o = render_options_c(options)
        b = backward_options_c(backward_options)
        self.handle = C.c_void_p()
        _check(renderer.lib.dvg_batch_create(renderer.ctx, arr, len(self.scenes), C.byref(o), C.byref(b),
                                             C.byref(self.handle)))
        renderer._children.add(self)

    def buffers(self, index: int):
        """(image tensor, target tensor, GradsC) aliasing the batch's device buffers of scene `index`."""
        img = C.c_void_p()
        tgt = C.c_void_p()
        g = GradsC()
        _check(self.renderer.lib.dvg_batch_buffers(self.handle, index, C.byref(img), C.byref(tgt), C.byref(g)))
        sc = self.scenes[index].scene
        n = sc.width * sc.height * 4
        return device_view(img.value, n), device_view(tgt.value, n), g

    def step(self, use_graph: bool = True) -> None:
        _check(self.renderer.lib.dvg_batch_step(self.handle, 1 if use_graph else 0))

    def losses(self) -> np.ndarray:
        out = np.zeros(len(self.scenes), np.float32)
        _check(self.renderer.lib.dvg_batch_losses(self.handle, _fp(out)))
        return out

    def autotune(self):
        """dvg_batch_autotune: returns the chosen (sample_layout, boundary_cell, fragment_slots, work_queue,
        forward_occupancy)."""
        t = TuningC()
        _check(self.renderer.lib.dvg_batch_autotune(self.handle, C.byref(t)))
        return _tuple(t)

    def set_tuning(self, sample_layout: int, boundary_cell: int, fragment_slots: int = 16, work_queue: int = 0,
                   forward_occupancy: int = 0) -> None:
        t = TuningC(sample_layout, boundary_cell, fragment_slots, work_queue, forward_occupancy)
        _check(self.renderer.lib.dvg_batch_set_tuning(self.handle, C.byref(t)))

    def set_adam(self, lr: float = 1e-2, betas=(0.9, 0.999), eps: float = 1e-8, points: bool = True,
                 paints: bool = False) -> None:
        """Adds Adam + on-device scene re-preparation to every step (dvg_batch_set_adam);
        lr=None clears it."""
        if lr is None:
            _check(self.renderer.lib.dvg_batch_set_adam(self.handle, None))
            return
        o = AdamOptionsC(lr, betas[0], betas[1], eps, (OPT_POINTS if points else 0) | (OPT_PAINTS if paints else 0))
        _check(self.renderer.lib.dvg_batch_set_adam(self.handle, C.byref(o)))

    def scene_params(self, index: int):
        """(points [total_points, 2], paint params [num_paints, 4]) of scene `index` as stepped so far."""
        d = self.scenes[index].packed.desc
        pts = np.zeros(2 * d.total_points, np.float32)
        pp = np.zeros(4 * d.num_paints, np.float32)
        _check(self.renderer.lib.dvg_batch_scene_params(self.handle, index, _fp(pts), _fp(pp)))
        return pts.reshape(-1, 2), pp.reshape(-1, 4)

    def close(self) -> None:
        if self.handle and self.renderer.ctx:
            self.renderer.lib.dvg_batch_destroy(self.handle)
        self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
