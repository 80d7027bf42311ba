"""Python surface of the rendering controller, named like the reference's `PyTurboNeRF`
module (src/api/python_bindings.cu:174-200, 305-419): `Camera`, `RenderPattern`,
`RenderFlags`, `RenderTarget` with `CPURenderBuffer` / `CUDARenderBuffer`, `RenderRequest` and
`Renderer(pattern, batch_size).submit(request)` with its `min_step_size` attribute.

The render itself is C++/CUDA inside libturbo_hot.so (tn_trainer_render -> tn_render); this
module only marshals arguments. Differences from the reference, by design of this library:
  * a request renders one NeRF, given as the `Trainer` whose device state holds it (grid,
    training box, network), with an identity transform;
  * lens distortion, spatial effects and the near/far plane overlays are not supported;
  * the render pattern only decides how the reference tiles the image for progressive display;
    the image does not depend on it, and the whole image is rendered in one submit;
  * render targets are headless: a host array (`CPURenderBuffer`) or a torch CUDA tensor
    (`CUDARenderBuffer`); `save_image` writes an 8-bit PNG.
"""
from __future__ import annotations

import ctypes
import enum
import struct
import zlib

import numpy as np

from .native import Bbox, CameraC, RenderStatsC, call

MIN_STEP_SIZE = 0.00169145586  # NeRFConstants::min_step_size


class RenderPattern(enum.IntEnum):
    """reference RenderPattern (src/models/render-pattern.cuh:6-10)"""
    LinearChunks = 0
    HexagonalGrid = 1
    RectangularGrid = 2


class RenderFlags(enum.IntFlag):
    """reference RenderFlags (src/utils/render-flags.cuh:7-10)"""
    Preview = 1 << 0
    Final = 1 << 1


class Camera:
    """Pinhole camera (reference Camera, src/models/camera.cuh:34-80): resolution (w, h),
    near / far distances, focal_length (fx, fy) and principal_point (cx, cy) in pixels, shift
    (fraction of the resolution) and transform (camera to world, 4 x 4 or 3 x 4)."""

    def __init__(self, resolution, near, far, focal_length, principal_point, shift, transform, dist_params=None):
        if dist_params is not None and any(float(v) != 0.0 for v in _dist_values(dist_params)):
            raise NotImplementedError("lens distortion is not supported by this renderer")
        self.resolution = (int(resolution[0]), int(resolution[1]))
        self.near = float(near)
        self.far = float(far)
        self.focal_length = (float(focal_length[0]), float(focal_length[1]))
        self.principal_point = (float(principal_point[0]), float(principal_point[1]))
        self.shift = (float(shift[0]), float(shift[1]))
        t = np.asarray(transform, np.float32)
        if t.shape not in ((4, 4), (3, 4)):
            raise ValueError("transform must be 4 x 4 or 3 x 4")
        self.transform = np.ascontiguousarray(t[:3, :4])

    def c_struct(self) -> CameraC:
        c = CameraC()
        c.width, c.height = self.resolution
        c.near, c.far = self.near, self.far
        c.focal_x, c.focal_y = self.focal_length
        c.principal_x, c.principal_y = self.principal_point
        c.shift_x, c.shift_y = self.shift
        for k, v in enumerate(self.transform.reshape(-1)):
            c.transform[k] = float(v)
        return c


def _dist_values(p):
    if isinstance(p, dict):
        return p.values()
    return [getattr(p, k, 0.0) for k in ("k1", "k2", "k3", "p1", "p2")]


class RenderTarget:
    """A render target of width x height pixels holding premultiplied RGBA floats."""

    def __init__(self):
        self.width = 0
        self.height = 0

    def set_size(self, width: int, height: int) -> None:
        self.width, self.height = int(width), int(height)

    def free(self) -> None:
        self.width = self.height = 0

    def _device_buffer(self):
        raise NotImplementedError

    def _finish(self, dev) -> None:
        raise NotImplementedError

    def get_rgba(self) -> np.ndarray:
        raise NotImplementedError

    def save_image(self, file_path: str) -> None:
        """8-bit RGBA PNG of the image, row 0 at the top."""
        rgba = np.clip(self.get_rgba(), 0.0, 1.0)
        img = (rgba * 255.0 + 0.5).astype(np.uint8)
        h, w = img.shape[:2]
        raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))

        def chunk(tag, data):
            return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

        png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
               chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
        with open(file_path, "wb") as f:
            f.write(png)


class CUDARenderBuffer(RenderTarget):
    """Device render target: `rgba` is a torch float32 CUDA tensor [height, width, 4]."""

    def __init__(self):
        super().__init__()
        self.rgba = None

    def set_size(self, width: int, height: int) -> None:
        super().set_size(width, height)
        self.rgba = None

    def free(self) -> None:
        super().free()
        self.rgba = None

    def _device_buffer(self):
        import torch
        if self.rgba is None or tuple(self.rgba.shape) != (self.height, self.width, 4):
            self.rgba = torch.empty((self.height, self.width, 4), dtype=torch.float32, device="cuda")
        return self.rgba

    def _finish(self, dev) -> None:
        pass

    def get_rgba(self) -> np.ndarray:
        if self.rgba is None:
            raise RuntimeError("nothing rendered into this buffer yet")
        return self.rgba.cpu().numpy()


class CPURenderBuffer(RenderTarget):
    """Host render target; get_rgba() returns a float32 array [height, width, 4]."""

    def __init__(self):
        super().__init__()
        self._rgba = None
        self._dev = None

    def free(self) -> None:
        super().free()
        self._rgba = None
        self._dev = None

    def _device_buffer(self):
        import torch
        if self._dev is None or tuple(self._dev.shape) != (self.height, self.width, 4):
            self._dev = torch.empty((self.height, self.width, 4), dtype=torch.float32, device="cuda")
        return self._dev

    def _finish(self, dev) -> None:
        self._rgba = dev.cpu().numpy()

    def get_rgba(self) -> np.ndarray:
        if self._rgba is None:
            raise RuntimeError("nothing rendered into this buffer yet")
        return self._rgba


class RenderModifiers:
    """reference RenderModifiers (its near/far plane overlays are not drawn here)."""

    def __init__(self):
        self.properties = None


class RenderRequest:
    """What to render: `camera`, `nerfs` (one Trainer after setup_data, whose device state
    holds the NeRF), `output` (a RenderTarget; resized to the camera's resolution), and the
    reference's flags and callbacks. A submit renders the whole image synchronously, so
    on_progress(1.0) and on_complete() are called once at its end; flags (preview or final)
    do not change the image, and on_cancel() is never called (there is nothing to cancel)."""

    def __init__(self, camera: Camera, nerfs, output: RenderTarget, modifiers: RenderModifiers | None = None,
                 flags: RenderFlags = RenderFlags.Final, on_complete=None, on_progress=None, on_cancel=None):
        self.camera = camera
        self.nerfs = list(nerfs)
        self.output = output
        self.modifiers = modifiers or RenderModifiers()
        self.flags = flags
        self.on_complete = on_complete
        self.on_progress = on_progress
        self.on_cancel = on_cancel
        self.stats: dict | None = None


class Renderer:
    """Rendering controller (reference NeRFRenderingController, src/controllers/
    nerf-rendering-controller.cu:16-80). batch_size is the sample budget of one round (the
    reference's 1 << 20 when asked for); 0 lets the library pick 8 samples per pixel within
    [2^20, 2^25]. The image does not depend on it."""

    def __init__(self, pattern: RenderPattern = RenderPattern.LinearChunks, batch_size: int = 0):
        self.pattern = RenderPattern(pattern)
        self.batch_size = int(batch_size)  # 0: the library picks the budget from the image size
        self.min_step_size = MIN_STEP_SIZE

    def submit(self, request: RenderRequest) -> dict:
        """Renders the request synchronously into request.output; returns (and stores in
        request.stats) the render statistics."""
        if len(request.nerfs) == 0:
            if request.on_complete:
                request.on_complete()
            return {}
        if len(request.nerfs) != 1:
            raise NotImplementedError("this renderer composites one NeRF per request")
        trainer = request.nerfs[0]
        cam = request.camera
        out = request.output
        if (out.width, out.height) != cam.resolution:
            out.set_size(*cam.resolution)
        dev = out._device_buffer()
        c = cam.c_struct()
        stats = RenderStatsC()
        crop = getattr(trainer.nerf, "render_bbox", None)
        crop = ctypes.byref(Bbox(*crop.as_tuple())) if crop is not None else None
        call("tn_trainer_render", trainer._handle(), ctypes.byref(c), crop, float(self.min_step_size),
             int(self.batch_size), ctypes.c_void_p(dev.data_ptr()), ctypes.byref(stats))
        out._finish(dev)
        request.stats = {"rays_hit": int(stats.rays_hit), "iterations": int(stats.iterations),
                         "samples": int(stats.samples), "steps": int(stats.steps), "tests": int(stats.tests)}
        if request.on_progress:
            request.on_progress(1.0)
        if request.on_complete:
            request.on_complete()
        return request.stats
