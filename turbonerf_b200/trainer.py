"""Python surface of the training controller, named like the reference's `PyTurboNeRF`
module (src/api/python_bindings.cu:240-255, 423-491): `BoundingBox`, `Trainer` with
`setup_data(batch_size)`, `train_step()`, `update_occupancy_grid(training_step)`,
`teardown()`, the `TrainingMetrics` / `OccupancyGridMetrics` results and the
`min_step_size` / `use_distortion_loss` / alpha-selection attributes.

The controller itself is C++ inside libturbo_hot.so (tn_trainer_*); this module only
marshals arguments. The reference's `Trainer(nerf)` takes a NeRF proxy holding a dataset
and a tiny-cuda-nn network; here `Trainer(scene)` takes a `SyntheticNeRF` (occupancy grid,
bounding box and the synthetic blob field that stands in for the network).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import native
from .native import Bbox, GridDesc, OccupancyMetricsC, TrainerDesc, TrainingMetricsC, TuneReport, Tuning, call

MIN_STEP_SIZE = 0.00169145586  # NeRFConstants::min_step_size
CONE_ANGLE = 1.0 / 256.0       # NeRFConstants::cone_angle


class BoundingBox:
    """Axis-aligned box, reference BoundingBox (src/models/bounding-box.cuh:8-23)."""

    def __init__(self, size: float | None = None):
        if size is None:
            self.min_x = self.min_y = self.min_z = self.max_x = self.max_y = self.max_z = 0.0
        else:
            h = 0.5 * float(size)
            self.min_x = self.min_y = self.min_z = -h
            self.max_x = self.max_y = self.max_z = h

    def size(self) -> float:
        return self.max_x - self.min_x

    def as_tuple(self):
        return (self.min_x, self.min_y, self.min_z, self.max_x, self.max_y, self.max_z)

    def __eq__(self, other):
        return isinstance(other, BoundingBox) and self.as_tuple() == other.as_tuple()

    def __ne__(self, other):
        return not self == other


@dataclass
class TrainingMetrics:
    step: int
    loss: float
    n_rays: int
    n_samples: int


@dataclass
class OccupancyGridMetrics:
    n_occupied: int
    n_total: int


class Dataset:
    """Posed images to train on (the reference's Dataset, src/models/dataset.h, loaded here from
    arrays instead of a transforms.json): `cameras`, one renderer.Camera per image, all of the
    images' resolution, and `images`, uint8 RGBA [n_images][height][width][4]."""

    def __init__(self, cameras, images):
        self.cameras = list(cameras)
        self.images = np.ascontiguousarray(images, dtype=np.uint8)
        if self.images.ndim != 4 or self.images.shape[3] != 4:
            raise ValueError("images must be [n_images][height][width][4] RGBA8")
        if len(self.cameras) != self.images.shape[0]:
            raise ValueError("one camera per image")
        h, w = self.images.shape[1:3]
        if any(c.resolution != (w, h) for c in self.cameras):
            raise ValueError("every camera must have the images' resolution")


@dataclass
class SyntheticNeRF:
    """What the trainer trains on: the cascaded occupancy grid (base size 1 = the reference's
    2^k level extents), the training box, and the blob field standing in for the network."""
    bounding_box: BoundingBox
    n_levels: int
    blobs: np.ndarray
    waves: np.ndarray
    density: np.ndarray | None = None   # [n_levels][res^3] float32 (None: zeros, like the reference)
    bitfield: np.ndarray | None = None  # [res^3] uint8 (None: all bits set, like the reference)
    resolution: int = 128
    base_size: float = 1.0
    render_bbox: BoundingBox | None = None  # renderer crop (reference NeRFProxy::render_bbox); None: bounding_box
    dataset: Dataset | None = None  # posed images to train on; None: the built-in synthetic rays

    @classmethod
    def from_scene(cls, scene) -> "SyntheticNeRF":
        b = BoundingBox()
        b.min_x, b.min_y, b.min_z, b.max_x, b.max_y, b.max_z = [float(v) for v in scene.bbox]
        g = scene.grid
        return cls(b, g.n_levels, scene.field.blobs, scene.field.waves, g.density, g.bitfield, g.resolution,
                   g.base_size)


class Trainer:
    """Training controller (reference NeRFTrainingController)."""

    def __init__(self, nerf: SyntheticNeRF, path: str = "fused", use_cuda_graph: bool = True,
                 n_rays_per_step: int = 1 << 14, occupancy_cells_per_step: int = 0,
                 distortion_lambda: float = 0.01, occupancy_threshold: float = 0.01 * MIN_STEP_SIZE,
                 n_grid_params: int = 16 * (1 << 19) * 2, n_mlp_params: int = 7168, beta2: float = 0.999,
                 max_steps_per_ray: int = 0, seed: int = 0x7B0, min_transmittance: float = 1e-4):
        if path not in ("fused", "plain"):
            raise ValueError("path must be 'fused' or 'plain'")
        self.nerf = nerf
        self.path = path
        self.use_cuda_graph = use_cuda_graph
        self.n_rays_per_step = n_rays_per_step
        self.occupancy_cells_per_step = occupancy_cells_per_step
        self.distortion_lambda = distortion_lambda
        self.occupancy_threshold = occupancy_threshold
        self.n_grid_params = n_grid_params
        self.n_mlp_params = n_mlp_params
        self.beta2 = beta2
        self.max_steps_per_ray = max_steps_per_ray
        self.seed = seed
        self.min_transmittance = min_transmittance  # NeRFConstants::min_transmittance
        # reference training settings (nerf-training-controller.h:75-78)
        self.alpha_selection_threshold = 1.0
        self.alpha_selection_probability = 1.0
        self.min_step_size = MIN_STEP_SIZE
        self.use_distortion_loss = False
        self._h = None
        self.n_touched_grads = 0

    # -- lifecycle -----------------------------------------------------------------------
    def setup_data(self, batch_size: int = 2 << 21, synthetic_grad_std: float = 1e-3) -> None:
        """Allocates every buffer, uploads the grid and the synthetic field, and seeds the
        parameter gradients (reference setup_data, nerf-training-controller.cu:27-85)."""
        if (self.alpha_selection_threshold < 1.0 and self.alpha_selection_probability < 1.0
                and self.nerf.dataset is None):
            raise NotImplementedError("alpha selection acts on image alpha; the synthetic ray source has none")
        self.teardown()
        d = TrainerDesc()
        call("tn_trainer_default_desc", ctypes.byref(d))
        n = self.nerf
        d.grid = GridDesc(n.n_levels, n.resolution, float(n.base_size), 0)
        d.bbox = Bbox(*n.bounding_box.as_tuple())
        d.batch_size = int(batch_size)
        d.n_rays_per_step = int(self.n_rays_per_step)
        d.min_step_size = float(self.min_step_size)
        d.max_steps_per_ray = int(self.max_steps_per_ray)
        d.min_transmittance = float(self.min_transmittance)
        d.use_distortion_loss = int(bool(self.use_distortion_loss))
        d.distortion_lambda = float(self.distortion_lambda)
        d.occupancy_threshold = float(self.occupancy_threshold)
        d.occupancy_cells_per_step = int(self.occupancy_cells_per_step)
        d.n_grid_params = int(self.n_grid_params)
        d.n_mlp_params = int(self.n_mlp_params)
        d.beta2 = float(self.beta2)
        d.path = native.TN_PATH_FUSED if self.path == "fused" else native.TN_PATH_PLAIN
        d.use_cuda_graph = int(bool(self.use_cuda_graph))
        d.seed = int(self.seed)
        h = ctypes.c_void_p()
        call("tn_trainer_create", ctypes.byref(h), ctypes.byref(d), None)
        self._h = h
        self._alpha_applied = None
        blobs = np.ascontiguousarray(n.blobs, np.float32)
        waves = np.ascontiguousarray(n.waves, np.float32)
        call("tn_trainer_set_synthetic_field", h, blobs.shape[0], blobs.ctypes.data_as(ctypes.c_void_p),
             waves.ctypes.data_as(ctypes.c_void_p))
        self._upload_grid()
        if n.dataset is not None:
            cams = (native.CameraC * len(n.dataset.cameras))(*[c.c_struct() for c in n.dataset.cameras])
            im = n.dataset.images
            call("tn_trainer_set_dataset", h, im.shape[0], im.shape[2], im.shape[1], cams,
                 im.ctypes.data_as(ctypes.c_void_p))
            self._apply_alpha_selection()
        touched = ctypes.c_uint32(0)
        call("tn_trainer_init_synthetic_gradients", h, float(synthetic_grad_std), ctypes.byref(touched))
        self.n_touched_grads = touched.value

    def use_hashgrid(self, spec=None) -> None:
        """Trains the multiresolution hash encoding with linear density and colour heads as the
        network (in place of the synthetic producer): real parameter gradients each step, the
        hash entries a step touches listed (trainer buffers 31 and 32). The trainer's grid section
        must hold the encoding's entries exactly (n_grid_params = 2 n_levels 2^log2_hashmap_size)
        and its MLP section the heads. spec: a hotpath.HashgridSpec (default: the reference's
        encoding for this NeRF's box size)."""
        from .hotpath import HashgridSpec
        if spec is None:
            spec = HashgridSpec.reference(self.nerf.bounding_box.size())
        call("tn_trainer_use_hashgrid", self._handle(), ctypes.byref(spec.desc()))
        self.hashgrid = spec

    def _upload_grid(self) -> None:
        """The NeRF's initial occupancy grid (densities and/or bitfield), when it has one."""
        n = self.nerf
        dens = None if n.density is None else np.ascontiguousarray(n.density, np.float32)
        bits = None if n.bitfield is None else np.ascontiguousarray(n.bitfield, np.uint8)
        call("tn_trainer_set_grid", self._handle(), dens.ctypes.data_as(ctypes.c_void_p) if dens is not None else None,
             bits.ctypes.data_as(ctypes.c_void_p) if bits is not None else None)

    def reset_training(self) -> None:
        """Clears the training data and starts over (reference reset_training,
        nerf-training-controller.cu:108-120, which frees the training buffers and runs
        setup_data again): parameters re-drawn from the seed, Adam moments and per-parameter
        steps zero, the step counter zero, the occupancy grid re-initialised and the NeRF's
        initial grid uploaded again, as setup_data does. Buffers and launch shapes are kept."""
        call("tn_trainer_reset", self._handle())
        self._upload_grid()

    def teardown(self) -> None:
        if self._h is not None:
            native.lib().tn_trainer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.teardown()
        except Exception:
            pass

    def _handle(self):
        if self._h is None:
            raise RuntimeError("call setup_data() first")
        return self._h

    def _apply_alpha_selection(self) -> None:
        """Hands the alpha-selection attributes to the controller when they changed (they act on
        dataset rays; the reference reads them on every step)."""
        cur = (float(self.alpha_selection_threshold), float(self.alpha_selection_probability))
        if self._h is not None and getattr(self, "_alpha_applied", None) != cur:
            if cur[0] < 1.0 and cur[1] < 1.0 and self.nerf.dataset is None:
                raise NotImplementedError("alpha selection acts on image alpha; the synthetic ray source has none")
            call("tn_trainer_set_alpha_selection", self._h, cur[0], cur[1])
            self._alpha_applied = cur

    # -- steps ---------------------------------------------------------------------------
    def train_step(self) -> TrainingMetrics:
        self._apply_alpha_selection()
        m = TrainingMetricsC()
        call("tn_trainer_train_step", self._handle(), ctypes.byref(m))
        return TrainingMetrics(m.step, m.loss, m.n_rays, m.n_samples)

    def train_step_async(self) -> None:
        """Enqueues one step without waiting (fused path: a graph replay)."""
        self._apply_alpha_selection()
        call("tn_trainer_train_step", self._handle(), None)

    def train_step_rays(self, ori, dir_, target_rgba, bg_rgb) -> TrainingMetrics:
        """One step on caller rays held in (preferably pinned) host memory, each
        [components][n_rays_per_step] float32; waits and returns the metrics."""
        m = TrainingMetricsC()
        arrs = [self._host_ptr(a) for a in (ori, dir_, target_rgba, bg_rgb)]
        call("tn_trainer_train_step_rays", self._handle(), self.n_rays_per_step, *arrs, ctypes.byref(m))
        return TrainingMetrics(m.step, m.loss, m.n_rays, m.n_samples)

    def train_step_rays_pipelined(self, ori, dir_, target_rgba, bg_rgb) -> TrainingMetrics | None:
        """The same step as train_step_rays for a loop that feeds rays from the host: enqueues
        this step and returns the metrics of the previous pipelined step (None on the first
        call), waiting for that step only. The host arrays must stay unchanged until the next
        call returns; sync_metrics() returns the last step's metrics."""
        m = TrainingMetricsC()
        arrs = [self._host_ptr(a) for a in (ori, dir_, target_rgba, bg_rgb)]
        call("tn_trainer_train_step_rays_pipelined", self._handle(), self.n_rays_per_step, *arrs, ctypes.byref(m))
        return None if m.step == 0 else TrainingMetrics(m.step, m.loss, m.n_rays, m.n_samples)

    @staticmethod
    def _host_ptr(a):
        try:
            import torch
            if isinstance(a, torch.Tensor):
                if a.is_cuda or not a.is_contiguous() or a.dtype != torch.float32:
                    raise ValueError("host rays must be contiguous float32 CPU tensors")
                return ctypes.c_void_p(a.data_ptr())
        except ImportError:
            pass
        a = np.ascontiguousarray(a, np.float32)
        return a.ctypes.data_as(ctypes.c_void_p)

    def sync_metrics(self) -> TrainingMetrics:
        m = TrainingMetricsC()
        call("tn_trainer_sync_metrics", self._handle(), ctypes.byref(m))
        return TrainingMetrics(m.step, m.loss, m.n_rays, m.n_samples)

    def update_occupancy_grid(self, training_step: int) -> OccupancyGridMetrics:
        m = OccupancyMetricsC()
        call("tn_trainer_update_occupancy_grid", self._handle(), int(training_step), ctypes.byref(m))
        return OccupancyGridMetrics(m.n_occupied, m.n_total)

    # -- launch shapes -------------------------------------------------------------------
    def autotune(self) -> dict:
        """Tunes the march (count block size, emit shape) and the fused loss kernel's block size
        on this trainer's batch; weights, optimizer state and the grid are left as they are.
        Returns the reports of the three tuners and the chosen shapes."""
        reps = (TuneReport * 3)()
        call("tn_trainer_autotune", self._handle(), reps)
        return {"count": reps[0].as_dict(), "emit": reps[1].as_dict(), "losses": reps[2].as_dict(),
                "tuning": self.tuning}

    def flush(self) -> None:
        """Completes a requested caller-ray step (the pipelined call leaves the last step's tail
        to run beside the next call's march) and waits for the trainer's stream."""
        call("tn_trainer_flush", self._handle())

    @property
    def tuning(self) -> dict:
        t = Tuning()
        call("tn_trainer_get_tuning", self._handle(), ctypes.byref(t))
        return t.as_dict()

    @tuning.setter
    def tuning(self, values: dict) -> None:
        t = Tuning()
        call("tn_trainer_get_tuning", self._handle(), ctypes.byref(t))
        for k, v in values.items():
            setattr(t, k, int(v))
        call("tn_trainer_set_tuning", self._handle(), ctypes.byref(t))

    # -- introspection -------------------------------------------------------------------
    def profile_step(self) -> list[float]:
        out = (ctypes.c_float * 16)()
        n = ctypes.c_uint32(0)
        call("tn_trainer_profile_step", self._handle(), out, 16, ctypes.byref(n))
        return [out[i] for i in range(n.value)]

    def stat(self, which: int) -> int:
        v = ctypes.c_uint64(0)
        call("tn_trainer_stat", self._handle(), which, ctypes.byref(v))
        return v.value

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        call("tn_trainer_stream", self._handle(), ctypes.byref(s))
        return s.value or 0

    def buffer(self, which: int, dtype=np.float32, count: int | None = None):
        """A device buffer of the trainer as a torch tensor view (no copy)."""
        import torch
        p = ctypes.c_void_p()
        nbytes = ctypes.c_uint64(0)
        call("tn_trainer_buffer", self._handle(), which, ctypes.byref(p), ctypes.byref(nbytes))
        itemsize = np.dtype(dtype).itemsize
        n = count if count is not None else nbytes.value // itemsize

        class _View:
            __cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str, "data": (p.value, False),
                                        "version": 3}

        return torch.as_tensor(_View(), device="cuda")


class FileManager:
    """`.turbo` snapshots, named like the reference's `FileManager` (python_bindings.cu:647-662,
    src/services/file-manager.cuh:34-198). The reference saves a NeRF proxy; here the trained
    state lives in the `Trainer`, so that is what `save` and `load` take. The file holds the
    reference's header, fp32 parameters ([hash grid | MLP]) and occupancy bitfield, then a resume
    block (Adam moments and step counts, grid densities, step counters) that the reference's
    loader does not read. `load` needs a trainer set up with the same parameter counts, grid and
    box; after it, training continues from the saved step exactly."""

    @staticmethod
    def save(trainer: Trainer, path: str, dataset_path: str | None = None) -> None:
        if dataset_path is None:
            dataset_path = getattr(trainer.nerf.dataset, "file_path", None) or ""
        call("tn_trainer_save", trainer._handle(), str(path).encode(), str(dataset_path).encode())

    @staticmethod
    def load(trainer: Trainer, path: str) -> None:
        call("tn_trainer_load", trainer._handle(), str(path).encode())

    @staticmethod
    def info(path: str) -> dict:
        """The header and resume block of a .turbo file (no GPU work)."""
        i = native.TurboInfoC()
        call("tn_turbo_file_info", str(path).encode(), ctypes.byref(i))
        return {"n_params": i.n_params, "file_bytes": i.file_bytes, "n_occ_grid_bits": i.n_occ_grid_bits,
                "aabb_scale": i.aabb_scale, "has_resume": bool(i.has_resume), "step_count": i.step_count,
                "n_levels": i.n_levels, "resolution": i.resolution, "dataset_path": i.dataset_path.decode()}
