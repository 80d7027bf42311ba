"""Seeded synthetic scenes and batches for TurboNeRF's training hot path.

The reference trains on photographs (a Lego scene fetched from the network); none is
available here, so every workload is synthetic and seeded:

* a density field made of isotropic Gaussian blobs, with colour = sigmoid of three
  fixed random sinusoids of the world position (the stand-in for the tiny-cuda-nn
  network that produces sigma/rgb upstream of the hot path);
* occupancy bitfields built by thresholding that field at cell centres;
* ray batches with origins on a sphere looking at the scene centre;
* packed per-sample batches for the compositor and distortion loss, with the
  per-ray sample counts of a truncated geometric distribution.

All arrays use the reference's structure-of-arrays layout (component c of item i at
buf[c * stride + i], src/workspaces/training-workspace.cuh:87-112 in the reference).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SEED = 0x7B0
MIN_STEP_SIZE = np.float32(0.00169145586)  # sqrt(3)/1024, src/utils/nerf-constants.cuh:7


# ---------------------------------------------------------------------------------------
# Morton helpers (vectorised; x -> bit 0, y -> bit 1, z -> bit 2 of each 3-bit group)
# ---------------------------------------------------------------------------------------
def _part1by2(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32) & np.uint32(0x3FF)
    v = (v | (v << np.uint32(16))) & np.uint32(0x030000FF)
    v = (v | (v << np.uint32(8))) & np.uint32(0x0300F00F)
    v = (v | (v << np.uint32(4))) & np.uint32(0x030C30C3)
    v = (v | (v << np.uint32(2))) & np.uint32(0x09249249)
    return v


def _compact1by2(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32) & np.uint32(0x09249249)
    v = (v | (v >> np.uint32(2))) & np.uint32(0x030C30C3)
    v = (v | (v >> np.uint32(4))) & np.uint32(0x0300F00F)
    v = (v | (v >> np.uint32(8))) & np.uint32(0x030000FF)
    v = (v | (v >> np.uint32(16))) & np.uint32(0x000003FF)
    return v


def morton3d(x, y, z) -> np.ndarray:
    return _part1by2(np.asarray(x)) | (_part1by2(np.asarray(y)) << np.uint32(1)) | (_part1by2(np.asarray(z)) << np.uint32(2))


def morton3d_invert(m) -> np.ndarray:
    return _compact1by2(np.asarray(m, dtype=np.uint32))


# ---------------------------------------------------------------------------------------
# Blob field
# ---------------------------------------------------------------------------------------
@dataclass
class BlobField:
    blobs: np.ndarray  # [n][5] float32: cx, cy, cz, std, peak
    waves: np.ndarray  # [3][4] float32: ax, ay, az, phase

    def density(self, p: np.ndarray) -> np.ndarray:
        """p: [..., 3] world positions (float64 math) -> density."""
        p = np.asarray(p, dtype=np.float64)
        s = np.zeros(p.shape[:-1])
        for cx, cy, cz, sd, pk in self.blobs.astype(np.float64):
            d2 = (p[..., 0] - cx) ** 2 + (p[..., 1] - cy) ** 2 + (p[..., 2] - cz) ** 2
            s += pk * np.exp(-d2 / (2.0 * sd * sd))
        return s

    def rgb(self, p: np.ndarray) -> np.ndarray:
        p = np.asarray(p, dtype=np.float64)
        out = []
        for ax, ay, az, ph in self.waves.astype(np.float64):
            a = ax * p[..., 0] + ay * p[..., 1] + az * p[..., 2] + ph
            out.append(1.0 / (1.0 + np.exp(-np.sin(a))))
        return np.stack(out, axis=-1)


def make_blob_field(rng: np.random.Generator, n_blobs: int = 8) -> BlobField:
    centers = rng.uniform(-1.0, 1.0, size=(n_blobs, 3))
    std = rng.uniform(0.1, 0.3, size=(n_blobs, 1))
    peak = rng.uniform(10.0, 100.0, size=(n_blobs, 1))
    blobs = np.concatenate([centers, std, peak], axis=1).astype(np.float32)
    waves = np.concatenate([rng.normal(0.0, 3.0, size=(3, 3)), rng.uniform(0, 2 * math.pi, size=(3, 1))],
                           axis=1).astype(np.float32)
    return BlobField(blobs=blobs, waves=waves)


# ---------------------------------------------------------------------------------------
# Occupancy grid
# ---------------------------------------------------------------------------------------
@dataclass
class Grid:
    n_levels: int
    resolution: int
    base_size: float
    bitfield: np.ndarray  # [R^3] uint8, Morton order, bit k = level k
    density: np.ndarray  # [n_levels][R^3] float32

    @property
    def volume(self) -> int:
        return self.resolution ** 3

    def level_size(self, k: int) -> float:
        return float(np.float32(self.base_size) * np.float32(1 << k))

    def as_dict(self):
        return dict(n_levels=self.n_levels, res=self.resolution, base=float(self.base_size), bitfield=self.bitfield)


def cell_centers(resolution: int, level_size: float) -> np.ndarray:
    """World-space centres of all cells of one level, in Morton order: [R^3, 3]."""
    m = np.arange(resolution ** 3, dtype=np.uint32)
    ix = morton3d_invert(m).astype(np.float64)
    iy = morton3d_invert(m >> np.uint32(1)).astype(np.float64)
    iz = morton3d_invert(m >> np.uint32(2)).astype(np.float64)
    vs = level_size / resolution
    half = resolution / 2
    return np.stack([(ix - half + 0.5) * vs, (iy - half + 0.5) * vs, (iz - half + 0.5) * vs], axis=1)


def build_grid(fld: BlobField, n_levels: int, base_size: float, resolution: int = 128,
               threshold: float = 0.01) -> Grid:
    V = resolution ** 3
    density = np.zeros((n_levels, V), np.float32)
    bits = np.zeros(V, np.uint8)
    for k in range(n_levels):
        ls = float(np.float32(base_size) * np.float32(1 << k))
        d = fld.density(cell_centers(resolution, ls)).astype(np.float32)
        density[k] = d
        bits |= ((d > np.float32(threshold)).astype(np.uint8) << np.uint8(k))
    return Grid(n_levels, resolution, float(base_size), bits, density)


# ---------------------------------------------------------------------------------------
# Rays
# ---------------------------------------------------------------------------------------
@dataclass
class RayBatch:
    n: int
    stride: int
    ori: np.ndarray  # [3][stride] float32
    dir: np.ndarray  # [3][stride] float32
    t: np.ndarray = field(default=None)
    t_max: np.ndarray = field(default=None)
    alive: np.ndarray = field(default=None)

    def as_dict(self):
        return dict(n=self.n, stride=self.stride, ori=self.ori, dir=self.dir, t=self.t, t_max=self.t_max,
                    alive=self.alive)


def sphere_rays(rng: np.random.Generator, n: int, radius: float = 4.0, jitter: float = 0.05,
                stride: int | None = None) -> RayBatch:
    """Origins uniform on a sphere of the given radius, directions toward the centre plus
    N(0, jitter) per component, normalised."""
    stride = stride or n
    o = rng.normal(size=(n, 3))
    o = radius * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o / np.linalg.norm(o, axis=1, keepdims=True) + rng.normal(0.0, jitter, size=(n, 3))
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    ori = np.zeros(3 * stride, np.float32)
    dr = np.zeros(3 * stride, np.float32)
    for c in range(3):
        ori[c * stride:c * stride + n] = o[:, c]
        dr[c * stride:c * stride + n] = d[:, c]
    return RayBatch(n=n, stride=stride, ori=ori, dir=dr)


def rays_init_bbox(rays: RayBatch, bbox, t_far: float = 3.0e38) -> RayBatch:
    """Bounding-box clip of the reference's ray set-up
    (src/utils/training-batch-kernels.cuh:122-150), in float32 numpy."""
    n, s = rays.n, rays.stride
    with np.errstate(divide="ignore", invalid="ignore"):
        o = [rays.ori[c * s:c * s + n] for c in range(3)]
        d = [rays.dir[c * s:c * s + n] for c in range(3)]
        inv = [np.float32(1.0) / dc for dc in d]
        lo = [np.float32(bbox[c]) for c in range(3)]
        hi = [np.float32(bbox[3 + c]) for c in range(3)]
        t1 = [(lo[c] - o[c]) * inv[c] for c in range(3)]
        t2 = [(hi[c] - o[c]) * inv[c] for c in range(3)]
        # swap when t1 > t2 (a NaN compares false and stays in place, as in the reference)
        a = [np.where(t1[c] > t2[c], t2[c], t1[c]) for c in range(3)]
        b = [np.where(t1[c] > t2[c], t1[c], t2[c]) for c in range(3)]
        tmin = np.fmax(a[0], np.fmax(a[1], a[2]))
        tmax = np.fmin(b[0], np.fmin(b[1], b[2]))
        hit = tmax >= tmin
        t_max = np.fmin(np.float32(t_far), tmax).astype(np.float32)
        t = np.fmax(np.float32(0.0), tmin + np.float32(1e-5)).astype(np.float32)
    alive = hit & ~(t_max < t)
    rays.t = np.where(alive, t, np.float32(0)).astype(np.float32)
    rays.t_max = np.where(alive, t_max, np.float32(0)).astype(np.float32)
    rays.alive = alive.astype(np.uint8)
    return rays


# ---------------------------------------------------------------------------------------
# Packed sample batches for the compositor / distortion loss
# ---------------------------------------------------------------------------------------
@dataclass
class SampleBatch:
    n_rays: int
    n_samples: int
    counts: np.ndarray  # [n_rays] uint32
    offsets: np.ndarray  # [n_rays] uint32 (exclusive scan of counts)
    sigma: np.ndarray  # [n_samples] float32
    rgb: np.ndarray  # [3][n_samples] float32
    t: np.ndarray  # [n_samples] float32 (world t)
    dt: np.ndarray  # [n_samples] float32 (world dt; also the compositor's dt)
    m_norm: np.ndarray  # [n_samples] float32
    dt_norm: np.ndarray  # [n_samples] float32
    target_rgba: np.ndarray  # [4][n_rays] float32
    bg_rgb: np.ndarray  # [3][n_rays] float32


def truncated_geometric_counts(rng, total: int, mean: float, lo: int = 1, hi: int = 1024) -> np.ndarray:
    p = 1.0 / mean
    out = []
    acc = 0
    while acc < total:
        c = rng.geometric(p, size=4096)
        c = c[(c >= lo) & (c <= hi)]
        for v in c:
            v = int(v)
            if acc + v >= total:
                v = total - acc
            out.append(v)
            acc += v
            if acc >= total:
                break
    return np.asarray(out, np.uint32)


def normalize_ray_t(t: np.ndarray, dt: np.ndarray, counts: np.ndarray, offsets: np.ndarray,
                    t_start: np.ndarray | None = None):
    """m_norm and dt_norm exactly as the reference's emit kernel computes them
    (src/utils/training-batch-kernels.cuh:424-425, 444-450, 476-480), in float32. The span
    runs from the ray's start t (t_start, default: its first sample) to the end of its last
    sample."""
    m = (t + np.float32(0.5) * dt).astype(np.float32)
    m_norm = np.zeros_like(t)
    dt_norm = np.zeros_like(t)
    c = counts.astype(np.int64)
    o = offsets.astype(np.int64)
    nz = c > 0
    first = o[nz]
    last = o[nz] + c[nz] - 1
    t_min = t[first] if t_start is None else np.asarray(t_start, np.float32)[nz]
    t_end = (t[last] + dt[last]).astype(np.float32)
    span = np.maximum((t_end - t_min).astype(np.float32), np.float32(1e-6))
    ray_of = np.repeat(np.arange(len(c))[nz], c[nz])
    span_s = np.zeros(len(c), np.float32)
    tmin_s = np.zeros(len(c), np.float32)
    span_s[nz] = span
    tmin_s[nz] = t_min
    mn = ((m - tmin_s[ray_of]) / span_s[ray_of]).astype(np.float32)
    m_norm[:] = np.clip(mn, np.float32(0), np.float32(1))
    dt_norm[:] = (dt / span_s[ray_of]).astype(np.float32)
    return m_norm, dt_norm


def make_sample_batch(seed: int, n_samples: int, mean: float = 48.0, max_count: int = 1024) -> SampleBatch:
    """Compositor/distortion workload: counts ~ truncated geometric (mean, 1..max_count),
    sigma = clip(exp(N(0,2)), 0, 1e4), rgb = sigmoid(N(0,1)),
    dt ~ U[0.5,2]*sqrt(3)/1024, t0 ~ U[0,1], target rgb U[0,1]^3 (alpha 1), bg U[0,1]^3."""
    rng = np.random.default_rng(seed)
    counts = truncated_geometric_counts(rng, n_samples, mean, 1, max_count)
    n_rays = len(counts)
    offsets = np.zeros(n_rays, np.uint32)
    offsets[1:] = np.cumsum(counts[:-1], dtype=np.uint64).astype(np.uint32)
    sigma = np.clip(np.exp(rng.normal(0.0, 2.0, n_samples)), 0.0, 1e4).astype(np.float32)
    rgb = (1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, 3 * n_samples)))).astype(np.float32)
    dt = (rng.uniform(0.5, 2.0, n_samples) * float(MIN_STEP_SIZE)).astype(np.float32)
    t0 = rng.uniform(0.0, 1.0, n_rays).astype(np.float32)
    t = np.zeros(n_samples, np.float32)
    # t strictly increasing inside each ray: t_j = t0 + sum_{i<j} dt_i (float32, sequential)
    ray_of = np.repeat(np.arange(n_rays), counts.astype(np.int64))
    csum = np.cumsum(dt.astype(np.float64))
    start = offsets.astype(np.int64)
    base = np.where(start > 0, csum[np.maximum(start - 1, 0)], 0.0)
    excl = csum - dt.astype(np.float64) - base[ray_of]
    t[:] = (t0[ray_of].astype(np.float64) + excl).astype(np.float32)
    m_norm, dt_norm = normalize_ray_t(t, dt, counts, offsets)
    target = np.concatenate([rng.uniform(0, 1, 3 * n_rays), np.ones(n_rays)]).astype(np.float32)
    bg = rng.uniform(0, 1, 3 * n_rays).astype(np.float32)
    return SampleBatch(n_rays, n_samples, counts, offsets, sigma, rgb, t, dt, m_norm, dt_norm, target, bg)


# ---------------------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------------------
@dataclass
class MarchScene:
    field: BlobField
    grid: Grid
    bbox: tuple
    rays: RayBatch
    cone_angle: float
    dt_min: float
    dt_max: float
    max_steps: int
    aabb_size: float


def march_scene_single(seed: int = SEED, n_rays: int = 4096) -> MarchScene:
    """Forward march + composite: 1 cascade of 128^3 over AABB [-1.5,1.5]^3 (base size 3),
    8 blobs, 4096 rays from a radius-4 sphere, dt = sqrt(3)/1024 fixed, <= 1024 steps."""
    rng = np.random.default_rng(seed)
    fld = make_blob_field(rng, 8)
    grid = build_grid(fld, n_levels=1, base_size=3.0)
    bbox = (-1.5, -1.5, -1.5, 1.5, 1.5, 1.5)
    rays = rays_init_bbox(sphere_rays(rng, n_rays), bbox)
    dt = float(MIN_STEP_SIZE)
    return MarchScene(fld, grid, bbox, rays, 0.0, dt, dt, 1024, 3.0)


def march_scene_cascaded(seed: int = SEED, n_rays: int = 1 << 14, n_levels: int = 5) -> MarchScene:
    """Full train step scene: 5 cascades (extents 1,2,4,8,16; base size 1 = the reference),
    the 8-blob field of the single-cascade scene, rays from a radius-4 sphere, the reference's
    cone-angle stepping: dt = clamp(t/256, dt_min, aabb*dt_min) (src/core/trainer.cu:102-104)."""
    rng = np.random.default_rng(seed)
    fld = make_blob_field(rng, 8)
    grid = build_grid(fld, n_levels=n_levels, base_size=1.0)
    aabb = float(1 << (n_levels - 1))
    h = aabb / 2
    bbox = (-h, -h, -h, h, h, h)
    rays = rays_init_bbox(sphere_rays(rng, n_rays), bbox)
    dt = float(MIN_STEP_SIZE)
    return MarchScene(fld, grid, bbox, rays, 1.0 / 256.0, dt, float(np.float32(aabb) * np.float32(dt)), 0, aabb)


# ---------------------------------------------------------------------------------------
# Several scenes in one batch
# ---------------------------------------------------------------------------------------
@dataclass
class MultiScene:
    scenes: list           # MarchScene per scene (grid may be None until built)
    ray_begin: np.ndarray  # [n_scenes] first ray of each scene in the shared arrays
    rays: RayBatch         # all scenes' rays, scene after scene (box clip applied per scene)


def multi_scene_params(seed: int = SEED, n_scenes: int = 16, ray_lo: int = 1 << 10, ray_hi: int = 1 << 16):
    """Per-scene parameters of the batched multi-scene workload: a blob field of 8-32 blobs,
    1-5 cascades, an AABB of size 0.5-16 (the coarsest level covers it), ray counts drawn
    log-uniform in [ray_lo, ray_hi]. The field's geometry is the single-cascade scene's scaled
    to the box: centres in +-A/3, standard deviations 0.1-0.3 A/3."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_scenes):
        n_blobs = int(rng.integers(8, 33))
        n_levels = int(rng.integers(1, 6))
        aabb = float(np.float32(np.exp(rng.uniform(np.log(0.5), np.log(16.0)))))
        n_rays = int(np.exp(rng.uniform(np.log(ray_lo), np.log(ray_hi))))
        fld = make_blob_field(rng, n_blobs)
        scale = aabb / 3.0
        fld.blobs[:, :4] *= np.float32(scale)
        out.append(dict(field=fld, n_levels=n_levels, aabb=aabb, n_rays=n_rays,
                        seed=int(rng.integers(0, 2**31 - 1))))
    return out


def make_multi_scene(params, resolution: int = 32, grids: bool = True) -> MultiScene:
    """Builds the scenes of multi_scene_params: grids (numpy, when grids is set), rays from a
    sphere of radius 4A/3 toward the centre (the single-cascade scene's geometry scaled), box
    clip, and the reference's cone stepping (dt = clamp(t/256, dt_min, max(A, 1) dt_min))."""
    total = sum(p["n_rays"] for p in params)
    ori = np.zeros(3 * total, np.float32)
    dr = np.zeros(3 * total, np.float32)
    t = np.zeros(total, np.float32)
    tmax = np.zeros(total, np.float32)
    alive = np.zeros(total, np.uint8)
    scenes, begins = [], []
    b = 0
    dt = float(MIN_STEP_SIZE)
    for p in params:
        A = p["aabb"]
        n_levels = p["n_levels"]
        base = float(np.float32(A) / np.float32(1 << (n_levels - 1)))
        h = A / 2
        bbox = (-h, -h, -h, h, h, h)
        rng = np.random.default_rng(p["seed"])
        r = rays_init_bbox(sphere_rays(rng, p["n_rays"], radius=4.0 * A / 3.0), bbox)
        n = p["n_rays"]
        for c in range(3):
            ori[c * total + b:c * total + b + n] = r.ori[c * n:(c + 1) * n]
            dr[c * total + b:c * total + b + n] = r.dir[c * n:(c + 1) * n]
        t[b:b + n], tmax[b:b + n], alive[b:b + n] = r.t[:n], r.t_max[:n], r.alive[:n]
        grid = build_grid(p["field"], n_levels, base, resolution) if grids else None
        dt_max = float(np.float32(max(A, 1.0)) * np.float32(dt))
        scenes.append(MarchScene(p["field"], grid, bbox, r, 1.0 / 256.0, dt, dt_max, 1024, A))
        begins.append(b)
        b += n
    rays = RayBatch(total, total, ori, dr, t, tmax, alive)
    return MultiScene(scenes, np.asarray(begins, np.uint32), rays)
