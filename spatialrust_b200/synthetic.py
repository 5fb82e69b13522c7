"""Seeded synthetic point clouds with the shapes of the benchmark workloads.

Every generator is deterministic for a given seed (numpy PCG64).  Georeferenced
clouds are generated in FP64 world coordinates and handed to the filters as
f32(world - cloud_origin) computed in FP64, the form in which SpatialRust holds
them (f32 position columns).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GEO_OFFSET = np.array([450000.0, 3900000.0, 50.0])


@dataclass
class Cloud:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    intensity: np.ndarray
    origin: np.ndarray  # FP64 world origin subtracted from the coordinates

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def xyz(self) -> np.ndarray:
        return np.stack([self.x, self.y, self.z], axis=1)


def uniform_cube(n: int = 100_000, extent: float = 100.0, seed: int = 0) -> Cloud:
    """Uniform point_xyzi cloud in [0, extent)^3, intensity U[0,1)."""
    rng = np.random.default_rng(seed)
    xyz = (rng.random((n, 3), dtype=np.float32) * np.float32(extent)).astype(np.float32)
    inten = rng.random(n, dtype=np.float32)
    return Cloud(np.ascontiguousarray(xyz[:, 0]), np.ascontiguousarray(xyz[:, 1]),
                 np.ascontiguousarray(xyz[:, 2]), inten, np.zeros(3))


def _box_surface(rng, n, centers, sizes):
    """n points uniformly on the surfaces (five faces, no bottom) of axis-aligned boxes."""
    nb = centers.shape[0]
    sx, sy, sz = sizes[:, 0], sizes[:, 1], sizes[:, 2]
    face_area = np.stack([sx * sy, sx * sz, sx * sz, sy * sz, sy * sz], axis=1)  # top, +-y, +-x
    box_area = face_area.sum(axis=1)
    box = rng.choice(nb, size=n, p=box_area / box_area.sum())
    face = np.empty(n, np.int64)
    for b in range(nb):
        idx = np.nonzero(box == b)[0]
        if idx.size:
            face[idx] = rng.choice(5, size=idx.size, p=face_area[b] / face_area[b].sum())
    u = rng.random(n)
    v = rng.random(n)
    c, s = centers[box], sizes[box]
    lo = c - s / 2.0
    pts = np.empty((n, 3))
    # top
    m = face == 0
    pts[m] = np.stack([lo[m, 0] + u[m] * s[m, 0], lo[m, 1] + v[m] * s[m, 1], lo[m, 2] + s[m, 2]], 1)
    for f, yside in ((1, 0.0), (2, 1.0)):
        m = face == f
        pts[m] = np.stack([lo[m, 0] + u[m] * s[m, 0], lo[m, 1] + yside * s[m, 1],
                           lo[m, 2] + v[m] * s[m, 2]], 1)
    for f, xside in ((3, 0.0), (4, 1.0)):
        m = face == f
        pts[m] = np.stack([lo[m, 0] + xside * s[m, 0], lo[m, 1] + u[m] * s[m, 1],
                           lo[m, 2] + v[m] * s[m, 2]], 1)
    return pts


def scan_mixture_world(n: int, seed: int, square: float = 200.0, n_boxes: int = 200,
                       offset=GEO_OFFSET) -> np.ndarray:
    """Georeferenced scan-like mixture in FP64 world coordinates:
    60% ground plane z ~ N(0, 0.02) over a square x square m area, 30% on the
    faces of n_boxes axis-aligned boxes (sides U[0.5, 8] m, centres uniform in
    the square, standing on the ground), 10% uniform clutter in square x square x 20 m."""
    rng = np.random.default_rng(seed)
    n_ground = int(round(n * 0.6))
    n_box = int(round(n * 0.3))
    n_clutter = n - n_ground - n_box
    ground = np.stack([rng.random(n_ground) * square, rng.random(n_ground) * square,
                       rng.normal(0.0, 0.02, n_ground)], axis=1)
    sizes = rng.uniform(0.5, 8.0, (n_boxes, 3))
    centers = np.stack([rng.random(n_boxes) * square, rng.random(n_boxes) * square,
                        sizes[:, 2] / 2.0], axis=1)
    boxes = _box_surface(rng, n_box, centers, sizes)
    clutter = np.stack([rng.random(n_clutter) * square, rng.random(n_clutter) * square,
                        rng.random(n_clutter) * 20.0], axis=1)
    pts = np.concatenate([ground, boxes, clutter], axis=0)
    perm = rng.permutation(n)
    return pts[perm] + np.asarray(offset, np.float64)


def georef_scan(n: int = 2_000_000, seed: int = 1, offset=GEO_OFFSET) -> Cloud:
    """Georeferenced 2M-point point_xyzi scan-like cloud (intensity Beta(2,5)),
    returned as f32(world - offset) computed in FP64."""
    world = scan_mixture_world(n, seed, offset=offset)
    rng = np.random.default_rng(seed + 1_000_003)
    inten = rng.beta(2.0, 5.0, n).astype(np.float32)
    origin = np.asarray(offset, np.float64)
    local = (world - origin).astype(np.float32)
    return Cloud(np.ascontiguousarray(local[:, 0]), np.ascontiguousarray(local[:, 1]),
                 np.ascontiguousarray(local[:, 2]), inten, origin)


def _random_rotations(rng, k):
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def shapes_scene(n: int = 5_000_000, seed: int = 2, noise: float = 0.005,
                 extent: float = 100.0) -> Cloud:
    """Radius-normal workload: 40% on 50 spheres (radius U[1,5]), 40% on 30
    randomly oriented 10x10 m planar patches, 20% on 20 cylinders (radius
    U[0.2,1], length 5 m, random axes), all inside extent^3 m, with N(0, noise)
    displacement along the surface normal."""
    rng = np.random.default_rng(seed)
    n_sph = int(round(n * 0.4))
    n_pl = int(round(n * 0.4))
    n_cyl = n - n_sph - n_pl
    margin = 8.0
    # spheres
    rad = rng.uniform(1.0, 5.0, 50)
    cen = rng.uniform(margin, extent - margin, (50, 3))
    area = rad ** 2
    which = rng.choice(50, size=n_sph, p=area / area.sum())
    d = rng.normal(size=(n_sph, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sph = cen[which] + d * (rad[which] + rng.normal(0.0, noise, n_sph))[:, None]
    # planes
    rot = _random_rotations(rng, 30)
    pc = rng.uniform(margin, extent - margin, (30, 3))
    which = rng.integers(0, 30, n_pl)
    uv = rng.uniform(-5.0, 5.0, (n_pl, 2))
    local = np.stack([uv[:, 0], uv[:, 1], rng.normal(0.0, noise, n_pl)], axis=1)
    pl = pc[which] + np.einsum("nij,nj->ni", rot[which], local)
    # cylinders
    crot = _random_rotations(rng, 20)
    cc = rng.uniform(margin, extent - margin, (20, 3))
    cr = rng.uniform(0.2, 1.0, 20)
    which = rng.choice(20, size=n_cyl, p=cr / cr.sum())
    th = rng.uniform(0.0, 2 * np.pi, n_cyl)
    h = rng.uniform(-2.5, 2.5, n_cyl)
    rr = cr[which] + rng.normal(0.0, noise, n_cyl)
    local = np.stack([rr * np.cos(th), rr * np.sin(th), h], axis=1)
    cyl = cc[which] + np.einsum("nij,nj->ni", crot[which], local)
    pts = np.concatenate([sph, pl, cyl], axis=0)
    pts = pts[rng.permutation(n)].astype(np.float32)
    inten = rng.random(n, dtype=np.float32)
    return Cloud(np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1]),
                 np.ascontiguousarray(pts[:, 2]), inten, np.zeros(3))


def batched_uneven(count: int = 256, lo: int = 10_000, hi: int = 1_000_000, seed: int = 3,
                   max_offset: float = 1e6, scale: float = 1.0, max_points: int | None = None):
    """Many uneven clouds: sizes log-uniform in [lo, hi], each the scan mixture with
    its own seed and a random FP64 origin offset up to max_offset m; per-cloud leaf
    in {0.05, 0.1, 0.2} m and radius 5 x leaf.  `scale` shrinks every size (tests).
    With max_points, generation stops once the clouds made (two at least) hold
    max_points or more; they are the first clouds of the full batch."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    sizes = np.maximum((sizes * scale).astype(np.int64), 16)
    leaves = rng.choice(np.array([0.05, 0.1, 0.2], np.float32), size=count)
    clouds, total = [], 0
    for i in range(count):
        off = rng.uniform(0.0, max_offset, 3)
        off[2] = rng.uniform(0.0, 100.0)
        c = georef_scan(int(sizes[i]), seed=seed * 100_003 + i, offset=off)
        clouds.append(c)
        total += c.n
        if max_points is not None and total >= max_points and len(clouds) >= 2:
            break
    k = len(clouds)
    return clouds, leaves[:k], (leaves[:k] * np.float32(5.0)).astype(np.float32)


def lidar_scene(seed: int = 4, n_boxes: int = 100, extent: float = 120.0):
    """Seeded scene for ray-cast LiDAR frames: the ground plane z = 0 plus
    n_boxes axis-aligned boxes (sides U[0.5, 8] m, standing on the ground,
    centres uniform within +-extent m).  Returns (lo, hi) box corners."""
    rng = np.random.default_rng(seed)
    sizes = rng.uniform(0.5, 8.0, (n_boxes, 3))
    centers = np.stack([rng.uniform(-extent, extent, n_boxes), rng.uniform(-extent, extent, n_boxes),
                        sizes[:, 2] / 2.0], axis=1)
    return centers - sizes / 2.0, centers + sizes / 2.0


def lidar_frame(seed: int = 0, scene=None, beams: int = 64, azimuths: int = 2048,
                elev_deg=(-25.0, 15.0), max_range: float = 120.0, noise: float = 0.02,
                sensor_height: float = 1.8) -> Cloud:
    """One spinning-LiDAR frame (beams x azimuths points, sensor frame): each
    ray's range is its first hit on the scene (ground or box, slab test), or
    max_range when nothing is hit, plus N(0, noise) range noise, clipped to
    (0, max_range]; intensity U[0, 1).  The sensor sits at a seeded position
    and yaw, sensor_height m above the ground, outside every box."""
    lo, hi = scene if scene is not None else lidar_scene()
    rng = np.random.default_rng(seed)
    for _ in range(1000):
        pos = np.array([rng.uniform(-60, 60), rng.uniform(-60, 60), sensor_height])
        if not np.any(np.all((pos >= lo - 0.5) & (pos <= hi + 0.5), axis=1)):
            break
    yaw = rng.uniform(0.0, 2.0 * np.pi)
    el = np.deg2rad(np.linspace(elev_deg[0], elev_deg[1], beams))
    az = yaw + np.arange(azimuths) * (2.0 * np.pi / azimuths)
    ce, se = np.cos(el)[:, None], np.sin(el)[:, None]
    d = np.stack([np.broadcast_to(ce * np.cos(az), (beams, azimuths)),
                  np.broadcast_to(ce * np.sin(az), (beams, azimuths)),
                  np.broadcast_to(se, (beams, azimuths))], axis=-1).reshape(-1, 3)
    t = np.full(d.shape[0], max_range)
    down = d[:, 2] < -1e-9
    t[down] = np.minimum(t[down], -pos[2] / d[down, 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        for b in range(lo.shape[0]):
            t1 = (lo[b] - pos) * inv
            t2 = (hi[b] - pos) * inv
            tn = np.nanmax(np.minimum(t1, t2), axis=1)
            tf = np.nanmin(np.maximum(t1, t2), axis=1)
            hit = (tn <= tf) & (tn > 0.0) & (tn < t)
            t[hit] = tn[hit]
    r = np.clip(t + rng.normal(0.0, noise, t.shape[0]), 1e-3, max_range)
    pts = (d * r[:, None]).astype(np.float32)
    inten = rng.random(pts.shape[0], dtype=np.float32)
    return Cloud(np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1]),
                 np.ascontiguousarray(pts[:, 2] + np.float32(sensor_height)), inten, np.zeros(3))


def map_chunk(n: int, seed: int) -> Cloud:
    """A map-chunk request: the georeferenced scan mixture with n points."""
    return georef_scan(n, seed=seed)


def unit_plane_grid(nx: int, ny: int, step: float, z: float = 0.0, x0: float = 0.0,
                    y0: float = 0.0) -> Cloud:
    """Regular grid in the plane z = const (the reference's planar test clouds)."""
    xs = []
    ys = []
    for i in range(nx):
        for j in range(ny):
            xs.append(np.float32(i) * np.float32(step) + np.float32(x0))
            ys.append(np.float32(j) * np.float32(step) + np.float32(y0))
    x = np.asarray(xs, np.float32)
    y = np.asarray(ys, np.float32)
    return Cloud(x, y, np.full_like(x, np.float32(z)), np.zeros_like(x), np.zeros(3))
