"""Seeded synthetic scenes and ray batches for the traversal benchmarks and parity tests.

No public dataset is involved: every input is generated here, deterministically, from a
splitmix64 counter stream (seed ``0x5EED0000 + config``). A uniform float is the top 24 bits of a
draw divided by 2**24; a normal draw is Box-Muller over two uniforms. Geometry is float32,
indices uint32. Shapes follow the five benchmark configurations:

1. ``cubes``: 10,000 unit cubes (12 triangles, 8 shared vertices each) on a 100 x 100 grid of
   spacing 2, jitter U(-0.3, 0.3) in x and z, scale U(0.5, 1.5), yaw U(0, 2 pi), resting on y = 0;
   a 1024 x 1024 pinhole camera (fov 60 deg vertical) at (0, 40, -69.28) pitched 30 deg down,
   plus one sun ray per hit toward normalise(0.3, 0.8, 0.2).
2. ``clusters``: triangles in clusters of 500; cluster centres U[-100, 100]^3, each triangle's
   first vertex uniform in a ball of radius 5 about its centre, its two edges log-normal
   (mu = ln 0.5, sigma = 0.8) long along independent uniform directions; 2048 x 2048 primaries
   from (0, 0, -250) looking +z, then cosine-hemisphere GI rays from the primary hits.
3. the same generator at 4M triangles with a mixed ray set.
4. many BLAS under a top level of rotated, scaled, translated instances.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MASK64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15


class Stream:
    """A splitmix64 counter stream: draw k is splitmix64's output for state seed + k * GOLDEN."""

    def __init__(self, seed: int):
        self.seed = seed & MASK64
        self.count = 0

    def raw(self, n: int) -> np.ndarray:
        k = np.arange(self.count + 1, self.count + 1 + n, dtype=np.uint64)
        self.count += n
        with np.errstate(over="ignore"):
            z = np.uint64(self.seed) + k * np.uint64(GOLDEN)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        return z

    def uniform(self, *shape) -> np.ndarray:
        """U[0, 1) in float64, 24-bit resolution."""
        n = int(np.prod(shape)) if shape else 1
        u = (self.raw(n) >> np.uint64(40)).astype(np.float64) / float(1 << 24)
        return u.reshape(shape) if shape else u[0]

    def range(self, lo, hi, *shape) -> np.ndarray:
        return lo + (hi - lo) * self.uniform(*shape)

    def normal(self, *shape) -> np.ndarray:
        """Box-Muller over (1 - u1, u2); one normal per pair of draws."""
        n = int(np.prod(shape))
        u = self.uniform(n, 2)
        z = np.sqrt(-2.0 * np.log(1.0 - u[:, 0])) * np.cos(2.0 * np.pi * u[:, 1])
        return z.reshape(shape)

    def unit_vectors(self, n: int) -> np.ndarray:
        u = self.uniform(n, 2)
        z = 2.0 * u[:, 0] - 1.0
        phi = 2.0 * np.pi * u[:, 1]
        r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
        return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def seed_for(config: int) -> int:
    return 0x5EED0000 + config


@dataclass
class Mesh:
    positions: np.ndarray  # (V, 3) float32
    indices: np.ndarray    # (3T,) uint32

    @property
    def triangles(self) -> int:
        return len(self.indices) // 3


@dataclass
class Instances:
    """Object-to-world models and their world-to-object rows (3 x 4 each), as the packers take."""
    model: np.ndarray  # (N, 3, 4) float32
    rows: np.ndarray   # (N, 3, 4) float32
    mesh: np.ndarray   # (N,) uint32
    casts: np.ndarray = field(default=None)  # (N,) bool; None: all cast shadows

    def __post_init__(self):
        if self.casts is None:
            self.casts = np.ones(len(self.mesh), bool)

    def __len__(self):
        return len(self.mesh)


def identity_instances(n_meshes: int = 1) -> Instances:
    eye = np.zeros((n_meshes, 3, 4), np.float32)
    eye[:, 0, 0] = eye[:, 1, 1] = eye[:, 2, 2] = 1.0
    return Instances(eye.copy(), eye.copy(), np.arange(n_meshes, dtype=np.uint32))


def affine_inverse_rows(model: np.ndarray) -> np.ndarray:
    """World-to-object rows of affine models (N,3,4), computed in float64 and rounded once."""
    m = model.astype(np.float64)
    a = m[:, :, :3]
    t = m[:, :, 3]
    ai = np.linalg.inv(a)
    rows = np.concatenate([ai, -np.einsum("nij,nj->ni", ai, t)[:, :, None]], axis=2)
    return rows.astype(np.float32)


# ---------------------------------------------------------------- geometry

_CUBE_V = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)], np.float64)
# 12 outward-wound triangles over the 8 corners (index = x + 2y + 4z).
_CUBE_T = np.array([
    0, 2, 1, 1, 2, 3,   # z = -0.5
    4, 5, 6, 5, 7, 6,   # z = +0.5
    0, 1, 4, 1, 5, 4,   # y = -0.5
    2, 6, 3, 3, 6, 7,   # y = +0.5
    0, 4, 2, 2, 4, 6,   # x = -0.5
    1, 3, 5, 3, 7, 5,   # x = +0.5
], np.uint32)


def cube_params(n_side: int = 100, config: int = 1):
    s = Stream(seed_for(config))
    u = s.uniform(n_side * n_side, 4)  # per cell: jitter x, jitter z, scale, yaw
    gz, gx = np.meshgrid(np.arange(n_side), np.arange(n_side), indexing="ij")
    cx = (gx.reshape(-1) - (n_side - 1) / 2.0) * 2.0 + (u[:, 0] * 0.6 - 0.3)
    cz = (gz.reshape(-1) - (n_side - 1) / 2.0) * 2.0 + (u[:, 1] * 0.6 - 0.3)
    scale = 0.5 + u[:, 2]
    yaw = u[:, 3] * 2.0 * np.pi
    return cx, cz, scale, yaw


def cube_models(n_side: int = 100, config: int = 1) -> np.ndarray:
    cx, cz, scale, yaw = cube_params(n_side, config)
    c, s_ = np.cos(yaw), np.sin(yaw)
    n = len(cx)
    m = np.zeros((n, 3, 4), np.float64)
    m[:, 0, 0], m[:, 0, 2] = c * scale, s_ * scale
    m[:, 1, 1] = scale
    m[:, 2, 0], m[:, 2, 2] = -s_ * scale, c * scale
    m[:, 0, 3], m[:, 1, 3], m[:, 2, 3] = cx, 0.5 * scale, cz
    return m


def cubes_merged(n_side: int = 100, config: int = 1) -> Mesh:
    """Config 1: every cube's 8 corners transformed into one world-space mesh."""
    m = cube_models(n_side, config)
    v = np.einsum("nij,kj->nki", m[:, :, :3], _CUBE_V) + m[:, None, :, 3]
    n = len(m)
    idx = (_CUBE_T[None, :] + (np.arange(n, dtype=np.uint32) * 8)[:, None]).reshape(-1)
    return Mesh(v.reshape(-1, 3).astype(np.float32), idx.astype(np.uint32))


def cubes_instanced(n_side: int = 100, config: int = 1):
    """Config 1b: one 12-triangle cube BLAS under n_side^2 instances."""
    m = cube_models(n_side, config)
    mesh = Mesh(_CUBE_V.astype(np.float32), _CUBE_T.copy())
    model = m.astype(np.float32)
    inst = Instances(model, affine_inverse_rows(m), np.zeros(len(m), np.uint32))
    return mesh, inst


def clusters(n_triangles: int, config: int = 2, per_cluster: int = 500, half: float = 100.0,
             radius: float = 5.0, stream: Stream | None = None) -> Mesh:
    """Config 2/3 cluster soup: unshared vertices, 3 per triangle."""
    s = stream or Stream(seed_for(config))
    n_clusters = (n_triangles + per_cluster - 1) // per_cluster
    centres = s.range(-half, half, n_clusters, 3)
    owner = np.minimum(np.arange(n_triangles) // per_cluster, n_clusters - 1)
    # per triangle: ball point (dir 2 + radius 1), two log-normal lengths, two directions
    ball_dir = s.unit_vectors(n_triangles)
    ball_r = radius * np.cbrt(s.uniform(n_triangles))
    l1 = np.exp(math.log(0.5) + 0.8 * s.normal(n_triangles))
    l2 = np.exp(math.log(0.5) + 0.8 * s.normal(n_triangles))
    d1 = s.unit_vectors(n_triangles)
    d2 = s.unit_vectors(n_triangles)
    a = centres[owner] + ball_dir * ball_r[:, None]
    b = a + d1 * l1[:, None]
    c = a + d2 * l2[:, None]
    pos = np.stack([a, b, c], axis=1).reshape(-1, 3).astype(np.float32)
    return Mesh(pos, np.arange(3 * n_triangles, dtype=np.uint32))


def quaternion_matrices(s: Stream, n: int) -> np.ndarray:
    """Uniformly random rotations (Shoemake's subgroup algorithm), (n, 3, 3) float64."""
    u = s.uniform(n, 3)
    a, b = np.sqrt(1.0 - u[:, 0]), np.sqrt(u[:, 0])
    t1, t2 = 2.0 * np.pi * u[:, 1], 2.0 * np.pi * u[:, 2]
    x, y, z, w = a * np.sin(t1), a * np.cos(t1), b * np.sin(t2), b * np.cos(t2)
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], axis=1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], axis=1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], axis=1),
    ], axis=1)


@dataclass
class MultiScene:
    meshes: list       # Mesh per BLAS
    instances: Instances
    half: float        # instances' translations lie in [-half, half]^3


def multi_blas(n_blas: int = 64, n_instances: int = 10_000, tri_lo: float = 2e3, tri_hi: float = 5e5,
               half: float = 500.0, scale=(0.5, 4.0), config: int = 4) -> MultiScene:
    """Config 4 / 5 scenes: n_blas cluster meshes with log-uniform triangle counts, under
    n_instances instances with uniform random rotations, uniform scales and translations in
    [-half, half]^3; each instance picks its BLAS uniformly."""
    s = Stream(seed_for(config))
    counts = np.round(np.exp(s.range(np.log(tri_lo), np.log(tri_hi), n_blas))).astype(np.int64)
    meshes = [clusters(int(c), stream=Stream(seed_for(config) ^ (0x9E37 * (k + 1)))) for k, c in enumerate(counts)]
    which = np.minimum((s.uniform(n_instances) * n_blas).astype(np.int64), n_blas - 1).astype(np.uint32)
    rot = quaternion_matrices(s, n_instances)
    sc = s.range(scale[0], scale[1], n_instances)
    tr = s.range(-half, half, n_instances, 3)
    model = np.concatenate([rot * sc[:, None, None], tr[:, :, None]], axis=2).astype(np.float32)
    return MultiScene(meshes, Instances(model, affine_inverse_rows(model), which), half)


def uneven_batches(n_batches: int = 64, lo: float = 1e3, hi: float = 2e6, half: float = 500.0, config: int = 4,
                   tmax: float = 1e30):
    """Config 4 ray batches: sizes log-uniform in [lo, hi], closest / any hit by a fair coin per
    batch, origins uniform in [-half, half]^3, directions uniform on the sphere. Returns a list
    of (rays, mode) with mode 0 closest, 2 any hit (casters within tmax)."""
    s = Stream(seed_for(config) + 0x100)
    sizes = np.round(np.exp(s.range(np.log(lo), np.log(hi), n_batches))).astype(np.int64)
    coins = s.uniform(n_batches) < 0.5
    out = []
    for n, any_hit in zip(sizes, coins):
        o = s.range(-half, half, int(n), 3)
        d = s.unit_vectors(int(n))
        out.append((pack_rays(o, d, 0.0, tmax), 2 if any_hit else 0))
    return out


# ---------------------------------------------------------------- rays

RAY_DTYPE = np.dtype([("o", np.float32, 3), ("tmin", np.float32), ("d", np.float32, 3), ("tmax", np.float32)])


def pack_normal(n: np.ndarray) -> np.ndarray:
    """Unit normals (N, 3) in the GI cache's octahedral pack2x16snorm word (gi_cache.wgsl
    gi_pack_normal)."""
    n = np.asarray(n, np.float64)
    p = n[:, :2] / np.abs(n).sum(axis=1, keepdims=True)
    sign = np.where(p >= 0.0, 1.0, -1.0)
    q = np.where(n[:, 2:3] >= 0.0, p, (1.0 - np.abs(p[:, ::-1])) * sign)
    s = np.round(np.clip(q, -1.0, 1.0) * 32767.0).astype(np.int64) & 0xFFFF
    return (s[:, 0] | (s[:, 1] << 16)).astype(np.uint32)


def gi_cells(points: np.ndarray, normals: np.ndarray, edge: float, stream: Stream) -> np.ndarray:
    """rt_gi_cell records (N, 8) uint32 at the given points: query point, cell edge, packed
    normal, a random key word."""
    n = len(points)
    out = np.zeros((n, 8), np.uint32)
    out[:, 0:3] = np.asarray(points, np.float32).view(np.uint32)
    out[:, 3] = np.float32(edge).view(np.uint32)
    out[:, 4] = pack_normal(normals)
    out[:, 5] = (stream.raw(n) >> np.uint64(32)).astype(np.uint32)
    return out


def pack_rays(o, d, tmin, tmax) -> np.ndarray:
    """(n, 8) float32 records: origin xyz, tmin, direction xyz, tmax (the 32-byte rt_ray)."""
    n = len(o)
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def pinhole(eye, forward, width, height, fov_deg=60.0, tile=(8, 4)) -> np.ndarray:
    """Unit primary directions through pixel centres, in tile order (tile = (tw, th) pixels,
    row-major tiles of row-major pixels) so that a warp of 32 rays covers one 8 x 4 tile."""
    f = np.asarray(forward, np.float64)
    f = f / np.linalg.norm(f)
    right = np.cross([0.0, 1.0, 0.0], f)
    right /= np.linalg.norm(right)
    up = np.cross(f, right)
    tw, th = tile
    assert width % tw == 0 and height % th == 0
    ty, tx, py, px = np.meshgrid(np.arange(height // th), np.arange(width // tw), np.arange(th),
                                 np.arange(tw), indexing="ij")
    x = (tx * tw + px).reshape(-1)
    y = (ty * th + py).reshape(-1)
    k = math.tan(math.radians(fov_deg) / 2.0)
    u = ((x + 0.5) / width * 2.0 - 1.0) * k * (width / height)
    v = (1.0 - (y + 0.5) / height * 2.0) * k
    d = f[None, :] + u[:, None] * right[None, :] + v[:, None] * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def cube_camera_rays(width=1024, height=1024) -> np.ndarray:
    eye = np.array([0.0, 40.0, -69.28])
    pitch = math.radians(30.0)
    fwd = np.array([0.0, -math.sin(pitch), math.cos(pitch)])
    d = pinhole(eye, fwd, width, height)
    return pack_rays(np.broadcast_to(eye, d.shape), d, 0.0, 1e30)


def cluster_camera_rays(width=2048, height=2048, eye=(0.0, 0.0, -250.0)) -> np.ndarray:
    d = pinhole(np.asarray(eye), [0.0, 0.0, 1.0], width, height)
    return pack_rays(np.broadcast_to(np.asarray(eye, np.float64), d.shape), d, 0.0, 1e30)


def offset_tmin(points: np.ndarray) -> np.ndarray:
    """The secondary-ray tmin: 1e-4 * max(1, |p|_inf)."""
    return (1e-4 * np.maximum(1.0, np.abs(points).max(axis=1))).astype(np.float32)


def sun_rays(hit_points: np.ndarray, sun=(0.3, 0.8, 0.2)) -> np.ndarray:
    s = np.asarray(sun, np.float64)
    s /= np.linalg.norm(s)
    d = np.broadcast_to(s, hit_points.shape)
    return pack_rays(hit_points, d, offset_tmin(hit_points), 1e30)


def hemisphere_rays(points: np.ndarray, normals: np.ndarray, incoming: np.ndarray, count: int,
                    stream: Stream, tmax=1e20) -> np.ndarray:
    """`count` cosine-weighted rays about the face normals (flipped toward the incoming ray's
    side), from the given hit points taken in turn."""
    k = np.arange(count) % len(points)
    p = points[k].astype(np.float64)
    n = normals[k].astype(np.float64)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    flip = np.einsum("ij,ij->i", n, incoming[k].astype(np.float64)) > 0.0
    n[flip] *= -1.0
    u = stream.uniform(count, 2)
    r = np.sqrt(u[:, 0])
    phi = 2.0 * np.pi * u[:, 1]
    lx, ly, lz = r * np.cos(phi), r * np.sin(phi), np.sqrt(np.maximum(0.0, 1.0 - u[:, 0]))
    helper = np.where(np.abs(n[:, 0:1]) > 0.9, [[0.0, 1.0, 0.0]], [[1.0, 0.0, 0.0]])
    t = np.cross(helper, n)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(n, t)
    d = t * lx[:, None] + b * ly[:, None] + n * lz[:, None]
    return pack_rays(p, d, offset_tmin(p), tmax)


def point_light_rays(points: np.ndarray, normals: np.ndarray, count: int, n_lights: int, half: float,
                     stream: Stream) -> np.ndarray:
    """Config 3 shadow rays: from the given hit points taken in turn toward one of n_lights point
    lights uniform in [-half, half]^3 (chosen uniformly), tmax = distance * (1 - 1e-4)."""
    lights = stream.range(-half, half, n_lights, 3)
    k = np.arange(count) % len(points)
    p = points[k].astype(np.float64)
    which = np.minimum((stream.uniform(count) * n_lights).astype(np.int64), n_lights - 1)
    v = lights[which] - p
    dist = np.maximum(np.linalg.norm(v, axis=1), 1e-30)
    return pack_rays(p, v / dist[:, None], offset_tmin(p), dist * (1.0 - 1e-4))


def hit_points(rays: np.ndarray, t: np.ndarray) -> np.ndarray:
    return (rays[:, 0:3].astype(np.float64) + rays[:, 4:7].astype(np.float64) * t[:, None].astype(np.float64))


def triangle_normals(mesh: Mesh, prim: np.ndarray) -> np.ndarray:
    tri = mesh.indices.reshape(-1, 3)[prim]
    a, b, c = (mesh.positions[tri[:, k]].astype(np.float64) for k in range(3))
    return np.cross(b - a, c - a)
