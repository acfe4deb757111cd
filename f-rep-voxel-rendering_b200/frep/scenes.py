"""Seeded synthetic scenes for the voxelize + render workloads, and the
reference's demo shapes (vulkan/src/shapes.cpp) restated with frep.csg.

The reference ships no dataset or benchmark scenes; these generators build the
workloads from the library's csg primitives (squared-distance spheres and
slab boxes as in vulkan/src/csg/lib.cpp:117-148):

* ``spheres_union``   — min-union of n random spheres (the small plain config)
* ``random_csg``      — n random spheres / boxes / capsules combined by a random
                        binary tree of min, max, max(a, -b) and polynomial
                        smooth-min (the large single-scene config)
* ``gyroid_stress``   — twisted gyroid lattice clipped to a box and smooth-
                        unioned with spheres (the stress config)
* ``animated_csg``    — random_csg plus spheres orbiting with T (a static part
                        and a moving part, for re-voxelization with reuse)

Every scene also carries its grid and camera so that a workload is one object.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import csg
from .csg import (Abs, Axes, Box, Cos, Diff, Dist2, Dot, Empty, Exp, Intersect, Max, Min, Norm2, Pow,
                  RotateX, RotateY, RotateZ, ScaleX, ScaleXYZ, Sin, Sphere, Sqrt, Square, T,
                  TranslateX, TranslateXYZ, TranslateY, Union, Vector3, X, Y, Z, f32)


@dataclass
class Scene:
    name: str
    shape: csg.Expr
    grid_dims: list
    low_vertex: tuple
    world_size: float
    camera: "object" = None
    width: int = 256
    height: int = 256
    shadow_mask: int = 0
    meta: dict = field(default_factory=dict)


# ---- primitives beyond lib.cpp -------------------------------------------------

def capsule(a, b, radius) -> csg.Expr:
    """Squared distance to the segment [a, b] minus radius^2; the segment
    parameter is clamped to [0, 1] with Min/Max."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ba = b - a
    inv_len2 = f32(1.0 / float(np.dot(ba.astype(np.float64), ba.astype(np.float64))))
    p = Axes()
    pa = Vector3(p.x - float(a[0]), p.y - float(a[1]), p.z - float(a[2]))
    t = Dot(pa, Vector3(float(ba[0]), float(ba[1]), float(ba[2]))) * inv_len2
    t = Max(Min(t, 1.0), 0.0)
    q = Vector3(float(a[0]) + t * float(ba[0]), float(a[1]) + t * float(ba[1]), float(a[2]) + t * float(ba[2]))
    return Dist2(Axes(), q) - f32(float(radius) ** 2)


def smooth_min(a, b, k: float) -> csg.Expr:
    """Polynomial smooth minimum: h = max(k - |a - b|, 0) / k;
    min(a, b) - h*h*k/4 (|x| = Sqrt(x*x) as in lib.cpp:68-71)."""
    h = Max(k - Abs(a - b), 0.0) / k
    return Min(a, b) - h * h * f32(k / 4.0)


# ---- workloads -----------------------------------------------------------------

def spheres_union(n: int = 16, seed: int = 1, width: int = 256, height: int = 256) -> Scene:
    """Min-union of n spheres, centres U[-1,1]^3, radii U[0.1,0.3]; grid
    {16, 4} (64^3) over [-1.5, 1.5]^3; orthographic camera looking down +z."""
    from . import Camera
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    radii = rng.uniform(0.1, 0.3, n).astype(np.float32)
    shape = None
    for c, r in zip(centers, radii):
        s = Sphere(Vector3(float(c[0]), float(c[1]), float(c[2])), float(r))
        shape = s if shape is None else Union(shape, s)
    cam = Camera(position=(0.0, 0.0, -3.0), forward=(0.0, 0.0, 1.0), initial_up=(0.0, 1.0, 0.0),
                 orthographic=True, ortho_width=3.0)
    return Scene("spheres_union", shape, [16, 4], (-1.5, -1.5, -1.5), 3.0, cam, width, height,
                 meta={"n": n, "seed": seed})


def _primitive(rng, kind: int, center, size) -> csg.Expr:
    cx, cy, cz = (float(v) for v in center)
    if kind == 0:
        return Sphere(Vector3(cx, cy, cz), float(size[0]))
    if kind == 1:
        hx, hy, hz = (float(v) for v in size)
        return Box(Vector3(cx - hx, cy - hy, cz - hz), Vector3(2 * hx, 2 * hy, 2 * hz))
    axis = rng.normal(size=3)
    axis = axis / np.linalg.norm(axis)
    half = float(size[1])
    a = np.array([cx, cy, cz]) - half * axis
    b = np.array([cx, cy, cz]) + half * axis
    return capsule(a, b, float(size[0]))


def random_csg(n: int = 256, seed: int = 2, grid_dims=(16, 16, 8), width: int = 1920,
               height: int = 1080, shadows: bool = True) -> Scene:
    """n primitives (sphere, axis-aligned box or capsule, uniformly), size
    parameters U[0.02, 0.2], centres U[-1, 1]^3, combined by a random binary
    tree. The tree pairs spatial neighbours (recursive split at a random axis'
    median) so that intersections and subtractions act on nearby shapes; node
    operators are min 45%, smooth-min (k ~ U[0.01, 0.1]) 35%, max(a, -b) 15%,
    max 5%. Perspective camera, 60 degrees, shadow ray toward light 0."""
    from . import Camera
    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, 3, n)
    centers = rng.uniform(-1.0, 1.0, (n, 3))
    sizes = rng.uniform(0.02, 0.2, (n, 3))
    prims = [_primitive(rng, int(k), c, s) for k, c, s in zip(kinds, centers, sizes)]

    def build(idx):
        if len(idx) == 1:
            return prims[idx[0]]
        axis = int(rng.integers(0, 3))
        order = idx[np.argsort(centers[idx, axis], kind="stable")]
        half = len(order) // 2
        a, b = build(order[:half]), build(order[half:])
        u = rng.random()
        if u < 0.45:
            return Min(a, b)
        if u < 0.80:
            return smooth_min(a, b, float(rng.uniform(0.01, 0.1)))
        if u < 0.95:
            return Max(a, -b)
        return Max(a, b)

    shape = build(np.arange(n))
    cam = Camera(position=(2.2, 1.6, 2.8), forward=(-2.2, -1.6, -2.8), initial_up=(0.0, 1.0, 0.0),
                 fov_deg=60.0)
    return Scene("random_csg", shape, list(grid_dims), (-1.25, -1.25, -1.25), 2.5, cam, width, height,
                 shadow_mask=1 if shadows else 0, meta={"n": n, "seed": seed})


def animated_csg(n: int = 256, n_moving: int = 4, seed: int = 2, grid_dims=(16, 16, 8), width: int = 1920,
                 height: int = 1080, shadows: bool = True) -> Scene:
    """A scene with a static part and a moving part: random_csg(n, seed) (the
    static part) min-unioned with n_moving spheres (radii U[0.08, 0.15]) that
    orbit the z axis, sphere i on a circle of radius U[0.4, 1.0] at height
    U[-0.6, 0.6], at angle 2 pi T + phase_i (one revolution per unit of T).
    At a given T only the cells near a sphere keep it in their shortened tape;
    every other cell's tape is the static part's, independent of T."""
    base = random_csg(n, seed, grid_dims, width, height, shadows)
    rng = np.random.default_rng(seed + 7919)
    shape = base.shape
    for _ in range(n_moving):
        r, z0 = float(rng.uniform(0.4, 1.0)), float(rng.uniform(-0.6, 0.6))
        phase, rad = float(rng.uniform(0.0, 2.0 * np.pi)), float(rng.uniform(0.08, 0.15))
        ang = f32(2.0 * np.pi) * T() + f32(phase)
        ball = Sqrt(Square(X() - f32(r) * Cos(ang)) + Square(Y() - f32(r) * Sin(ang)) + Square(Z() - z0)) - rad
        shape = Min(shape, ball)
    base.name = "animated_csg"
    base.shape = shape
    base.meta = {"n": n, "n_moving": n_moving, "seed": seed}
    return base


# ---- the reference's demo shapes (vulkan/src/shapes.cpp:5-117) ---------------------

def Screw():
    shape = Box((-15, -2, -2), (30, 4, 4))
    shape = RotateX(shape, X())
    scale = 2 * Exp(X() / 40)
    shape = ScaleXYZ(shape, Vector3(1, scale, scale))
    shape = RotateZ(shape, T() / 2)
    shape = RotateY(shape, T() / 5)
    return shape


def ElasticCube():
    shape = Box((-10, -10, -10), (20, 20, 20))
    scale = 1 / (1 + Pow(Y() / 5, 4))
    shape = ScaleX(shape, scale)
    shape = ScaleX(shape, 1 + 0.2 * Sin(Z() + 10 * T()))
    radius = (1 + 0.1 * Sin(T())) * 10
    shape = Diff(shape, Sphere((0, 0, 0), radius))
    shape = RotateY(shape, T() / 5)
    return shape


def TangleCube():
    shape = Norm2(Axes() * Axes()) - 8 * Norm2(Axes()) + 25
    return ScaleXYZ(shape, 4)


def Morph():
    shape1 = Norm2(Axes() * Axes()) - 8 * Norm2(Axes()) + 25
    shape1 = ScaleXYZ(shape1, 4)
    shape2 = Sphere((0, 0, 0), 10)
    blend = (1 + Sin(T())) / 2
    shape = blend * shape1 + (1 - blend) * shape2
    return RotateY(shape, T() / 5)


def Menger(level: int):
    if level <= 0:
        return Box((0, 0, 0), (1, 1, 1))
    third = float(np.float32(1) / np.float32(3))
    block = ScaleXYZ(Menger(level - 1), Vector3(third, third, 1))
    menger = Empty()
    for x in range(3):
        for y in range(3):
            if not (x == 1 and y == 1):
                tb = TranslateXYZ(block, Vector3(float(np.float32(x) / np.float32(3)),
                                                 float(np.float32(y) / np.float32(3)), 0))
                menger = Union(menger, tb)
    return menger


def MengerSponge(level: int):
    shape = Menger(level)
    shape = TranslateXYZ(shape, Vector3(-0.5, -0.5, -0.5))
    shape = ScaleXYZ(shape, Vector3(30, 30, 10))
    return Diff(shape, Sphere((10, 10, 0), 10))


def TwistedTower(level: int, angle: float = 0.3, scale: float = 0.8):
    box = Box((-0.5, 0, -0.5), (1, 1, 1))
    if level <= 0:
        return box
    shape = TwistedTower(level - 1, angle, scale)
    shape = ScaleXYZ(shape, scale)
    shape = RotateY(shape, angle)
    shape = TranslateY(shape, scale)
    return Union(shape, box)


def OrganicBalls():
    s1 = Sphere((10, 0, 0), 8)
    s1 = TranslateX(s1, 5 * Sin(T()))
    s2 = Sphere((-10, 0, 0), 10)
    f = Min(Min(X(), Y()), Sqrt(X() * Y()) - 40)
    return f(s1, s2, Z(), T())


DEMO_SHAPES = {
    "Screw": lambda level: Screw(),
    "ElasticCube": lambda level: ElasticCube(),
    "TangleCube": lambda level: TangleCube(),
    "Morph": lambda level: Morph(),
    "MengerSponge": MengerSponge,
    "TwistedTower": TwistedTower,
    "OrganicBalls": lambda level: OrganicBalls(),
}


# ---- batching / serving workload --------------------------------------------------

BATCH_RESOLUTIONS = (64, 128, 256, 512, 1024)

# Branching per effective resolution when no tuned choice is given: 16 at the
# root, then the largest factors that leave a last level of at least 4.
DEFAULT_BRANCHING = {64: (16, 4), 128: (16, 8), 256: (16, 16), 512: (16, 8, 4), 1024: (16, 16, 4)}


def orbit_camera(rng, distance: float = 4.1, fov_deg: float = 60.0):
    """A perspective camera on a sphere around the origin, looking at it, at a
    random azimuth and an elevation in [-0.35, 1.0] rad."""
    from . import Camera
    az = float(rng.uniform(0.0, 2.0 * np.pi))
    el = float(rng.uniform(-0.35, 1.0))
    pos = (distance * np.cos(el) * np.cos(az), distance * np.sin(el), distance * np.cos(el) * np.sin(az))
    return Camera(position=pos, forward=tuple(-v for v in pos), initial_up=(0.0, 1.0, 0.0), fov_deg=fov_deg)


def _batch_scene(job):
    """One scene of batch_workload, its shape flattened to DAG arrays so that
    it crosses a process boundary."""
    i, seed, count, res, dims, width, height, shadows = job
    sc = random_csg(count, seed=seed, grid_dims=dims, width=width, height=height, shadows=shadows)
    sc.name = "batch"
    sc.meta.update(index=i, res=res)
    sc.shape = sc.shape.flatten()
    return sc


def batch_jobs(n_scenes: int = 512, seed: int = 3, width: int = 512, height: int = 512, shadows: bool = True,
               branching: dict | None = None, min_prims: int = 4, max_prims: int = 1024) -> list:
    """The scene descriptions of batch_workload without building them: one
    tuple (index, seed, primitive count, resolution, grid dims, width,
    height, shadows) per scene; batch_scene(job) builds one."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(min_prims), np.log(max_prims), n_scenes))
    counts = np.clip(np.round(counts), min_prims, max_prims).astype(int)
    res = rng.choice(np.array(BATCH_RESOLUTIONS), n_scenes)
    br = dict(DEFAULT_BRANCHING)
    br.update(branching or {})
    return [(i, seed * 1_000_003 + i, int(counts[i]), int(res[i]), tuple(br[int(res[i])]), width, height, shadows)
            for i in range(n_scenes)]


def batch_scene(job):
    """One scene of batch_workload from its batch_jobs entry, its shape a
    compiled frep.Tape."""
    from . import Tape
    sc = _batch_scene(job)
    sc.shape = Tape.from_dag(*sc.shape)
    return sc


def batch_workload(n_scenes: int = 512, seed: int = 3, width: int = 512, height: int = 512,
                   shadows: bool = True, branching: dict | None = None, min_prims: int = 4,
                   max_prims: int = 1024, processes: int = 0) -> list:
    """Independent scenes as in random_csg with primitive counts log-uniform in
    [min_prims, max_prims] and effective resolutions drawn uniformly from
    BATCH_RESOLUTIONS. `branching` maps an effective resolution to grid dims
    (default DEFAULT_BRANCHING). Scene i's meta holds its index, primitive
    count and resolution; its shape is a compiled frep.Tape. `processes` > 1
    builds the expressions in that many spawned worker processes (expression
    building is Python-bound: about 0.25 ms per primitive)."""
    from . import Tape
    jobs = batch_jobs(n_scenes, seed, width, height, shadows, branching, min_prims, max_prims)
    if processes > 1 and n_scenes > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pool:
            out = pool.map(_batch_scene, jobs, chunksize=max(1, n_scenes // (4 * processes)))
    else:
        out = [_batch_scene(j) for j in jobs]
    for sc in out:
        sc.shape = Tape.from_dag(*sc.shape)
    return out


def jitter_tape(wide: np.ndarray, rng, rel: float = 0.1):
    """A new scene of the same structure: the wide tape `wide` with every
    constant (centres, sizes, blend radii) scaled by U[1 - rel, 1 + rel].
    Returns a compiled frep.Tape. Used to draw many distinct scenes of the
    batching distribution without building their expressions again."""
    from . import Tape
    w = np.array(wide, dtype=np.uint64, copy=True)
    is_const = (w & np.uint64(0xFF)) == np.uint64(0)
    bits = (w[is_const] >> np.uint64(32)).astype(np.uint32)
    vals = bits.view(np.float32) * rng.uniform(1.0 - rel, 1.0 + rel, bits.size).astype(np.float32)
    w[is_const] = (w[is_const] & np.uint64(0xFFFFFFFF)) | (vals.view(np.uint32).astype(np.uint64) << np.uint64(32))
    return Tape.from_wide(w)


# ---- stress workload ---------------------------------------------------------------

def stress_gyroid(n_spheres: int = 64, seed: int = 5, period: float = 0.05, thickness: float = 0.3,
                  grid_dims=(16, 16, 4, 4), width: int = 1920, height: int = 1080) -> Scene:
    """A gyroid lattice sin(kx)cos(ky) + sin(ky)cos(kz) + sin(kz)cos(kx),
    k = 2 pi / period, as a sheet |g| - thickness, domain-warped by a z-twist
    (x, y rotated about z by 2 pi T z: T in [0, 1) sweeps the twist through
    one full turn per unit of z), intersected (max) with the box [-1, 1]^3 and
    smooth-unioned (k = 0.05) with n_spheres random spheres (centres U[-1.2,
    1.2]^3, radii U[0.05, 0.2]). Default grid {16, 16, 4, 4} = 4096^3 over
    [-1.3, 1.3]^3; perspective camera at 60 degrees with a shadow ray per
    hit. Animated: re-voxelize per frame at T = frame / frames."""
    from . import Camera
    rng = np.random.default_rng(seed)
    k = 2.0 * np.pi / period
    ang = f32(2.0 * np.pi) * T() * Z()
    c, s = Cos(ang), Sin(ang)
    xt = c * X() - s * Y()
    yt = s * X() + c * Y()
    kx, ky, kz = f32(k) * xt, f32(k) * yt, f32(k) * Z()
    g = Sin(kx) * Cos(ky) + Sin(ky) * Cos(kz) + Sin(kz) * Cos(kx)
    sheet = (Abs(g) - f32(thickness)) / f32(k)
    box = Max(Max(Abs(X()), Abs(Y())), Abs(Z())) - 1.0
    shape = Max(sheet, box)
    centers = rng.uniform(-1.2, 1.2, (n_spheres, 3))
    radii = rng.uniform(0.05, 0.2, n_spheres)
    balls = [Sqrt(Dist2(Axes(), Vector3(*map(float, cc)))) - float(r) for cc, r in zip(centers, radii)]
    while len(balls) > 1:  # balanced smooth-union tree
        nxt = [smooth_min(balls[i], balls[i + 1], 0.05) for i in range(0, len(balls) - 1, 2)]
        if len(balls) % 2:
            nxt.append(balls[-1])
        balls = nxt
    shape = smooth_min(shape, balls[0], 0.05)
    cam = Camera(position=(2.4, 1.7, 3.0), forward=(-2.4, -1.7, -3.0), initial_up=(0.0, 1.0, 0.0), fov_deg=60.0)
    return Scene("stress_gyroid", shape, list(grid_dims), (-1.3, -1.3, -1.3), 2.6, cam, width, height,
                 shadow_mask=1, meta={"n_spheres": n_spheres, "seed": seed, "period": period})
