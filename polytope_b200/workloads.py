"""Synthetic workloads (seeded, deterministic) used by the tests and the bench.

* :func:`small_scene`   -- ground quad + icosphere-5 + quad area light, 320x240, 8 spp, depth 4
* :func:`microbench`    -- displaced icosphere-8 (1,310,720 faces) + 16,777,216 rays
* :func:`instanced_scene` -- the displaced sphere instanced 5x with seeded rigid transforms
  (Lambert or mirror), ground, 3x3 quad light, constant environment 0.2; 1920x1080, 64 spp, depth 8

Emission and environment radiance are multiplied by 255 as the reference's PBRT parser does for
``AreaLightSource "diffuse" "L"`` and ``LightSource "infinite" "L"`` (pbrt_parser.cpp:1270-1287,
1331-1348).
"""
from __future__ import annotations

import numpy as np

from . import MAT_LAMBERT, MAT_MIRROR, Mesh, icosphere, microbench_rays

SMALL_CAMERA = dict(eye=(0.0, 1.5, 5.0), look_at=(0.0, 1.0, 0.0), up=(0.0, 1.0, 0.0), fov=45.0)
INSTANCED_CAMERA = dict(eye=(0.0, 4.0, 14.0), look_at=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov=45.0)


def translate(tx, ty, tz) -> np.ndarray:
    m = np.eye(4, dtype=np.float32)
    m[:3, 3] = (tx, ty, tz)
    return m


def quad(y: float, half: float, material=MAT_LAMBERT, albedo=(0.7, 0.7, 0.7), is_light=False, emission=(0, 0, 0)) -> Mesh:
    """Axis-aligned square of side 2*half in the plane y, as two triangles."""
    x = np.array([-half, half, half, -half], np.float32)
    z = np.array([-half, -half, half, half], np.float32)
    yy = np.full(4, y, np.float32)
    return Mesh(x, yy, z, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), material=material, albedo=albedo,
                is_light=is_light, emission=emission)


def small_scene(level: int = 5):
    """Ground 20x20 at y=0 + icosphere (radius 1, centre y=1) Lambert 0.7, 2x2 light at y=4, L=10."""
    x, y, z, f = icosphere(level, 1.0, 0.0, 0)
    ground = quad(0.0, 10.0)
    sphere = Mesh(x, y, z, f, object_to_world=translate(0, 1, 0), albedo=(0.7, 0.7, 0.7))
    light = quad(4.0, 1.0, is_light=True, emission=(10 * 255.0,) * 3)
    return [ground, sphere, light], None


SMALL_RENDER = dict(width=320, height=240, spp=8, max_depth=4, seed=1, camera=SMALL_CAMERA)


def microbench(n_rays: int = 16_777_216, level: int = 8, seed_mesh: int = 7, seed_rays: int = 11):
    """(meshes, rays): displaced icosphere (amplitude 0.05) and the half closest / half any-hit rays."""
    x, y, z, f = icosphere(level, 1.0, 0.05, seed_mesh)
    return [Mesh(x, y, z, f)], microbench_rays(n_rays, 3.0, seed_rays)


def _rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def instanced_scene(level: int = 8, instances: int = 5, seed: int = 3, noise_seed: int = 7):
    """The displaced sphere instanced with seeded rigid transforms over a ground quad, a 3x3 light
    and a constant environment 0.2.  Returns (meshes, env)."""
    x, y, z, f = displaced_sphere(level, noise_seed)
    rng = np.random.default_rng(seed)
    meshes = [quad(0.0, 20.0)]
    for _ in range(instances):
        R = _rotation(rng)
        t = rng.uniform(-4.0, 4.0, 3)
        s = rng.uniform(0.5, 1.5)
        M = np.eye(4)
        M[:3, :3] = R * s
        M[:3, 3] = t
        inv = np.linalg.inv(M)
        if rng.uniform() < 0.5:
            mat, alb = MAT_MIRROR, (1.0, 1.0, 1.0)
        else:
            mat, alb = MAT_LAMBERT, tuple(rng.uniform(0.2, 0.9, 3))
        meshes.append(Mesh(x, y, z, f, object_to_world=M.astype(np.float32), world_to_object=inv.astype(np.float32),
                           material=mat, albedo=alb))
    meshes.append(quad(8.0, 1.5, is_light=True, emission=(10 * 255.0,) * 3))
    return meshes, (0.2 * 255.0,) * 3


INSTANCED_RENDER = dict(width=1920, height=1080, spp=64, max_depth=8, seed=1, camera=INSTANCED_CAMERA)


# ---- many scenes: batched renders and the serving pool ---------------------------------------

def boxes(n: int, rng, lo: float = -3.0, hi: float = 3.0, size=(0.05, 0.5)):
    """n random axis-aligned boxes, 12 triangles each: packed (x, y, z, faces)."""
    c = rng.uniform(lo, hi, (n, 3))
    h = rng.uniform(size[0], size[1], (n, 3)) * 0.5
    corners = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                        [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)
    quads = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (3, 2, 6, 7), (0, 3, 7, 4), (1, 5, 6, 2)]
    tri = np.array([[q[0], q[1], q[2]] for q in quads] + [[q[0], q[2], q[3]] for q in quads], np.uint32)
    v = (c[:, None, :] + h[:, None, :] * corners[None, :, :]).reshape(-1, 3).astype(np.float32)
    f = (tri[None, :, :] + 8 * np.arange(n, dtype=np.uint32)[:, None, None]).reshape(-1, 3)
    return v[:, 0], v[:, 1], v[:, 2], f


_ICO_CACHE = {}


def displaced_sphere(level: int, seed: int = 7):
    key = (level, seed)
    if key not in _ICO_CACHE:
        _ICO_CACHE[key] = icosphere(level, 1.0, 0.05, seed)
    return _ICO_CACHE[key]


def batch_scene(total_tris: int, rng, noise_seed: int = 7):
    """A displaced icosphere plus seeded boxes (12 triangles each) totalling about total_tris,
    Lambert albedo uniform in [0.2, 0.9]^3, a 2x2 quad light and a dim constant environment."""
    level = 2
    while 20 * 4 ** (level + 1) <= max(320, total_tris // 2) and level < 8:
        level += 1
    x, y, z, f = displaced_sphere(level, noise_seed)
    meshes = [Mesh(x, y, z, f, albedo=tuple(rng.uniform(0.2, 0.9, 3)))]
    nb = max(0, (total_tris - len(f)) // 12)
    if nb:
        bx, by, bz, bf = boxes(nb, rng)
        meshes.append(Mesh(bx, by, bz, bf, albedo=tuple(rng.uniform(0.2, 0.9, 3))))
    meshes.append(quad(4.0, 1.0, is_light=True, emission=(10 * 255.0,) * 3))
    return meshes, (0.2 * 255.0,) * 3


BATCH_CAMERA = dict(eye=(0.0, 1.0, 7.0), look_at=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov=50.0)


def batched_workload(n_scenes: int = 256, seed: int = 23, min_tris: int = 1000, max_tris: int = 500_000,
                     resolutions=(64, 128, 256, 512), spps=(4, 16, 64), max_depth: int = 6):
    """Uneven scenes: triangle counts log-uniform in [min_tris, max_tris], resolution and spp drawn
    per scene.  Returns a list of (meshes, env, render dict)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        tris = int(np.exp(rng.uniform(np.log(min_tris), np.log(max_tris))))
        meshes, env = batch_scene(tris, rng)
        res = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        out.append((meshes, env, dict(width=res, height=res, spp=spp, max_depth=max_depth, seed=k + 1,
                                      camera=BATCH_CAMERA)))
    return out


def serving_pool(n_scenes: int = 32, seed: int = 19, min_tris: int = 100_000, max_tris: int = 4_000_000):
    """Resident scenes built like the instanced scene: the displaced sphere instanced with seeded
    rigid transforms (Lambert or mirror) over a ground quad, a 3x3 light and environment 0.2;
    triangle counts log-uniform in [min_tris, max_tris]."""
    rng = np.random.default_rng(seed)
    pool = []
    for _ in range(n_scenes):
        tris = int(np.exp(rng.uniform(np.log(min_tris), np.log(max_tris))))
        level = 6 if tris < 400_000 else (7 if tris < 1_500_000 else 8)
        per = 20 * 4 ** level
        k = int(np.clip(round(tris / per), 1, 12))
        meshes, env = instanced_scene(level=level, instances=k, seed=int(rng.integers(1 << 30)))
        pool.append((meshes, env))
    return pool


SERVE_CAMERA = INSTANCED_CAMERA
