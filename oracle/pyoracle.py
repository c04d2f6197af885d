"""ctypes bindings for the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg.  Two libraries are wrapped:

* ``oracle/liboracle.so``        -- the CPU restatement of the reference path (oracle.cpp)
* ``oracle/_ref/libpolyref.so``  -- the reference's own sources compiled by oracle/Makefile

Both take the same mesh descriptor layout as the product's ``pt_mesh_desc``.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpolyref.so")

PRIM_NONE = 0xFFFFFFFF

RAY_DTYPE = np.dtype([("org", "<f4", 3), ("tmax", "<f4"), ("dir", "<f4", 3), ("flags", "<u4")])
HIT_DTYPE = np.dtype([("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
NODE_DTYPE = np.dtype([("bb", "<f4", 6), ("offset", "<u4"), ("num_faces", "<u2"), ("axis", "<u2")])

_fp = C.POINTER(C.c_float)
_up = C.POINTER(C.c_uint32)


class MeshDesc(C.Structure):
    _fields_ = [
        ("x", _fp), ("y", _fp), ("z", _fp), ("num_vertices", C.c_uint32),
        ("fv0", _up), ("fv1", _up), ("fv2", _up), ("num_faces", C.c_uint32),
        ("nx", _fp), ("ny", _fp), ("nz", _fp),
        ("object_to_world", C.c_float * 16), ("world_to_object", C.c_float * 16),
        ("material", C.c_uint32), ("albedo", C.c_float * 3),
        ("is_light", C.c_int32), ("emission", C.c_float * 3),
    ]


class RenderDesc(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_depth", C.c_uint32),
        ("seed", C.c_uint64), ("flags", C.c_uint32),
        ("eye", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3), ("fov", C.c_float),
    ]


def _f(a):
    return a.ctypes.data_as(_fp) if a is not None else None


def _u(a):
    return a.ctypes.data_as(_up) if a is not None else None


def mesh_descs(meshes: Sequence) -> tuple:
    """Build a ctypes array of MeshDesc from objects with the attributes of
    ``polytope_b200.Mesh`` (x, y, z, faces, object_to_world, world_to_object, material, albedo,
    is_light, emission, normals).  Returns (array, keepalive)."""
    arr = (MeshDesc * len(meshes))()
    keep = []
    for i, m in enumerate(meshes):
        x = np.ascontiguousarray(m.x, np.float32)
        y = np.ascontiguousarray(m.y, np.float32)
        z = np.ascontiguousarray(m.z, np.float32)
        f = np.ascontiguousarray(m.faces, np.uint32)
        f0, f1, f2 = (np.ascontiguousarray(f[:, k]) for k in range(3))
        keep += [x, y, z, f0, f1, f2]
        d = arr[i]
        d.x, d.y, d.z, d.num_vertices = _f(x), _f(y), _f(z), len(x)
        d.fv0, d.fv1, d.fv2, d.num_faces = _u(f0), _u(f1), _u(f2), len(f0)
        if getattr(m, "normals", None) is not None:
            n = np.ascontiguousarray(m.normals, np.float32)
            nx, ny, nz = (np.ascontiguousarray(n[:, k]) for k in range(3))
            keep += [nx, ny, nz]
            d.nx, d.ny, d.nz = _f(nx), _f(ny), _f(nz)
        d.object_to_world[:] = [float(v) for v in np.asarray(m.object_to_world, np.float32).ravel()]
        d.world_to_object[:] = [float(v) for v in np.asarray(m.world_to_object, np.float32).ravel()]
        d.material = int(m.material)
        d.albedo[:] = [float(v) for v in m.albedo]
        d.is_light = int(bool(m.is_light))
        d.emission[:] = [float(v) for v in m.emission]
    return arr, keep


def _load(path: str, prefix: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
    lib = C.CDLL(path)
    vp = C.c_void_p
    getattr(lib, f"{prefix}_scene_create").restype = vp
    getattr(lib, f"{prefix}_scene_create").argtypes = [C.POINTER(MeshDesc), C.c_uint32, C.c_int, _fp]
    getattr(lib, f"{prefix}_scene_destroy").argtypes = [vp]
    getattr(lib, f"{prefix}_num_nodes").restype = C.c_uint32
    getattr(lib, f"{prefix}_num_nodes").argtypes = [vp]
    getattr(lib, f"{prefix}_get_tree").argtypes = [vp, vp, _up]
    getattr(lib, f"{prefix}_trace").argtypes = [vp, vp, C.c_uint64, vp, _up, _up, C.c_int]
    getattr(lib, f"{prefix}_hit_frames").argtypes = [vp, vp, C.c_uint64, _fp]
    getattr(lib, f"{prefix}_render_rows").argtypes = [vp, C.POINTER(RenderDesc), C.c_uint32, C.c_uint32, _fp, _up, C.c_int]
    getattr(lib, f"{prefix}_bbox_hits").argtypes = [_fp, _fp, _fp, C.c_float]
    getattr(lib, f"{prefix}_bbox_hits").restype = C.c_int
    return lib


_oracle_lib: Optional[C.CDLL] = None
_ref_lib: Optional[C.CDLL] = None


def oracle_lib() -> C.CDLL:
    global _oracle_lib
    if _oracle_lib is None:
        lib = _load(ORACLE_SO, "orc")
        lib.orc_num_prims.restype = C.c_uint32
        lib.orc_num_prims.argtypes = [C.c_void_p]
        lib.orc_get_world.argtypes = [C.c_void_p, _fp]
        lib.orc_camera_rays.argtypes = [_fp, _fp, _fp, C.c_float, C.c_uint32, C.c_uint32, C.c_void_p]
        lib.orc_f64_diff.restype = C.c_float
        lib.orc_f64_diff.argtypes = [C.c_float] * 4
        lib.orc_sincos_2pi.argtypes = [C.c_float, _fp, _fp]
        lib.orc_philox.argtypes = [_up, C.c_uint64]
        lib.orc_wald.argtypes = [_fp, _fp, _fp, C.c_float, _fp]
        lib.orc_wald.restype = C.c_int
        lib.orc_gamma.argtypes = [C.c_int]
        lib.orc_gamma.restype = C.c_float
        lib.orc_apply_point.argtypes = [_fp, _fp]
        lib.orc_compact_shape.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_uint32, _up]
        lib.orc_world_to_local.argtypes = [_fp, _fp, _fp, _fp, _fp]
        lib.orc_mirror_sample.argtypes = [_fp, _fp]
        lib.orc_normalize.argtypes = [_fp]
        lib.orc_film_to_rgba8.argtypes = [_fp, C.c_uint32, C.c_void_p]
        _oracle_lib = lib
    return _oracle_lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> C.CDLL:
    global _ref_lib
    if _ref_lib is None:
        lib = _load(REF_SO, "ref")
        lib.ref_camera_rays.argtypes = [C.POINTER(RenderDesc), C.c_void_p]
        _ref_lib = lib
    return _ref_lib


class _Scene:
    prefix = ""

    def __init__(self, meshes, env=None):
        self.lib = self._lib()
        arr, self._keep = mesh_descs(meshes)
        envp = None
        if env is not None:
            self._env = np.asarray(env, np.float32)
            envp = _f(self._env)
        self.h = getattr(self.lib, f"{self.prefix}_scene_create")(arr, len(meshes), int(env is not None), envp)
        self.num_faces = int(sum(len(m.faces) for m in meshes))

    def _lib(self):
        raise NotImplementedError

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, f"{self.prefix}_scene_destroy")(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def tree(self):
        n = getattr(self.lib, f"{self.prefix}_num_nodes")(self.h)
        nodes = np.zeros(n, NODE_DTYPE)
        pairs = np.zeros((self.num_faces, 2), np.uint32)
        getattr(self.lib, f"{self.prefix}_get_tree")(self.h, nodes.ctypes.data, _u(pairs))
        return nodes, pairs

    def trace(self, rays: np.ndarray, threads: int = 0, counts: bool = False):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(len(rays), HIT_DTYPE)
        nt = np.zeros(len(rays), np.uint32) if counts else None
        tt = np.zeros(len(rays), np.uint32) if counts else None
        getattr(self.lib, f"{self.prefix}_trace")(self.h, rays.ctypes.data, len(rays), hits.ctypes.data,
                                                   _u(nt), _u(tt), threads)
        return (hits, nt, tt) if counts else hits

    def hit_frames(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros((len(rays), 12), np.float32)
        getattr(self.lib, f"{self.prefix}_hit_frames")(self.h, rays.ctypes.data, len(rays), _f(out))
        return out

    def render(self, desc: dict, rows: Optional[tuple] = None, threads: int = 0):
        rd = render_desc(desc)
        w, h = rd.width, rd.height
        rgb = np.zeros((h, w, 3), np.float32)
        prim = np.full((h, w), PRIM_NONE, np.uint32)
        r0, r1 = rows if rows is not None else (0, h)
        getattr(self.lib, f"{self.prefix}_render_rows")(self.h, C.byref(rd), r0, r1, _f(rgb), _u(prim), threads)
        return rgb, prim


class OracleScene(_Scene):
    """The CPU restatement (oracle.cpp)."""
    prefix = "orc"

    def _lib(self):
        return oracle_lib()

    def world_triangles(self):
        out = np.zeros((self.num_faces, 3, 3), np.float32)
        self.lib.orc_get_world(self.h, _f(out))
        return out


class RefScene(_Scene):
    """The reference's own code (oracle/_ref/libpolyref.so)."""
    prefix = "ref"

    def _lib(self):
        return ref_lib()


def render_desc(d: dict) -> RenderDesc:
    rd = RenderDesc()
    rd.width, rd.height = d["width"], d["height"]
    rd.spp, rd.max_depth = d["spp"], d["max_depth"]
    rd.seed = d.get("seed", 1)
    rd.flags = d.get("flags", 0)
    cam = d["camera"]
    rd.eye[:] = cam["eye"]
    rd.look_at[:] = cam["look_at"]
    rd.up[:] = cam["up"]
    rd.fov = cam["fov"]
    return rd


def camera_rays_oracle(desc: dict) -> np.ndarray:
    cam = desc["camera"]
    e, l, u = (np.asarray(cam[k], np.float32) for k in ("eye", "look_at", "up"))
    out = np.zeros(desc["width"] * desc["height"], RAY_DTYPE)
    oracle_lib().orc_camera_rays(_f(e), _f(l), _f(u), cam["fov"], desc["width"], desc["height"], out.ctypes.data)
    return out


def camera_rays_ref(desc: dict) -> np.ndarray:
    rd = render_desc(desc)
    out = np.zeros(desc["width"] * desc["height"], RAY_DTYPE)
    ref_lib().ref_camera_rays(C.byref(rd), out.ctypes.data)
    return out


def bbox_hits(lib_name: str, bb, o, d, min_t=float("inf")) -> bool:
    lib = oracle_lib() if lib_name == "orc" else ref_lib()
    a = [np.asarray(v, np.float32) for v in (bb, o, d)]
    return bool(getattr(lib, f"{lib_name}_bbox_hits")(_f(a[0]), _f(a[1]), _f(a[2]), min_t))


def f64_diff(a, b, c, d) -> float:
    return float(oracle_lib().orc_f64_diff(a, b, c, d))


def sincos_2pi(u: float):
    s, c = C.c_float(), C.c_float()
    oracle_lib().orc_sincos_2pi(u, C.byref(s), C.byref(c))
    return s.value, c.value


def philox(counter, seed: int):
    c = np.asarray(counter, np.uint32).copy()
    oracle_lib().orc_philox(_u(c), seed)
    return c


def wald(tri9, o, d, min_t=float("inf")):
    tri = np.asarray(tri9, np.float32).ravel()
    oo, dd = np.asarray(o, np.float32), np.asarray(d, np.float32)
    out = np.zeros(4, np.float32)
    ok = oracle_lib().orc_wald(_f(tri), _f(oo), _f(dd), min_t, _f(out))
    return (bool(ok), out)


def compact_shape(low, high):
    """Compaction of a hand-made tree: returns [(tag, offset)] in DFS order."""
    n = len(low)
    lo = (C.c_int * n)(*low)
    hi = (C.c_int * n)(*high)
    out = np.zeros(2 * n, np.uint32)
    oracle_lib().orc_compact_shape(lo, hi, n, _u(out))
    return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(n)]


def world_to_local(t1, n, t2, w):
    a = [np.asarray(v, np.float32) for v in (t1, n, t2, w)]
    out = np.zeros(3, np.float32)
    oracle_lib().orc_world_to_local(_f(a[0]), _f(a[1]), _f(a[2]), _f(a[3]), _f(out))
    return out


def mirror_sample(v):
    a = np.asarray(v, np.float32)
    out = np.zeros(3, np.float32)
    oracle_lib().orc_mirror_sample(_f(a), _f(out))
    return out


def normalize(v):
    a = np.array(v, np.float32)
    oracle_lib().orc_normalize(_f(a))
    return a


def film_to_rgba8(rgb: np.ndarray) -> np.ndarray:
    """The film as PNGFilm::Output stores it (oracle restatement): (H, W, 4) uint8."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    out = np.zeros((h, w, 4), np.uint8)
    oracle_lib().orc_film_to_rgba8(_f(rgb), h * w, out.ctypes.data)
    return out


def ref_png_film(rgb: np.ndarray, path) -> None:
    """The reference's PNGFilm::Output (oracle/_ref): a float film (H, W, 3) through a BoxFilter of
    one sample per pixel, quantised and encoded with lodepng into `path`."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    f = ref_lib().ref_png_film
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_char_p]
    f.restype = None
    f(rgb.ctypes.data, w, h, os.fsencode(str(path)))


def ref_png_decode(path) -> np.ndarray:
    """A PNG file decoded by the reference's lodepng (oracle/_ref): (H, W, 4) uint8."""
    f = ref_lib().ref_png_decode
    f.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p, C.c_size_t]
    f.restype = C.c_uint
    w, h = C.c_uint32(), C.c_uint32()
    cap = 1 << 26
    buf = np.zeros(cap, np.uint8)
    err = f(os.fsencode(str(path)), C.byref(w), C.byref(h), buf.ctypes.data, cap)
    if err:
        raise ValueError(f"lodepng error {err}")
    return buf[:w.value * h.value * 4].reshape(h.value, w.value, 4).copy()


def ref_load_ply(path: str):
    """The reference's own ply_parser::parse_file (oracle/_ref): (x, y, z, faces, normals or None)."""
    lib = ref_lib()
    f = lib.ref_load_ply
    f.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int)] + [C.c_void_p] * 9
    nv, nf, hn = C.c_uint32(0), C.c_uint32(0), C.c_int(0)
    f(str(path).encode(), C.byref(nv), C.byref(nf), C.byref(hn), *([None] * 9))
    a = [np.zeros(nv.value, np.float32) for _ in range(6)]
    fv = [np.zeros(nf.value, np.uint32) for _ in range(3)]
    f(str(path).encode(), C.byref(nv), C.byref(nf), C.byref(hn), *[v.ctypes.data for v in a + fv])
    normals = np.stack(a[3:], 1) if hn.value else None
    return a[0], a[1], a[2], np.stack(fv, 1), normals


def ref_load_obj(path: str):
    """The reference's own obj_parser::parse_file (oracle/_ref): (x, y, z, faces)."""
    lib = ref_lib()
    f = lib.ref_load_obj
    f.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)] + [C.c_void_p] * 6
    nv, nf = C.c_uint32(0), C.c_uint32(0)
    f(str(path).encode(), C.byref(nv), C.byref(nf), *([None] * 6))
    a = [np.zeros(nv.value, np.float32) for _ in range(3)]
    fv = [np.zeros(nf.value, np.uint32) for _ in range(3)]
    f(str(path).encode(), C.byref(nv), C.byref(nf), *[v.ctypes.data for v in a + fv])
    return a[0], a[1], a[2], np.stack(fv, 1) if nf.value else np.zeros((0, 3), np.uint32)


def ref_load_pbrt(path: str) -> dict:
    """The reference's own pbrt_parser::parse_file (oracle/_ref) on a well-formed file: render
    settings, camera and, per shape, geometry, transforms, material and radiance."""
    lib = ref_lib()
    lib.ref_pbrt_load.restype = C.c_void_p
    lib.ref_pbrt_load.argtypes = [C.c_char_p]
    lib.ref_pbrt_free.argtypes = [C.c_void_p]
    lib.ref_pbrt_info.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ref_pbrt_mesh.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p] + [C.c_void_p] * 9
    h = lib.ref_pbrt_load(str(path).encode())
    try:
        u = np.zeros(6, np.uint32)
        f = np.zeros(29, np.float32)
        lib.ref_pbrt_info(h, u.ctypes.data, f.ctypes.data)
        out = dict(width=int(u[0]), height=int(u[1]), spp=int(u[2]), max_depth=int(u[3]),
                   env=tuple(f[0:3]) if u[5] else None, eye=f[3:6].copy(), look_at=f[6:9].copy(), up=f[9:12].copy(),
                   fov=float(f[12]), camera_to_world=f[13:29].reshape(4, 4).copy(), meshes=[])
        for i in range(int(u[4])):
            mu = np.zeros(5, np.uint32)
            mf = np.zeros(38, np.float32)
            lib.ref_pbrt_mesh(h, i, mu.ctypes.data, mf.ctypes.data, *([None] * 9))
            nv, nf = int(mu[0]), int(mu[1])
            a = [np.zeros(nv, np.float32) for _ in range(6)]
            fv = [np.zeros(nf, np.uint32) for _ in range(3)]
            lib.ref_pbrt_mesh(h, i, mu.ctypes.data, mf.ctypes.data, *[v.ctypes.data for v in a + fv])
            out["meshes"].append(dict(x=a[0], y=a[1], z=a[2], faces=np.stack(fv, 1) if nf else np.zeros((0, 3), np.uint32),
                                      normals=np.stack(a[3:], 1) if mu[2] else None, material=int(mu[3]),
                                      is_light=bool(mu[4]), object_to_world=mf[0:16].reshape(4, 4).copy(),
                                      normal_inverse=mf[16:32].reshape(4, 4).copy(), albedo=mf[32:35].copy(),
                                      emission=mf[35:38].copy()))
        return out
    finally:
        lib.ref_pbrt_free(h)

