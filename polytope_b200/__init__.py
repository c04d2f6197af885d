"""polytope_b200 -- B200-native ray/path-tracing hot path of Polytope, behind a C ABI.

This package is a thin ctypes layer over ``polytope_b200/lib/libpolytope_b200.so`` (built from
``polytope_b200/csrc``; declared in ``include/polytope_b200.h``).  The classes mirror the
reference's own interfaces (paths relative to the Polytope source tree):

* :class:`Mesh`        -- ``poly::Mesh`` + ``poly::mesh_geometry`` (src/cpu/shapes/mesh.h:17-113)
* :class:`Scene`       -- ``poly::Scene`` (src/cpu/scenes/Scene.h:17-35); ``Scene.intersect`` is
  ``Scene::intersect`` (Scene.cpp:12-31) for a batch of rays
* :func:`bvh_build`    -- ``poly::bvh::bound`` + ``compact`` (src/cpu/acceleration/bvh.cpp:36-395, 652-698)
* :class:`GpuRunner`   -- ``poly::AbstractRunner`` (src/cpu/runners/AbstractRunner.h:38-45):
  ``run()`` renders the frame, ``output()`` returns the film

There is no CPU fallback: the library needs a CUDA device for every call that launches work, and
importing the package fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpolytope_b200.so")

PT_OK, PT_EINVAL, PT_ENOMEM, PT_ETIMEOUT, PT_ECUDA, PT_ESTACK, PT_ECANCELED = 0, -1, -2, -3, -4, -5, -6
REQ_QUEUED, REQ_ADMITTED, REQ_DONE, REQ_CANCELLED = 0, 1, 2, 3
PRIM_NONE = 0xFFFFFFFF
MAT_LAMBERT, MAT_MIRROR = 1, 2
RAY_ANY_HIT = 1
MEM_DEVICE = 1
RENDER_NEE, RENDER_JITTER, RENDER_WAVEFRONT, RENDER_PERSISTENT, RENDER_FUSED = 1, 2, 4, 8, 16

RAY_DTYPE = np.dtype([("org", "<f4", 3), ("tmax", "<f4"), ("dir", "<f4", 3), ("flags", "<u4")])
HIT_DTYPE = np.dtype([("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
NODE_DTYPE = np.dtype([("bb", "<f4", 6), ("offset", "<u4"), ("num_faces", "<u2"), ("axis", "<u2")])

_fp = C.POINTER(C.c_float)
_up = C.POINTER(C.c_uint32)
_vp = C.c_void_p


class PolytopeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"polytope_b200 error {code}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [
        ("x", _fp), ("y", _fp), ("z", _fp), ("num_vertices", C.c_uint32),
        ("fv0", _up), ("fv1", _up), ("fv2", _up), ("num_faces", C.c_uint32),
        ("nx", _fp), ("ny", _fp), ("nz", _fp),
        ("object_to_world", C.c_float * 16), ("world_to_object", C.c_float * 16),
        ("material", C.c_uint32), ("albedo", C.c_float * 3),
        ("is_light", C.c_int32), ("emission", C.c_float * 3),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("meshes", C.POINTER(MeshDesc)), ("num_meshes", C.c_uint32),
        ("nodes", _vp), ("num_nodes", C.c_uint32), ("leaf_pairs", _up),
        ("has_env", C.c_int32), ("env", C.c_float * 3),
    ]


class SceneInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_uint32), ("num_prims", C.c_uint32), ("num_meshes", C.c_uint32),
                ("max_depth", C.c_uint32), ("device_bytes", C.c_uint64)]


class Camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float)]


class RenderDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_depth", C.c_uint32),
                ("seed", C.c_uint64), ("flags", C.c_uint32), ("wave_paths", C.c_uint32), ("camera", Camera)]


class TraceTuning(C.Structure):
    _fields_ = [("shared_stack", C.c_uint32), ("queue_chunk", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class BatchItem(C.Structure):
    _fields_ = [("scene", _vp), ("desc", RenderDesc)]


PIPELINE_FUSED, PIPELINE_WAVEFRONT, PIPELINE_PATHS = 0, 1, 2
SERVE_OLDEST_FIRST, SERVE_FAIR_SHARE = 0, 1


class BatchTuning(C.Structure):
    _fields_ = [("wave_pixels", C.c_uint64), ("threads_per_block", C.c_uint32), ("stack_depth", C.c_uint32),
                ("queue_chunk", C.c_uint32), ("pipeline", C.c_uint32)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class BatchTuneResult(C.Structure):
    _fields_ = [("tuning", BatchTuning), ("ms", C.c_float)]


class TuningClass(C.Structure):
    """pt_tuning_class: the device and the bucketed scale of a batch a cached tuning is reused for."""
    _fields_ = [("device", C.c_char * 64), ("sm_count", C.c_uint32), ("compute_capability", C.c_uint32),
                ("items_log2", C.c_uint32), ("pixels_log2", C.c_uint32), ("samples_log2", C.c_uint32),
                ("faces_log2", C.c_uint32), ("tree_depth", C.c_uint32), ("max_depth", C.c_uint32),
                ("flags", C.c_uint32)]

    def as_dict(self):
        d = {k: int(getattr(self, k)) for k, _ in self._fields_[1:]}
        d["device"] = bytes(self.device).split(b"\0", 1)[0].decode("utf-8", errors="replace")
        return d


class ServerConfig(C.Structure):
    _fields_ = [("max_inflight", C.c_uint32), ("memory_budget", C.c_uint64), ("wave_pixels", C.c_uint64),
                ("tuning", BatchTuning), ("policy", C.c_uint32), ("host_budget", C.c_uint64)]


class MeshData(C.Structure):
    _fields_ = [("x", _fp), ("y", _fp), ("z", _fp), ("num_vertices", C.c_uint32),
                ("fv0", _up), ("fv1", _up), ("fv2", _up), ("num_faces", C.c_uint32),
                ("nx", _fp), ("ny", _fp), ("nz", _fp), ("u", _fp), ("v", _fp)]


class PbrtInfo(C.Structure):
    _fields_ = [("num_meshes", C.c_uint32), ("has_env", C.c_int32), ("env", C.c_float * 3),
                ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_depth", C.c_uint32),
                ("camera", Camera)]


class RequestTiming(C.Structure):
    _fields_ = [("admitted_ms", C.c_double), ("first_wave_ms", C.c_double), ("last_wave_ms", C.c_double),
                ("done_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("waves", C.c_uint64), ("completed", C.c_uint64), ("rays_traced", C.c_uint64), ("busy_ms", C.c_double),
                ("pending", C.c_uint64), ("active", C.c_uint64), ("device_bytes_in_use", C.c_uint64),
                ("blocked_ms", C.c_double), ("host_bytes_in_use", C.c_uint64), ("plan_ms", C.c_double),
                ("retire_wait_ms", C.c_double), ("waves_launched", C.c_uint64), ("cancelled", C.c_uint64)]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C polytope_b200/csrc` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    i, u32, u64 = C.c_int, C.c_uint32, C.c_uint64
    sig = {
        "pt_last_error": (C.c_char_p, []),
        "pt_version": (C.c_char_p, []),
        "pt_bvh_build": (i, [C.POINTER(MeshDesc), u32, i, _vp, _up, _up]),
        "pt_scene_create": (i, [C.POINTER(SceneDesc), C.POINTER(_vp)]),
        "pt_scene_create_two_level": (i, [C.POINTER(SceneDesc), C.POINTER(_vp)]),
        "pt_scene_destroy": (i, [_vp]),
        "pt_scene_get_info": (i, [_vp, C.POINTER(SceneInfo)]),
        "pt_trace": (i, [_vp, _vp, u64, _vp, u32, _vp]),
        "pt_trace_counted": (i, [_vp, _vp, u64, _vp, _vp, _vp, u32, _vp]),
        "pt_render": (i, [_vp, C.POINTER(RenderDesc), _vp, _vp, u32, _vp]),
        "pt_scene_set_trace_tuning": (i, [_vp, C.POINTER(TraceTuning)]),
        "pt_scene_get_trace_tuning": (i, [_vp, C.POINTER(TraceTuning)]),
        "pt_trace_autotune": (i, [_vp, _vp, u64, _vp, C.POINTER(TraceTuning), C.POINTER(C.c_float)]),
        "pt_render_noalloc": (i, [_vp, C.POINTER(RenderDesc), _vp, _vp, _vp]),
        "pt_scene_status": (i, [_vp, _vp]),
        "pt_render_rgba8": (i, [_vp, C.POINTER(RenderDesc), _vp, _vp, u32, _vp]),
        "pt_film_to_rgba8": (i, [_vp, u32, u32, _vp, u32, _vp]),
        "pt_load_ply": (i, [C.c_char_p, C.POINTER(MeshData)]),
        "pt_load_obj": (i, [C.c_char_p, C.POINTER(MeshData)]),
        "pt_mesh_data_free": (None, [C.POINTER(MeshData)]),
        "pt_write_png": (i, [C.c_char_p, _vp, u32, u32]),
        "pt_load_pbrt": (i, [C.c_char_p, C.POINTER(_vp)]),
        "pt_pbrt_get_info": (i, [_vp, C.POINTER(PbrtInfo)]),
        "pt_pbrt_get_meshes": (i, [_vp, C.POINTER(C.POINTER(MeshDesc))]),
        "pt_pbrt_free": (None, [_vp]),
        "pt_batch_default_tuning": (i, [C.POINTER(BatchTuning)]),
        "pt_batch_create": (i, [C.POINTER(BatchItem), u32, C.POINTER(BatchTuning), C.POINTER(_vp)]),
        "pt_batch_run": (i, [_vp, _vp]),
        "pt_batch_output": (i, [_vp, u32, _vp, _vp, C.POINTER(u64)]),
        "pt_batch_destroy": (i, [_vp]),
        "pt_batch_autotune": (i, [C.POINTER(BatchItem), u32, C.POINTER(BatchTuning), C.POINTER(C.c_double),
                                  C.POINTER(BatchTuneResult), C.POINTER(u32)]),
        "pt_tuning_class_of": (i, [C.POINTER(BatchItem), u32, C.POINTER(TuningClass)]),
        "pt_tuning_cache_get": (i, [C.c_char_p, C.POINTER(TuningClass), C.POINTER(BatchTuning), C.POINTER(C.c_double),
                                    C.POINTER(i)]),
        "pt_tuning_cache_put": (i, [C.c_char_p, C.POINTER(TuningClass), C.POINTER(BatchTuning), C.c_double]),
        "pt_batch_autotune_cached": (i, [C.POINTER(BatchItem), u32, C.c_char_p, C.POINTER(BatchTuning),
                                         C.POINTER(C.c_double), C.POINTER(i)]),
        "pt_server_create": (i, [C.POINTER(ServerConfig), C.POINTER(_vp)]),
        "pt_server_submit": (i, [_vp, _vp, C.POINTER(RenderDesc), C.POINTER(u64)]),
        "pt_server_poll": (i, [_vp, u64, C.POINTER(i), C.POINTER(C.c_double)]),
        "pt_server_timing": (i, [_vp, u64, C.POINTER(RequestTiming)]),
        "pt_server_wait": (i, [_vp, u64, u32, C.POINTER(i)]),
        "pt_server_fetch": (i, [_vp, u64, _vp, _vp]),
        "pt_server_get_stats": (i, [_vp, C.POINTER(ServerStats)]),
        "pt_server_destroy": (i, [_vp]),
        "pt_server_cancel": (i, [_vp, u64]),
        "pt_gen_icosphere": (i, [u32, C.c_float, C.c_float, u64, _fp, _fp, _fp, _up, _up, _up, _up, _up]),
        "pt_gen_rays": (i, [u64, C.c_float, u64, _vp]),
        "pt_host_f64_diff_emulated": (C.c_float, [C.c_float] * 4),
        "pt_selftest_device": (i, [i, _vp, _vp, u32, u64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    # messages can quote bytes of a malformed input file, which need not be UTF-8
    return lib.pt_last_error().decode("utf-8", errors="replace")


def check(rc: int) -> None:
    if rc != PT_OK:
        raise PolytopeError(rc, last_error())


def version() -> str:
    return lib.pt_version().decode()


def _f(a):
    return a.ctypes.data_as(_fp) if a is not None else None


def _u(a):
    return a.ctypes.data_as(_up) if a is not None else None


@dataclass
class Mesh:
    """One mesh instance (poly::Mesh): packed vertices, faces, transform, material, emission."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    faces: np.ndarray                      # (F, 3) uint32 vertex indices
    object_to_world: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    world_to_object: Optional[np.ndarray] = None
    material: int = MAT_LAMBERT
    albedo: Sequence[float] = (0.7, 0.7, 0.7)
    is_light: bool = False
    emission: Sequence[float] = (0.0, 0.0, 0.0)
    normals: Optional[np.ndarray] = None   # (V, 3) packed vertex normals

    def __post_init__(self):
        self.x = np.ascontiguousarray(self.x, np.float32)
        self.y = np.ascontiguousarray(self.y, np.float32)
        self.z = np.ascontiguousarray(self.z, np.float32)
        self.faces = np.ascontiguousarray(self.faces, np.uint32).reshape(-1, 3)
        self.object_to_world = np.asarray(self.object_to_world, np.float32).reshape(4, 4)
        if self.world_to_object is None:
            self.world_to_object = np.linalg.inv(self.object_to_world.astype(np.float64)).astype(np.float32)
        self.world_to_object = np.asarray(self.world_to_object, np.float32).reshape(4, 4)


def mesh_descs(meshes: Sequence[Mesh]):
    """ctypes array of MeshDesc (same layout as pt_mesh_desc) plus the arrays it points into.
    Meshes built on the same face (and normal) arrays get the same column arrays, so their
    descriptors share every geometry pointer (what pt_scene_create_two_level keys instances on)."""
    arr = (MeshDesc * len(meshes))()
    keep = []
    columns = {}

    def cols(a, dtype):
        key = (a.__array_interface__["data"][0], a.shape, a.strides, np.dtype(dtype).str)
        if key not in columns:
            c = np.ascontiguousarray(a, dtype)
            columns[key] = tuple(np.ascontiguousarray(c[:, j]) for j in range(3))
            keep.extend(columns[key])
        return columns[key]

    for k, m in enumerate(meshes):
        f0, f1, f2 = cols(m.faces, np.uint32)
        keep += [m.x, m.y, m.z]
        d = arr[k]
        d.x, d.y, d.z, d.num_vertices = _f(m.x), _f(m.y), _f(m.z), len(m.x)
        d.fv0, d.fv1, d.fv2, d.num_faces = _u(f0), _u(f1), _u(f2), len(f0)
        if m.normals is not None:
            nx, ny, nz = cols(m.normals, np.float32)
            d.nx, d.ny, d.nz = _f(nx), _f(ny), _f(nz)
        d.object_to_world[:] = [float(v) for v in m.object_to_world.ravel()]
        d.world_to_object[:] = [float(v) for v in m.world_to_object.ravel()]
        d.material = int(m.material)
        d.albedo[:] = [float(v) for v in m.albedo]
        d.is_light = int(bool(m.is_light))
        d.emission[:] = [float(v) for v in m.emission]
    return arr, keep


def bvh_build(meshes: Sequence[Mesh], threads: int = 0):
    """The reference SAH BVH (node-for-node identical): returns (nodes, leaf_pairs)."""
    arr, keep = mesh_descs(meshes)
    faces = sum(len(m.faces) for m in meshes)
    # one build: a tree over F faces has at most 2F - 1 nodes
    n = C.c_uint32(max(1, 2 * faces - 1))
    nodes = np.zeros(n.value, NODE_DTYPE)
    pairs = np.zeros((faces, 2), np.uint32)
    check(lib.pt_bvh_build(arr, len(meshes), threads, nodes.ctypes.data, C.byref(n), _u(pairs)))
    return nodes[:n.value].copy(), pairs


def scene_desc(meshes: Sequence[Mesh], env=None, nodes=None, leaf_pairs=None):
    """pt_scene_desc of the meshes (plus the arrays it points into, to keep alive)."""
    arr, keep = mesh_descs(meshes)
    d = SceneDesc()
    d.meshes = arr
    d.num_meshes = len(meshes)
    keep.append(arr)
    if nodes is not None:
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        pairs = np.ascontiguousarray(leaf_pairs, np.uint32)
        keep += [nodes, pairs]
        d.nodes = nodes.ctypes.data
        d.num_nodes = len(nodes)
        d.leaf_pairs = _u(pairs)
    d.has_env = int(env is not None)
    if env is not None:
        d.env[:] = [float(v) for v in env]
    return d, keep


class TwoLevelInfo(C.Structure):
    _fields_ = [("num_instances", C.c_uint32), ("num_geometries", C.c_uint32), ("blas_nodes", C.c_uint32),
                ("blas_faces", C.c_uint32), ("tlas_nodes", C.c_uint32), ("max_depth", C.c_uint32),
                ("tlas_depth", C.c_uint32), ("num_prims", C.c_uint32), ("device_bytes", C.c_uint64)]


lib.pt_two_level_plan.restype = C.c_int
lib.pt_two_level_plan.argtypes = [C.POINTER(SceneDesc), C.POINTER(TwoLevelInfo)]


def two_level_plan(meshes: Sequence[Mesh], env=None) -> dict:
    """pt_two_level_plan: what a two-level scene of these meshes would hold (host only)."""
    d, keep = scene_desc(list(meshes), env)
    info = TwoLevelInfo()
    check(lib.pt_two_level_plan(C.byref(d), C.byref(info)))
    return {k: int(getattr(info, k)) for k, _ in info._fields_}


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor (device pointers for MEM_DEVICE calls)."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Scene:
    """poly::Scene on the GPU: meshes (Shapes and Lights), optional constant environment, BVH."""

    def __init__(self, meshes: Sequence[Mesh], env: Optional[Sequence[float]] = None,
                 nodes: Optional[np.ndarray] = None, leaf_pairs: Optional[np.ndarray] = None,
                 two_level: bool = False):
        """two_level: pt_scene_create_two_level -- meshes sharing their vertex and face arrays
        become instances of one object-space geometry under a top-level tree."""
        self.meshes = list(meshes)
        self.two_level = two_level
        d, keep = scene_desc(self.meshes, env, nodes, leaf_pairs)
        h = _vp()
        check((lib.pt_scene_create_two_level if two_level else lib.pt_scene_create)(C.byref(d), C.byref(h)))
        self.handle = h
        self.prim_base = np.concatenate([[0], np.cumsum([len(m.faces) for m in self.meshes])]).astype(np.int64)

    def close(self):
        if getattr(self, "handle", None):
            lib.pt_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> SceneInfo:
        inf = SceneInfo()
        check(lib.pt_scene_get_info(self.handle, C.byref(inf)))
        return inf

    def intersect(self, rays, hits=None, device: bool = False, stream: int = 0, counts: bool = False):
        """Scene::intersect for a batch: numpy (host) arrays, or torch CUDA tensors with device=True
        (asynchronous on `stream`).  Returns hits (and node/face test counts with counts=True)."""
        nbytes = lambda x: x.numel() * x.element_size() if hasattr(x, "numel") else x.nbytes
        if device:
            # counts come from byte sizes, so a tensor of any element type is read correctly
            if nbytes(rays) % RAY_DTYPE.itemsize:
                raise ValueError("device rays must be a whole number of 32-byte pt_ray records")
            n = nbytes(rays) // RAY_DTYPE.itemsize
        else:
            rays = np.ascontiguousarray(rays, RAY_DTYPE)
            n = len(rays)
        if hits is None:
            if device:
                raise ValueError("device calls need a preallocated hits tensor")
            hits = np.zeros(n, HIT_DTYPE)
        if nbytes(hits) < n * HIT_DTYPE.itemsize:
            raise ValueError(f"hits buffer holds {nbytes(hits)} bytes, {n} hits need {n * HIT_DTYPE.itemsize}")
        flags = MEM_DEVICE if device else 0
        if counts:
            if device:
                raise ValueError("counts are host-only here")
            nt = np.zeros(n, np.uint32)
            tt = np.zeros(n, np.uint32)
            check(lib.pt_trace_counted(self.handle, _ptr(rays), n, _ptr(hits), nt.ctypes.data, tt.ctypes.data, 0, None))
            return hits, nt, tt
        check(lib.pt_trace(self.handle, _ptr(rays), n, _ptr(hits), flags, stream or None))
        return hits

    def status(self, stream: int = 0) -> int:
        """pt_scene_status: waits for `stream`, then returns (and clears) the scene's device error
        status -- PT_OK, or PT_ESTACK when a kernel of an asynchronous call met a traversal guard."""
        rc = lib.pt_scene_status(self.handle, stream or None)
        if rc not in (PT_OK, PT_ESTACK):
            check(rc)
        return rc

    def set_trace_tuning(self, shared_stack: int, queue_chunk: int):
        check(lib.pt_scene_set_trace_tuning(self.handle, C.byref(TraceTuning(shared_stack, queue_chunk))))

    def trace_tuning(self) -> dict:
        t = TraceTuning()
        check(lib.pt_scene_get_trace_tuning(self.handle, C.byref(t)))
        return t.as_dict()

    def autotune_trace(self, d_rays, d_hits, n: int):
        """Times the ray-query launch shapes on device buffers; keeps and returns the fastest."""
        t, ms = TraceTuning(), C.c_float(0)
        check(lib.pt_trace_autotune(self.handle, _ptr(d_rays), n, _ptr(d_hits), C.byref(t), C.byref(ms)))
        return t.as_dict(), float(ms.value)

    def prim_to_mesh_face(self, prim: np.ndarray):
        prim = np.asarray(prim, np.int64)
        m = np.searchsorted(self.prim_base, prim, side="right") - 1
        return m, prim - self.prim_base[m]


def render_desc(width, height, spp, max_depth, camera, seed=1, flags=0, wave_paths=0) -> RenderDesc:
    rd = RenderDesc()
    rd.width, rd.height, rd.spp, rd.max_depth = width, height, spp, max_depth
    rd.seed, rd.flags, rd.wave_paths = seed, flags, wave_paths
    rd.camera.eye[:] = camera["eye"]
    rd.camera.look_at[:] = camera["look_at"]
    rd.camera.up[:] = camera["up"]
    rd.camera.fov_deg = camera["fov"]
    return rd


def render(scene: Scene, width: int, height: int, spp: int, max_depth: int, camera: dict, seed: int = 1,
           flags: int = 0, wave_paths: int = 0):
    """One frame: returns (rgb film (H, W, 3) float32, primary prim ids (H, W) uint32)."""
    rd = render_desc(width, height, spp, max_depth, camera, seed, flags, wave_paths)
    rgb = np.zeros((height, width, 3), np.float32)
    prim = np.zeros((height, width), np.uint32)
    check(lib.pt_render(scene.handle, C.byref(rd), rgb.ctypes.data, prim.ctypes.data, 0, None))
    return rgb, prim


def render_rgba8(scene: Scene, width: int, height: int, spp: int, max_depth: int, camera: dict, seed: int = 1,
                 flags: int = 0, wave_paths: int = 0):
    """One frame as the reference's PNG output stores it, quantised on the device
    (pt_render_rgba8): returns (RGBA8 (H, W, 4) uint8, primary prim ids (H, W) uint32)."""
    rd = render_desc(width, height, spp, max_depth, camera, seed, flags, wave_paths)
    rgba = np.zeros((height, width, 4), np.uint8)
    prim = np.zeros((height, width), np.uint32)
    check(lib.pt_render_rgba8(scene.handle, C.byref(rd), rgba.ctypes.data, prim.ctypes.data, 0, None))
    return rgba, prim


def load_ply(path: str, **mesh_kwargs) -> Mesh:
    """A PLY file as a Mesh (pt_load_ply); keyword arguments go to Mesh (transform, material...).
    Vertex uv, when present, is in the returned mesh's `uv` attribute."""
    return _load_mesh(lib.pt_load_ply, path, mesh_kwargs)


def load_obj(path: str, **mesh_kwargs) -> Mesh:
    """A Wavefront OBJ file as a Mesh (pt_load_obj, the reference's obj_parser rules)."""
    return _load_mesh(lib.pt_load_obj, path, mesh_kwargs)


def _load_mesh(loader, path, mesh_kwargs) -> Mesh:
    d = MeshData()
    check(loader(str(path).encode(), C.byref(d)))
    try:
        nv, nf = d.num_vertices, d.num_faces
        arr = lambda p, n, dt: np.ctypeslib.as_array(p, (n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
        x, y, z = (arr(getattr(d, k), nv, np.float32) for k in ("x", "y", "z"))
        faces = np.stack([arr(getattr(d, k), nf, np.uint32) for k in ("fv0", "fv1", "fv2")], 1) if nf else np.zeros((0, 3), np.uint32)
        normals = np.stack([arr(getattr(d, k), nv, np.float32) for k in ("nx", "ny", "nz")], 1) if bool(d.nx) else None
        uv = np.stack([arr(getattr(d, k), nv, np.float32) for k in ("u", "v")], 1) if bool(d.u) else None
    finally:
        lib.pt_mesh_data_free(C.byref(d))
    m = Mesh(x, y, z, faces, normals=normals, **mesh_kwargs)
    m.uv = uv
    return m


@dataclass
class PbrtScene:
    """A PBRT scene file as read by pt_load_pbrt: meshes (Scene::Shapes order), the environment
    (None without LightSource "infinite") and the render settings of its scene block."""
    meshes: list
    env: Optional[tuple]
    width: int
    height: int
    spp: int
    max_depth: int
    camera: dict

    def render_args(self) -> dict:
        return dict(width=self.width, height=self.height, spp=self.spp, max_depth=self.max_depth, camera=self.camera)


def load_pbrt(path: str) -> PbrtScene:
    """A PBRT scene file (pt_load_pbrt), copied into Mesh objects (instances share nothing here)."""
    h = C.c_void_p()
    check(lib.pt_load_pbrt(str(path).encode(), C.byref(h)))
    try:
        info = PbrtInfo()
        check(lib.pt_pbrt_get_info(h, C.byref(info)))
        descs = C.POINTER(MeshDesc)()
        check(lib.pt_pbrt_get_meshes(h, C.byref(descs)))
        meshes = []
        for k in range(info.num_meshes):
            d = descs[k]
            nv, nf = d.num_vertices, d.num_faces
            arr = lambda ptr, n, dt: np.ctypeslib.as_array(ptr, (n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
            x, y, z = (arr(getattr(d, c), nv, np.float32) for c in ("x", "y", "z"))
            faces = np.stack([arr(getattr(d, c), nf, np.uint32) for c in ("fv0", "fv1", "fv2")], 1) if nf \
                else np.zeros((0, 3), np.uint32)
            normals = np.stack([arr(getattr(d, c), nv, np.float32) for c in ("nx", "ny", "nz")], 1) if bool(d.nx) else None
            meshes.append(Mesh(x, y, z, faces,
                               object_to_world=np.array(d.object_to_world[:], np.float32).reshape(4, 4),
                               world_to_object=np.array(d.world_to_object[:], np.float32).reshape(4, 4),
                               material=int(d.material), albedo=tuple(d.albedo[:]), is_light=bool(d.is_light),
                               emission=tuple(d.emission[:]), normals=normals))
        cam = dict(eye=tuple(info.camera.eye[:]), look_at=tuple(info.camera.look_at[:]), up=tuple(info.camera.up[:]),
                   fov=float(info.camera.fov_deg))
        env = tuple(info.env[:]) if info.has_env else None
        return PbrtScene(meshes, env, info.width, info.height, info.spp, info.max_depth, cam)
    finally:
        lib.pt_pbrt_free(h)


def film_to_rgba8(rgb_dev_ptr: int, width: int, height: int) -> np.ndarray:
    """A device film (width*height*3 floats at rgb_dev_ptr) as the reference's PNG bytes:
    (height, width, 4) uint8, quantised on the device."""
    out = np.zeros((height, width, 4), np.uint8)
    check(lib.pt_film_to_rgba8(rgb_dev_ptr, width, height, out.ctypes.data, 0, None))
    return out


def write_png(path: str, rgba: np.ndarray):
    """RGBA8 pixels (H, W, 4) to a PNG file."""
    rgba = np.ascontiguousarray(rgba, np.uint8)
    check(lib.pt_write_png(str(path).encode(), rgba.ctypes.data, rgba.shape[1], rgba.shape[0]))


class GpuRunner:
    """AbstractRunner shape: ``run()`` is the render call (spawn + join of the CPU runner threads),
    ``output()`` returns the film (PNGFilm::Output minus the PNG quantization)."""

    def __init__(self, scene: Scene, width: int, height: int, spp: int, max_depth: int, camera: dict,
                 seed: int = 1, flags: int = 0):
        self.scene, self.width, self.height, self.spp = scene, width, height, spp
        self.max_depth, self.camera, self.seed, self.flags = max_depth, camera, seed, flags
        self._film = None

    def run(self):
        self._film = render(self.scene, self.width, self.height, self.spp, self.max_depth, self.camera,
                            self.seed, self.flags)

    def output(self):
        if self._film is None:
            raise RuntimeError("run() first")
        return self._film


def icosphere(level: int, radius: float = 1.0, noise_amp: float = 0.0, seed: int = 0):
    """Packed (x, y, z, faces) of the seeded displaced icosphere generator."""
    nv, nf = C.c_uint32(0), C.c_uint32(0)
    check(lib.pt_gen_icosphere(level, radius, noise_amp, seed, None, None, None, C.byref(nv), None, None, None, C.byref(nf)))
    x, y, z = (np.zeros(nv.value, np.float32) for _ in range(3))
    f0, f1, f2 = (np.zeros(nf.value, np.uint32) for _ in range(3))
    check(lib.pt_gen_icosphere(level, radius, noise_amp, seed, _f(x), _f(y), _f(z), C.byref(nv), _u(f0), _u(f1), _u(f2), C.byref(nf)))
    return x, y, z, np.stack([f0, f1, f2], axis=1)


def microbench_rays(n: int, origin_radius: float = 3.0, seed: int = 11) -> np.ndarray:
    rays = np.zeros(n, RAY_DTYPE)
    check(lib.pt_gen_rays(n, origin_radius, seed, rays.ctypes.data))
    return rays


def f64_diff_emulated_host(a: float, b: float, c: float, d: float) -> float:
    return float(lib.pt_host_f64_diff_emulated(a, b, c, d))


def selftest_device(which: int, inp: np.ndarray, n: int, seed: int = 0) -> np.ndarray:
    if which == 3:
        out = np.zeros(n, np.uint32)
    elif which == 0:
        out = np.zeros(n, np.float32)
    elif which == 1:
        out = np.zeros((n, 2), np.float32)
    else:
        out = np.zeros((n, 4), np.uint32)
    inp = np.ascontiguousarray(inp)
    check(lib.pt_selftest_device(which, inp.ctypes.data, out.ctypes.data, n, seed))
    return out


# ---- batched renders -------------------------------------------------------------------------

def default_tuning() -> BatchTuning:
    t = BatchTuning()
    check(lib.pt_batch_default_tuning(C.byref(t)))
    return t


def _batch_items(jobs):
    """jobs: sequence of (Scene, RenderDesc)."""
    arr = (BatchItem * len(jobs))()
    for k, (scene, rd) in enumerate(jobs):
        arr[k].scene = scene.handle
        arr[k].desc = rd
    return arr


class Batch:
    """Many renders in one persistent, CUDA-graph-captured launch (pt_batch_*)."""

    def __init__(self, jobs, tuning: Optional[BatchTuning] = None):
        self.jobs = list(jobs)
        self._items = _batch_items(self.jobs)
        h = _vp()
        check(lib.pt_batch_create(self._items, len(self.jobs), C.byref(tuning) if tuning is not None else None, C.byref(h)))
        self.handle = h

    def run(self, stream: int = 0):
        check(lib.pt_batch_run(self.handle, stream or None))

    def output(self, i: int):
        rd = self.jobs[i][1]
        rgb = np.zeros((rd.height, rd.width, 3), np.float32)
        prim = np.zeros((rd.height, rd.width), np.uint32)
        check(lib.pt_batch_output(self.handle, i, rgb.ctypes.data, prim.ctypes.data, None))
        return rgb, prim

    def rays_traced(self) -> int:
        r = C.c_uint64(0)
        check(lib.pt_batch_output(self.handle, 0, None, None, C.byref(r)))
        return int(r.value)

    def close(self):
        if getattr(self, "handle", None):
            lib.pt_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(jobs, max_results: int = 64):
    """Coordinate-descent search of the batch launch shape; returns (best tuning, best ms, trials)."""
    items = _batch_items(list(jobs))
    best = BatchTuning()
    ms = C.c_double(0)
    res = (BatchTuneResult * max_results)()
    n = C.c_uint32(max_results)
    check(lib.pt_batch_autotune(items, len(jobs), C.byref(best), C.byref(ms), res, C.byref(n)))
    trials = [(res[k].tuning.as_dict(), float(res[k].ms)) for k in range(n.value)]
    return best, float(ms.value), trials


def tuning_class(jobs) -> TuningClass:
    """The class (device and bucketed scale) of a batch, the key of the tuning cache."""
    jobs = list(jobs)
    cls = TuningClass()
    check(lib.pt_tuning_class_of(_batch_items(jobs), len(jobs), C.byref(cls)))
    return cls


def tuning_cache_get(path, cls: TuningClass):
    """(tuning, ms) stored for the class in the JSON cache file, or None."""
    t, ms, found = BatchTuning(), C.c_double(0), C.c_int(0)
    check(lib.pt_tuning_cache_get(os.fsencode(path), C.byref(cls), C.byref(t), C.byref(ms), C.byref(found)))
    return (t, float(ms.value)) if found.value else None


def tuning_cache_put(path, cls: TuningClass, tuning: BatchTuning, ms: float) -> None:
    """Store (or replace) the class's tuning in the JSON cache file."""
    check(lib.pt_tuning_cache_put(os.fsencode(path), C.byref(cls), C.byref(tuning), float(ms)))


def autotune_cached(jobs, path):
    """pt_batch_autotune_cached: (best tuning, ms, True) from the cache file when the batch's class
    is there, else the search's (best, ms, False), stored in the file before return."""
    jobs = list(jobs)
    best, ms, hit = BatchTuning(), C.c_double(0), C.c_int(0)
    check(lib.pt_batch_autotune_cached(_batch_items(jobs), len(jobs), os.fsencode(path), C.byref(best), C.byref(ms),
                                       C.byref(hit)))
    return best, float(ms.value), bool(hit.value)


# ---- serving loop ---------------------------------------------------------------------------

class Server:
    """Continuous batching of render requests over resident scenes (pt_server_*)."""

    def __init__(self, max_inflight: int = 64, memory_budget: int = 0, wave_pixels: int = 1 << 20,
                 tuning: Optional[BatchTuning] = None, policy: int = 0, host_budget: int = 0):
        cfg = ServerConfig()
        cfg.max_inflight = max_inflight
        cfg.memory_budget = memory_budget
        cfg.wave_pixels = wave_pixels
        cfg.tuning = tuning if tuning is not None else default_tuning()
        cfg.policy = policy
        cfg.host_budget = host_budget
        h = _vp()
        check(lib.pt_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h
        self._desc = {}

    def submit(self, scene: Scene, rd: RenderDesc) -> int:
        t = C.c_uint64(0)
        check(lib.pt_server_submit(self.handle, scene.handle, C.byref(rd), C.byref(t)))
        self._desc[t.value] = rd
        return int(t.value)

    def poll(self, ticket: int):
        st, lat = C.c_int(0), C.c_double(0)
        check(lib.pt_server_poll(self.handle, ticket, C.byref(st), C.byref(lat)))
        return st.value, lat.value

    def timing(self, ticket: int) -> dict:
        t = RequestTiming()
        check(lib.pt_server_timing(self.handle, ticket, C.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in t._fields_}

    def wait(self, ticket: int, timeout_ms: int = 60000) -> int:
        st = C.c_int(0)
        check(lib.pt_server_wait(self.handle, ticket, timeout_ms, C.byref(st)))
        return st.value

    def fetch(self, ticket: int):
        rd = self._desc.pop(ticket)
        rgb = np.zeros((rd.height, rd.width, 3), np.float32)
        prim = np.zeros((rd.height, rd.width), np.uint32)
        check(lib.pt_server_fetch(self.handle, ticket, rgb.ctypes.data, prim.ctypes.data))
        return rgb, prim

    def cancel(self, ticket: int) -> None:
        """pt_server_cancel: a queued request ends at once; an admitted one after the waves already
        queued with its work (its state then reads REQ_CANCELLED)."""
        check(lib.pt_server_cancel(self.handle, ticket))

    def stats(self) -> dict:
        s = ServerStats()
        check(lib.pt_server_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if getattr(self, "handle", None):
            lib.pt_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
