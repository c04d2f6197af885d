"""GPU parity of the render call (pt_render) against the patched reference render loop
(fixtures from oracle/_ref) and the CPU oracle.  With the shared counter RNG and the shared
sin/cos the film is bit-exact; the stated image tolerance (relative RMSE <= 1e-6, per-pixel mean
error <= 1e-6) is therefore met with margin, and primary-hit ids are exact."""
import numpy as np
import pytest

from conftest import assert_bit_equal, load_golden
import polytope_b200 as pb
from polytope_b200 import workloads as W
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

REL_RMSE_TOL = 1e-6
MEAN_ERR_TOL = 1e-6


def image_errors(a, b):
    a, b = a.astype(np.float64), b.astype(np.float64)
    rmse = np.sqrt(((a - b) ** 2).mean())
    rel = rmse / max(np.sqrt((b ** 2).mean()), 1e-30)
    return rel, np.abs(a - b).mean() / max(np.abs(b).mean(), 1e-30)


PIPELINES = [pb.RENDER_FUSED, pb.RENDER_WAVEFRONT, pb.RENDER_PERSISTENT]


@pytest.mark.parametrize("pipeline", PIPELINES, ids=["fused", "wavefront", "persistent"])
def test_small_scene_render_matches_reference_fixture(cuda_device, pipeline):
    g = load_golden("small_scene.npz")
    meshes, env = W.small_scene()
    scene = pb.Scene(meshes, env)
    for flags, key in ((pb.RENDER_NEE, "nee"), (0, "bsdf")):
        rgb, prim = pb.render(scene, 80, 60, 4, 4, W.SMALL_CAMERA, seed=1, flags=flags | pipeline)
        rel, mean = image_errors(rgb, g[f"rgb_{key}"])
        assert rel <= REL_RMSE_TOL and mean <= MEAN_ERR_TOL, (key, rel, mean)
        assert_bit_equal(rgb, g[f"rgb_{key}"], f"film {key}")
        assert_bit_equal(prim, g[f"prim_{key}"], f"primary ids {key}")


@pytest.mark.parametrize("pipeline", PIPELINES, ids=["fused", "wavefront", "persistent"])
def test_small_scene_full_config_matches_oracle(cuda_device, pipeline):
    """320x240, 8 spp, depth 4, NEE: the full small configuration against the CPU oracle."""
    meshes, env = W.small_scene()
    scene = pb.Scene(meshes, env)
    d = W.SMALL_RENDER
    rgb, prim = pb.render(scene, d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                          pb.RENDER_NEE | pipeline)
    o = po.OracleScene(meshes, env)
    orgb, oprim = o.render(dict(d, flags=1))
    assert_bit_equal(prim, oprim, "primary ids")
    assert_bit_equal(rgb, orgb, "film")
    assert rgb.mean() > 1.0


@pytest.mark.parametrize("pipeline", PIPELINES, ids=["fused", "wavefront", "persistent"])
def test_coincident_faces_render_matches_oracle(cuda_device, pipeline):
    """The small scene with every sphere face listed twice (the copy's vertices rotated), so that
    MinT rises on many camera, bounce and shadow rays; the film must still equal the oracle's."""
    import dataclasses
    meshes, env = W.small_scene(level=3)
    sph = meshes[1]
    meshes[1] = dataclasses.replace(sph, faces=np.concatenate([sph.faces, sph.faces[:, [1, 2, 0]]]))
    scene = pb.Scene(meshes, env)
    rgb, prim = pb.render(scene, 96, 72, 4, 4, W.SMALL_CAMERA, seed=3, flags=pb.RENDER_NEE | pipeline)
    orgb, oprim = po.OracleScene(meshes, env).render(
        dict(width=96, height=72, spp=4, max_depth=4, seed=3, camera=W.SMALL_CAMERA, flags=1))
    assert_bit_equal(prim, oprim, "primary ids")
    assert_bit_equal(rgb, orgb, "film")


@pytest.mark.parametrize("pipeline", PIPELINES, ids=["fused", "wavefront", "persistent"])
def test_instanced_scene_matches_reference_fixture(cuda_device, pipeline):
    g = load_golden("instanced_small.npz")
    im, env = W.instanced_scene(level=4)
    scene = pb.Scene(im, env)
    rgb, prim = pb.render(scene, 64, 40, 2, 8, W.INSTANCED_CAMERA, seed=1, flags=pb.RENDER_NEE | pipeline)
    assert_bit_equal(prim, g["prim"], "primary ids")
    assert_bit_equal(rgb, g["rgb"], "film")


@pytest.mark.parametrize("flags", [pb.RENDER_JITTER | pb.RENDER_NEE, pb.RENDER_JITTER,
                                   pb.RENDER_JITTER | pb.RENDER_NEE | pb.RENDER_WAVEFRONT,
                                   pb.RENDER_JITTER | pb.RENDER_NEE | pb.RENDER_PERSISTENT,
                                   pb.RENDER_JITTER | pb.RENDER_NEE | pb.RENDER_FUSED])
def test_jitter_and_small_waves(cuda_device, flags):
    meshes, env = W.small_scene(level=3)
    scene = pb.Scene(meshes, env)
    d = dict(width=48, height=36, spp=5, max_depth=6, seed=77, camera=W.SMALL_CAMERA)
    # a wave size that is not a multiple of the pixel count splits samples across waves
    rgb, prim = pb.render(scene, 48, 36, 5, 6, W.SMALL_CAMERA, seed=77, flags=flags, wave_paths=1000)
    rgb2, _ = pb.render(scene, 48, 36, 5, 6, W.SMALL_CAMERA, seed=77, flags=flags)
    assert_bit_equal(rgb, rgb2, "wave size independence")
    orgb, oprim = po.OracleScene(meshes, env).render(dict(d, flags=flags))
    assert_bit_equal(rgb, orgb, "film")
    assert_bit_equal(prim, oprim, "prim")


def test_pipeline_flags_exclude_each_other(cuda_device):
    meshes, env = W.small_scene(level=1)
    scene = pb.Scene(meshes, env)
    for bad in (pb.RENDER_WAVEFRONT | pb.RENDER_PERSISTENT, pb.RENDER_FUSED | pb.RENDER_PERSISTENT,
                pb.RENDER_FUSED | pb.RENDER_WAVEFRONT, 32):
        with pytest.raises(pb.PolytopeError) as e:
            pb.render(scene, 8, 8, 1, 2, W.SMALL_CAMERA, flags=bad)
        assert e.value.code == pb.PT_EINVAL


def test_device_memory_render_is_asynchronous_and_reports_through_scene_status(cuda_device):
    """With PT_MEM_DEVICE pt_render only queues its kernels on the given stream (nothing in the call
    waits for the frame); frames queued back to back on one stream and on a second stream equal the
    host-memory renders, and pt_scene_status reports no guard failure afterwards."""
    import ctypes as C
    import torch
    meshes, env = W.small_scene(level=3)
    scene = pb.Scene(meshes, env)
    frames = [(64, 48, 3, 1, pb.RENDER_NEE), (40, 30, 2, 5, pb.RENDER_NEE | pb.RENDER_JITTER),
              (33, 17, 4, 9, pb.RENDER_NEE | pb.RENDER_FUSED), (50, 20, 2, 2, pb.RENDER_NEE | pb.RENDER_WAVEFRONT)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = []
    for k, (w, h, spp, seed, flags) in enumerate(frames):
        rd = pb.render_desc(w, h, spp, 4, W.SMALL_CAMERA, seed, flags)
        rgb = torch.full((w * h * 3,), float("nan"), dtype=torch.float32, device=cuda_device)
        prim = torch.zeros(w * h, dtype=torch.int32, device=cuda_device)
        st = streams[k % 2]
        rgb.record_stream(st)
        prim.record_stream(st)
        pb.check(pb.lib.pt_render(scene.handle, C.byref(rd), rgb.data_ptr(), prim.data_ptr(), pb.MEM_DEVICE,
                                  st.cuda_stream))
        outs.append((rgb, prim, st))
    for st in streams:
        assert scene.status(st.cuda_stream) == pb.PT_OK
    for (w, h, spp, seed, flags), (rgb, prim, st) in zip(frames, outs):
        exp_rgb, exp_prim = pb.render(scene, w, h, spp, 4, W.SMALL_CAMERA, seed, flags)
        assert_bit_equal(rgb.cpu().numpy().reshape(h, w, 3), exp_rgb, f"film {w}x{h}")
        assert_bit_equal(prim.cpu().numpy().view(np.uint32).reshape(h, w), exp_prim, f"prim {w}x{h}")


def test_runner_interface(cuda_device):
    meshes, env = W.small_scene(level=2)
    scene = pb.Scene(meshes, env)
    r = pb.GpuRunner(scene, 32, 24, 2, 3, W.SMALL_CAMERA, flags=pb.RENDER_NEE)
    with pytest.raises(RuntimeError):
        r.output()
    r.run()
    rgb, prim = r.output()
    assert rgb.shape == (24, 32, 3) and prim.shape == (24, 32)


def test_film_to_rgba8_matches_reference_quantisation(cuda_device):
    import ctypes as C
    import torch
    rng = np.random.default_rng(3)
    h, w = 37, 53
    rgb = rng.uniform(0, 300, (h, w, 3)).astype(np.float32)
    rgb[0, 0] = (0.0, 0.5, 254.99)
    rgb[0, 1] = (255.0, 1e9, 127.9999)
    exp = po.film_to_rgba8(rgb)
    d = torch.from_numpy(rgb).cuda()
    assert_bit_equal(pb.film_to_rgba8(d.data_ptr(), w, h), exp, "rgba8, host output")
    out = torch.zeros(h * w * 4, dtype=torch.uint8, device="cuda")
    pb.check(pb.lib.pt_film_to_rgba8(d.data_ptr(), w, h, out.data_ptr(), pb.MEM_DEVICE, None))
    torch.cuda.synchronize()
    assert_bit_equal(out.cpu().numpy().reshape(h, w, 4), exp, "rgba8, device output")
    # a rendered film, quantised on the device, equals the oracle's quantisation of the same film
    meshes, env = W.small_scene(level=3)
    scene = pb.Scene(meshes, env)
    rd = pb.render_desc(64, 48, 4, 4, W.SMALL_CAMERA, 5, pb.RENDER_NEE)
    film = torch.zeros(64 * 48 * 3, dtype=torch.float32, device="cuda")
    pb.check(pb.lib.pt_render(scene.handle, C.byref(rd), film.data_ptr(), None, pb.MEM_DEVICE, None))
    torch.cuda.synchronize()
    host_film = film.cpu().numpy().reshape(48, 64, 3)
    assert_bit_equal(pb.film_to_rgba8(film.data_ptr(), 64, 48), po.film_to_rgba8(host_film), "rendered film")
    # the render call with the output step on the device: host bytes, and device bytes queued on a stream
    rgba, prim = pb.render_rgba8(scene, 64, 48, 4, 4, W.SMALL_CAMERA, 5, pb.RENDER_NEE)
    assert_bit_equal(rgba, po.film_to_rgba8(host_film), "pt_render_rgba8 host")
    assert_bit_equal(prim, pb.render(scene, 64, 48, 4, 4, W.SMALL_CAMERA, 5, pb.RENDER_NEE)[1], "pt_render_rgba8 prim")
    dbytes = torch.zeros(64 * 48 * 4, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    pb.check(pb.lib.pt_render_rgba8(scene.handle, C.byref(rd), dbytes.data_ptr(), None, pb.MEM_DEVICE, st.cuda_stream))
    assert scene.status(st.cuda_stream) == pb.PT_OK
    assert_bit_equal(dbytes.cpu().numpy().reshape(48, 64, 4), po.film_to_rgba8(host_film), "pt_render_rgba8 device")
