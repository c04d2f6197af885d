"""The opt-in two-level (instanced) scene layout, pt_scene_create_two_level, on the device.

The reference has no such layout (it flattens every instance into one world-space tree,
pbrt_parser.cpp:1439-1472, bvh.cpp:36-130), so parity is stated against the flattened scene,
which is itself bit-exact with the reference:
  * closest-hit primitive ids equal the flattened scene's wherever the first hit is unambiguous:
    a differing id is allowed only where the flattened scene's t for that ray and the two-level t
    agree to 1e-4 relative (two faces at the same distance: a shared edge or coincident faces);
  * t of equal ids agrees to T_REL (1e-5) relative; any-hit outcomes agree on >= 99.9 % of rays;
  * films at equal spp agree within REL_RMSE_TOL relative RMSE and MEAN_TOL relative mean absolute
    error, primary ids on >= 99.9 % of pixels;
  * the same two-level frame is bit-identical through pt_render's fused (default) and persistent
    pipelines, batches and the serving loop on the fused and path pipelines, pt_render_noalloc and
    pt_render_rgba8 (the persistent kernel's resumable walk makes the fused kernel's hits).
Scene: the instanced workload (the displaced sphere instanced five times with seeded rigid
transforms, Lambert or mirror, over a ground quad, a 3x3 light, environment 0.2)."""
import numpy as np
import pytest

from conftest import assert_bit_equal
import polytope_b200 as pb
from polytope_b200 import workloads as W

pytestmark = pytest.mark.gpu

T_REL = 1e-5
REL_RMSE_TOL = 2e-2
MEAN_TOL = 5e-3


@pytest.fixture(scope="module")
def scenes():
    meshes, env = W.instanced_scene(level=6)
    flat = pb.Scene(meshes, env)
    two = pb.Scene(meshes, env, two_level=True)
    yield meshes, env, flat, two
    two.close()
    flat.close()


def random_rays(n, seed):
    rng = np.random.default_rng(seed)
    org = rng.normal(size=(n, 3))
    org = 12.0 * org / np.linalg.norm(org, axis=1)[:, None]
    tgt = rng.uniform(-4.5, 4.5, (n, 3))
    d = tgt - org
    rays = np.zeros(n, pb.RAY_DTYPE)
    rays["org"] = org
    rays["dir"] = d / np.linalg.norm(d, axis=1)[:, None]
    rays["tmax"] = np.inf
    rays["flags"][1::2] = pb.RAY_ANY_HIT
    rays["tmax"][1::2] = np.linalg.norm(d, axis=1)[1::2]
    return rays


def test_two_level_scene_holds_a_fifth_of_the_memory(scenes):
    meshes, env, flat, two = scenes
    plan = pb.two_level_plan(meshes, env)
    assert plan["num_instances"] == len(meshes) and plan["num_geometries"] == 3
    fb, tb = flat.info().device_bytes, two.info().device_bytes
    assert tb == plan["device_bytes"]
    assert fb / tb > 4.0, (fb, tb)


def test_two_level_hits_match_the_flattened_scene(scenes):
    meshes, env, flat, two = scenes
    rays = random_rays(400_000, 3)
    hf, ht = flat.intersect(rays), two.intersect(rays)
    closest = rays["flags"] == 0
    a, b = hf[closest], ht[closest]
    same = a["prim"] == b["prim"]
    assert same.mean() > 0.999, same.mean()
    both = same & (a["prim"] != pb.PRIM_NONE)
    assert both.sum() > 50_000
    rel = np.abs(a["t"][both] - b["t"][both]) / a["t"][both]
    assert rel.max() <= T_REL, rel.max()
    # a differing id: both rays hit, at the same distance (an edge or coincident faces)
    diff = ~same
    assert ((a["prim"][diff] != pb.PRIM_NONE) & (b["prim"][diff] != pb.PRIM_NONE)).all()
    assert (np.abs(a["t"][diff] - b["t"][diff]) <= 1e-4 * a["t"][diff]).all()
    anyf = hf["prim"][~closest] != pb.PRIM_NONE
    anyt = ht["prim"][~closest] != pb.PRIM_NONE
    assert (anyf == anyt).mean() > 0.999
    # device pointers and the counted form give the same hits
    import torch
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda")
    two.intersect(d_rays, d_hits, device=True)
    torch.cuda.synchronize()
    assert d_hits.cpu().numpy().tobytes() == ht.tobytes()
    hc, nt, tt = two.intersect(rays[:50_000], counts=True)
    assert hc.tobytes() == ht[:50_000].tobytes() and nt.min() >= 1
    assert two.status() == pb.PT_OK


def test_two_level_render_matches_the_flattened_film(scenes):
    meshes, env, flat, two = scenes
    args = (160, 120, 8, 8, W.INSTANCED_CAMERA, 1, pb.RENDER_NEE)
    frgb, fprim = pb.render(flat, *args)
    trgb, tprim = pb.render(two, *args)
    a, b = trgb.astype(np.float64), frgb.astype(np.float64)
    rel_rmse = np.sqrt(((a - b) ** 2).mean()) / np.sqrt((b ** 2).mean())
    rel_mean = np.abs(a - b).mean() / np.abs(b).mean()
    assert rel_rmse <= REL_RMSE_TOL and rel_mean <= MEAN_TOL, (rel_rmse, rel_mean)
    assert (tprim == fprim).mean() >= 0.999
    assert b.mean() > 1.0


def test_two_level_frame_is_the_same_through_every_route(scenes):
    """The persistent path kernel's resumable two-level walk (walk_step_two_level) and the fused
    kernel's traverse_two_level make the same hits, so a two-level frame is bit-identical through
    pt_render's default and fused pipelines, batches and the serving loop on both their pipelines
    (mixed with a flattened item), pt_render_noalloc and pt_render_rgba8."""
    import ctypes as C
    import torch
    meshes, env, flat, two = scenes
    fl = pb.RENDER_NEE | pb.RENDER_JITTER
    rd = pb.render_desc(64, 48, 4, 6, W.INSTANCED_CAMERA, 5, fl)
    rgb, prim = pb.render(two, 64, 48, 4, 6, W.INSTANCED_CAMERA, 5, fl | pb.RENDER_FUSED)
    for name, extra, wave in (("default", 0, 0), ("persistent", pb.RENDER_PERSISTENT, 0), ("persistent, small waves", 0, 1000)):
        r2, p2 = pb.render(two, 64, 48, 4, 6, W.INSTANCED_CAMERA, 5, fl | extra, wave)
        assert_bit_equal(r2, rgb, f"pt_render {name}")
        assert_bit_equal(p2, prim, f"pt_render {name} primary ids")
    f_rgb, _ = pb.render(flat, 64, 48, 4, 6, W.INSTANCED_CAMERA, 5, fl)
    for pipe in (pb.PIPELINE_FUSED, pb.PIPELINE_PATHS):
        t = pb.default_tuning()
        t.pipeline = pipe
        b = pb.Batch([(two, rd), (flat, rd)], t)  # a two-level and a flattened item in one launch
        b.run()
        assert_bit_equal(b.output(0)[0], rgb, f"batch {pipe}, two-level item")
        assert_bit_equal(b.output(0)[1], prim, f"batch {pipe}, two-level primary ids")
        assert_bit_equal(b.output(1)[0], f_rgb, f"batch {pipe}, flattened item")
        b.close()
        srv = pb.Server(max_inflight=4, wave_pixels=1 << 12, tuning=t)
        tk = [srv.submit(two, rd), srv.submit(flat, rd)]
        assert srv.wait(tk[0], 60000) == pb.REQ_DONE and srv.wait(tk[1], 60000) == pb.REQ_DONE
        assert_bit_equal(srv.fetch(tk[0])[0], rgb, f"served {pipe}, two-level")
        assert_bit_equal(srv.fetch(tk[1])[0], f_rgb, f"served {pipe}, flattened")
        srv.close()
    out = torch.full((64 * 48 * 3,), float("nan"), dtype=torch.float32, device="cuda")
    pb.check(pb.lib.pt_render_noalloc(two.handle, C.byref(rd), out.data_ptr(), None, None))
    torch.cuda.synchronize()
    assert_bit_equal(out.cpu().numpy().reshape(48, 64, 3), rgb, "pt_render_noalloc")
    rgba, _ = pb.render_rgba8(two, 64, 48, 4, 6, W.INSTANCED_CAMERA, 5, pb.RENDER_NEE | pb.RENDER_JITTER)
    from oracle import pyoracle as po
    assert_bit_equal(rgba, po.film_to_rgba8(rgb), "pt_render_rgba8")


def test_two_level_scene_refuses_the_wavefront_pipeline(scenes):
    meshes, env, flat, two = scenes
    with pytest.raises(pb.PolytopeError) as e:
        pb.render(two, 8, 8, 1, 2, W.INSTANCED_CAMERA, 1, pb.RENDER_WAVEFRONT)
    assert e.value.code == pb.PT_EINVAL
    rd = pb.render_desc(8, 8, 1, 2, W.INSTANCED_CAMERA)
    for pipe in (pb.PIPELINE_WAVEFRONT,):
        t = pb.default_tuning()
        t.pipeline = pipe
        with pytest.raises(pb.PolytopeError) as e:
            pb.Batch([(two, rd)], t)
        assert e.value.code == pb.PT_EINVAL
        srv = pb.Server(max_inflight=2, tuning=t)
        with pytest.raises(pb.PolytopeError) as e:
            srv.submit(two, rd)
        assert e.value.code == pb.PT_EINVAL
        srv.close()
