"""GPU parity on the batched and serving workloads themselves, against the CPU oracle (and, for
one box scene, a fixture rendered by the reference's own patched render loop).

The oracle is pinned to the compiled reference on these scene kinds (tests/test_oracle_golden.py:
batched-workload scenes with boxes, serving-pool scenes), so a film equal to the oracle's here is
the reference's film.  Every GPU route is checked: pt_render under each pipeline, one batch under
each batch pipeline, and the serving loop under each pipeline with all requests in flight at once.
Films and primary-hit ids must be equal bit for bit (the stated image tolerance, relative RMSE
<= 1e-6 and per-pixel mean error <= 1e-6, is therefore met with margin).

Batched workload (256 scenes, seed 23): scenes 1, 3, 12 and 21 -- 25,582 / 494,590 / 1,570 /
360,574 faces among 1,705 / 34,389 / 104 / 23,221 axis-aligned boxes, at their own resolution,
spp and depth 6.  Serving pool (32 scenes, seed 19): scene 5 (four level-6 instances, Lambert and
mirror, 327,684 faces) and scene 22 (two level-8 instances, 2,621,444 faces), depth 5.  Frames
whose full oracle render would take more than a few seconds are compared on a stated band of
rows (the oracle renders only those rows; the GPU renders the whole frame)."""
import os

import numpy as np
import pytest

from conftest import assert_bit_equal, load_golden
import polytope_b200 as pb
from polytope_b200 import workloads as W
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
PIPELINES = {"fused": pb.RENDER_FUSED, "wavefront": pb.RENDER_WAVEFRONT, "persistent": pb.RENDER_PERSISTENT}
BATCH_PIPELINES = {"fused": pb.PIPELINE_FUSED, "wavefront": pb.PIPELINE_WAVEFRONT, "paths": pb.PIPELINE_PATHS}

# batched-workload scene index -> rows the oracle renders (None: the whole frame)
C4_SCENES = {1: None, 3: (248, 264), 12: None, 21: (120, 136)}
# serving-pool scene index -> request (resolution, spp) and oracle rows
C5_SCENES = {5: (256, 4, (120, 136)), 22: (128, 16, None)}


def camera_of(rd):
    return dict(eye=tuple(rd.camera.eye), look_at=tuple(rd.camera.look_at), up=tuple(rd.camera.up),
                fov=rd.camera.fov_deg)


def desc_dict(rd, flags):
    return dict(width=rd.width, height=rd.height, spp=rd.spp, max_depth=rd.max_depth, seed=rd.seed,
                camera=camera_of(rd), flags=flags)


def band(a, rows):
    return a if rows is None else a[rows[0]:rows[1]]


@pytest.fixture(scope="module")
def c4():
    work = W.batched_workload(256)
    out = []
    for k, rows in C4_SCENES.items():
        meshes, env, d = work[k]
        scene = pb.Scene(meshes, env)
        flags = pb.RENDER_NEE | (pb.RENDER_JITTER if k % 2 else 0)
        rd = pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"], flags)
        o = po.OracleScene(meshes, env)
        orgb, oprim = o.render(desc_dict(rd, flags), rows=rows, threads=THREADS)
        out.append(dict(index=k, meshes=meshes, scene=scene, oracle=o, rd=rd, rows=rows, rgb=orgb, prim=oprim))
    yield out
    for c in out:
        c["oracle"].close()
        c["scene"].close()


@pytest.fixture(scope="module")
def c5():
    pool = W.serving_pool(32)
    out = []
    for k, (res, spp, rows) in C5_SCENES.items():
        meshes, env = pool[k]
        scene = pb.Scene(meshes, env)
        rd = pb.render_desc(res, res, spp, 5, W.SERVE_CAMERA, 100 + k, pb.RENDER_NEE)
        o = po.OracleScene(meshes, env)
        orgb, oprim = o.render(desc_dict(rd, pb.RENDER_NEE), rows=rows, threads=THREADS)
        out.append(dict(index=k, scene=scene, oracle=o, rd=rd, rows=rows, rgb=orgb, prim=oprim))
    yield out
    for c in out:
        c["oracle"].close()
        c["scene"].close()


def check_against_oracle(c, rgb, prim, what):
    rows = c["rows"]
    assert rgb.shape == (c["rd"].height, c["rd"].width, 3)
    assert_bit_equal(band(prim, rows), band(c["prim"], rows), f"{what}: primary ids")
    assert_bit_equal(band(rgb, rows), band(c["rgb"], rows), f"{what}: film")
    assert band(rgb, rows).mean() > 0.05, what


def render_with(c, flags):
    rd = c["rd"]
    return pb.render(c["scene"], rd.width, rd.height, rd.spp, rd.max_depth, camera_of(rd), rd.seed, rd.flags | flags)


@pytest.mark.parametrize("pipeline", list(PIPELINES), ids=list(PIPELINES))
def test_batched_workload_scenes_pt_render_match_oracle(cuda_device, c4, pipeline):
    for c in c4:
        rgb, prim = render_with(c, PIPELINES[pipeline])
        check_against_oracle(c, rgb, prim, f"C4 scene {c['index']} pt_render {pipeline}")


@pytest.mark.parametrize("pipeline", list(BATCH_PIPELINES), ids=list(BATCH_PIPELINES))
def test_batched_workload_scenes_in_one_batch_match_oracle(cuda_device, c4, pipeline):
    t = pb.default_tuning()
    t.pipeline = BATCH_PIPELINES[pipeline]
    b = pb.Batch([(c["scene"], c["rd"]) for c in c4], t)
    b.run()
    for i, c in enumerate(c4):
        rgb, prim = b.output(i)
        check_against_oracle(c, rgb, prim, f"C4 scene {c['index']} batch {pipeline}")
    b.close()


@pytest.mark.parametrize("pipeline", list(BATCH_PIPELINES), ids=list(BATCH_PIPELINES))
def test_batched_workload_scenes_served_match_oracle(cuda_device, c4, pipeline):
    t = pb.default_tuning()
    t.pipeline = BATCH_PIPELINES[pipeline]
    srv = pb.Server(max_inflight=16, wave_pixels=1 << 20, tuning=t)
    tickets = [srv.submit(c["scene"], c["rd"]) for c in c4]  # all in flight together
    for tk, c in zip(tickets, c4):
        assert srv.wait(tk, 120000) == 2
        rgb, prim = srv.fetch(tk)
        check_against_oracle(c, rgb, prim, f"C4 scene {c['index']} served {pipeline}")
    srv.close()


def test_box_scene_matches_reference_fixture(cuda_device):
    """The batched workload's scene 12 at its own 64x64, 64 spp, depth 6: the whole film and the
    primary ids equal the reference's patched render loop (fixture made by oracle/_ref), through
    pt_render under each pipeline and through a batch; rays aimed at its box corners and edge
    midpoints give the reference's hits and per-ray node and face test counts."""
    from golden.make_golden import BOX_SCENE_INDEX
    g = load_golden("batch_box_scene.npz")
    meshes, env, d = W.batched_workload(256)[BOX_SCENE_INDEX]
    scene = pb.Scene(meshes, env)
    for name, fl in PIPELINES.items():
        rgb, prim = pb.render(scene, d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                              pb.RENDER_NEE | fl)
        assert_bit_equal(rgb, g["rgb"], f"film {name}")
        assert_bit_equal(prim, g["prim"], f"prim {name}")
    b = pb.Batch([(scene, pb.render_desc(d["width"], d["height"], d["spp"], d["max_depth"], d["camera"], d["seed"],
                                         pb.RENDER_NEE))])
    b.run()
    assert_bit_equal(b.output(0)[0], g["rgb"], "batch film")
    b.close()
    hits, nt, tt = scene.intersect(g["rays"], counts=True)
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f], g["hits"][f], f)
    assert_bit_equal(nt, g["node_tests"], "node tests")
    assert_bit_equal(tt, g["tri_tests"], "face tests")


def test_box_edge_and_corner_rays_on_the_largest_batch_scene(cuda_device, c4):
    """Rays at exact box corners and edge midpoints of the 494,590-face scene (34,389 boxes), where
    Wald edge functions come out exactly zero and the emulated FP64 fallback decides; closest hits,
    any-hit outcomes and per-ray node/face test counts equal the oracle's."""
    from golden.make_golden import box_edge_rays
    c = next(c for c in c4 if c["index"] == 3)
    rays = box_edge_rays(c["meshes"][1], 40000, 20000, 71)
    anyhit = rays.copy()
    anyhit["flags"] = pb.RAY_ANY_HIT
    anyhit["tmax"] = 7.5
    rays = np.concatenate([rays, anyhit])
    hits, nt, tt = c["scene"].intersect(rays, counts=True)
    ohits, ont, ott = c["oracle"].trace(rays, counts=True)
    closest = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f][closest], ohits[f][closest], f)
    assert_bit_equal(nt[closest], ont[closest], "node tests")
    assert_bit_equal(tt[closest], ott[closest], "face tests")
    assert_bit_equal(hits["prim"][~closest] != pb.PRIM_NONE, ohits["prim"][~closest] != pb.PRIM_NONE, "any-hit")
    assert (hits["prim"][closest] != pb.PRIM_NONE).mean() > 0.3
    # the device-pointer path gives the same hits
    import torch
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda")
    c["scene"].intersect(d_rays, d_hits, device=True)
    torch.cuda.synchronize()
    assert d_hits.cpu().numpy().tobytes() == hits.tobytes()
    assert c["scene"].status() == pb.PT_OK


@pytest.mark.parametrize("pipeline", list(PIPELINES), ids=list(PIPELINES))
def test_serving_pool_scenes_pt_render_match_oracle(cuda_device, c5, pipeline):
    for c in c5:
        rgb, prim = render_with(c, PIPELINES[pipeline])
        check_against_oracle(c, rgb, prim, f"C5 scene {c['index']} pt_render {pipeline}")


@pytest.mark.parametrize("pipeline", list(BATCH_PIPELINES), ids=list(BATCH_PIPELINES))
def test_serving_pool_scenes_served_match_oracle(cuda_device, c5, c4, pipeline):
    """Requests on the two pool scenes in flight together with the batched scenes' requests."""
    t = pb.default_tuning()
    t.pipeline = BATCH_PIPELINES[pipeline]
    srv = pb.Server(max_inflight=16, wave_pixels=1 << 19, tuning=t)
    everything = c5 + c4
    tickets = [srv.submit(c["scene"], c["rd"]) for c in everything]
    for tk, c in zip(tickets, everything):
        assert srv.wait(tk, 120000) == 2
        rgb, prim = srv.fetch(tk)
        check_against_oracle(c, rgb, prim, f"scene {c['index']} served {pipeline}")
    srv.close()
