"""pt_render_noalloc: the render for callers that cannot allocate device memory during the call
(an application that owns the device-memory budget, or a frame loop that cannot pay cudaFree's
device-wide synchronisation).  It keeps its scratch in a fixed device array inside the library;
its films must equal pt_render's (tolerance: identical bits, well inside the relative RMSE
<= 1e-6 used by the other render tests), on consecutive calls that reuse that array.

This file is collected last on purpose, and passes both alone in a fresh process and after the
rest of the suite."""
import ctypes as C

import numpy as np
import pytest

import polytope_b200 as pb
from polytope_b200 import workloads as W

pytestmark = pytest.mark.gpu


def render_noalloc(scene, desc, torch, device):
    n = desc.width * desc.height
    rgb = torch.full((n * 3,), float("nan"), dtype=torch.float32, device=device)
    prim = torch.full((n,), 7, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)
    pb.check(pb.lib.pt_render_noalloc(scene.handle, C.byref(desc), rgb.data_ptr(), prim.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    return (rgb.cpu().numpy().reshape(desc.height, desc.width, 3),
            prim.cpu().numpy().view(np.uint32).reshape(desc.height, desc.width))


def test_noalloc_render_matches_pt_render_on_consecutive_calls(cuda_device):
    import torch
    meshes, env = W.small_scene(level=3)
    scene = pb.Scene(meshes, env)
    # calls in a row with different frames: each reuses (and must clear) the scratch; the last two
    # have more paths than one wave of the fixed array (262,144), so their waves loop over it
    frames = ((64, 48, 3, 1, pb.RENDER_NEE, 0), (40, 30, 2, 5, pb.RENDER_NEE | pb.RENDER_JITTER, 0),
              (256, 256, 8, 2, pb.RENDER_NEE, 0), (97, 61, 5, 3, pb.RENDER_NEE | pb.RENDER_FUSED, 7001))
    for (w, h, spp, seed, flags, wave) in frames:
        desc = pb.render_desc(w, h, spp, 4, W.SMALL_CAMERA, seed, flags, wave)
        got_rgb, got_prim = render_noalloc(scene, desc, torch, cuda_device)
        exp_rgb, exp_prim = pb.render(scene, w, h, spp, 4, W.SMALL_CAMERA, seed, flags)
        assert got_rgb.tobytes() == exp_rgb.tobytes(), (w, h, spp)
        assert got_prim.tobytes() == exp_prim.tobytes(), (w, h, spp)
        assert exp_rgb.mean() > 0
    assert scene.status() == pb.PT_OK


def test_noalloc_rejects_frames_above_its_limit(cuda_device):
    import torch
    meshes, env = W.small_scene(level=2)
    scene = pb.Scene(meshes, env)
    for (w, h) in ((1024, 1024), (600, 600), (512, 513)):
        out = torch.zeros(w * h * 3, dtype=torch.float32, device=cuda_device)  # a valid buffer, never written
        desc = pb.render_desc(w, h, 1, 2, W.SMALL_CAMERA)
        rc = pb.lib.pt_render_noalloc(scene.handle, C.byref(desc), out.data_ptr(), None, None)
        assert rc == pb.PT_EINVAL and "limit" in pb.last_error(), (w, h)
        assert float(out.abs().sum()) == 0.0
    # the other pipelines are refused, not silently replaced by the fused one
    out = torch.zeros(16 * 16 * 3, dtype=torch.float32, device=cuda_device)
    for fl in (pb.RENDER_PERSISTENT, pb.RENDER_WAVEFRONT):
        desc = pb.render_desc(16, 16, 1, 2, W.SMALL_CAMERA, 1, fl)
        assert pb.lib.pt_render_noalloc(scene.handle, C.byref(desc), out.data_ptr(), None, None) == pb.PT_EINVAL
    assert float(out.abs().sum()) == 0.0
