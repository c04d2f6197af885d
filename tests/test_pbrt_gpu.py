"""A PBRT scene read by pt_load_pbrt renders on the GPU exactly as the CPU oracle renders the same
meshes, camera and settings; a shape without a material is refused by pt_scene_create."""
import numpy as np
import pytest

from conftest import assert_bit_equal
import polytope_b200 as pb
from oracle import pyoracle as po
from test_pbrt_cpu import write_assets, write_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pipeline", [pb.RENDER_FUSED, pb.RENDER_WAVEFRONT, pb.RENDER_PERSISTENT], ids=["fused", "wavefront", "persistent"])
def test_pbrt_scene_renders_like_the_oracle(cuda_device, tmp_path, pipeline):
    s = pb.load_pbrt(write_scene(tmp_path))
    scene = pb.Scene(s.meshes, s.env)
    rgb, prim = pb.render(scene, s.width, s.height, s.spp, s.max_depth, s.camera, seed=5, flags=pb.RENDER_NEE | pipeline)
    orgb, oprim = po.OracleScene(s.meshes, s.env).render(dict(s.render_args(), seed=5, flags=1))
    assert_bit_equal(prim, oprim, "primary ids")
    assert_bit_equal(rgb, orgb, "film")
    assert rgb.mean() > 0.5 and (prim != pb.PRIM_NONE).mean() > 0.3


def test_shape_without_material_is_refused(cuda_device, tmp_path):
    write_assets(tmp_path)
    (tmp_path / "s.pbrt").write_text('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\n'
                                     'Shape "plymesh" "string filename" [ "quad.ply" ]\nWorldEnd\n')
    s = pb.load_pbrt(tmp_path / "s.pbrt")
    assert s.meshes[0].material == 0
    with pytest.raises(pb.PolytopeError) as e:
        pb.Scene(s.meshes, s.env)
    assert e.value.code == pb.PT_EINVAL
