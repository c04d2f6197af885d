"""Host side of the two-level (instanced) scene layout: pt_two_level_plan runs the same host build
as pt_scene_create_two_level (geometry sharing, object-space trees with the reference SAH build, the
top-level tree) without a device."""
import numpy as np
import pytest

import polytope_b200 as pb
from polytope_b200 import workloads as W


def test_instanced_scene_shares_one_geometry():
    meshes, env = W.instanced_scene(level=4)
    plan = pb.two_level_plan(meshes, env)
    assert plan["num_instances"] == 7          # ground, five sphere instances, light
    assert plan["num_geometries"] == 3         # the five instances share the sphere
    sphere = len(meshes[1].faces)
    assert plan["blas_faces"] == sphere + 2 + 2
    assert plan["num_prims"] == sum(len(m.faces) for m in meshes)
    # each geometry's tree is the reference build of that mesh alone (object space: identity transform)
    alone = pb.Mesh(meshes[1].x, meshes[1].y, meshes[1].z, meshes[1].faces)
    nodes, _ = pb.bvh_build([alone])
    assert plan["blas_nodes"] >= len(nodes)
    assert plan["tlas_nodes"] == 2 * 7 - 1 and plan["tlas_depth"] <= 3


def test_memory_of_the_full_instanced_scene():
    meshes, env = W.instanced_scene()
    plan = pb.two_level_plan(meshes, env)
    flat_bytes = 32 * len(pb.bvh_build(meshes)[0]) + 48 * plan["num_prims"]
    assert flat_bytes / plan["device_bytes"] > 4.5, (flat_bytes, plan["device_bytes"])


def test_meshes_without_shared_arrays_are_their_own_geometries():
    meshes, env = W.small_scene(level=2)
    plan = pb.two_level_plan(meshes, env)
    assert plan["num_instances"] == plan["num_geometries"] == 3


def test_bad_inputs_are_refused():
    meshes, env = W.instanced_scene(level=2)
    proj = list(meshes)
    m = np.array(proj[1].object_to_world, np.float32)
    m[3, 0] = 0.5  # not affine
    proj[1] = pb.Mesh(proj[1].x, proj[1].y, proj[1].z, proj[1].faces, object_to_world=m)
    with pytest.raises(pb.PolytopeError) as e:
        pb.two_level_plan(proj, env)
    assert e.value.code == pb.PT_EINVAL and "affine" in str(e.value)
    sing = list(meshes)
    sing[1] = pb.Mesh(sing[1].x, sing[1].y, sing[1].z, sing[1].faces, object_to_world=np.diag([1, 0, 1, 1]).astype(np.float32),
                      world_to_object=np.eye(4, dtype=np.float32))  # singular: no inverse to carry rays with
    with pytest.raises(pb.PolytopeError):
        pb.two_level_plan(sing, env)
