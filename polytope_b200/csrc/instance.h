// instance.h -- the two-level scene layout (pt_scene_create_two_level): one bottom-level tree per
// distinct mesh geometry, in object space, and a top-level tree over the instances' world boxes.
//
// The reference has no such layout: pbrt_parser.cpp:1439-1472 turns every ObjectInstance into its
// own Mesh and bvh::bound (bvh.cpp:36-130) builds one world-space tree over all of them, baking
// each instance's vertices with Transform::ApplyInPlace.  The two-level mode keeps one copy of a
// shared geometry instead; rays are carried into each instance's object space for its bottom-level
// tree, so hits are not bit-identical to the flattened tree's (see pt_scene_create_two_level).
#pragma once

#include <cstdint>

namespace pt {

struct DeviceInstance {  // 128 B
    float w2o[12];        // world -> object, rows of the 3x4 affine inverse of object_to_world
    float o2w[16];        // the mesh's object_to_world (row-major), applied as Transform::ApplyInPlace
    uint32_t node_base;   // root of the instance's bottom-level tree in the shared node array
    uint32_t face_base;   // first leaf-ordered face record of that tree
    uint32_t prim_base;   // global primitive id of the mesh's face 0 (the flattened scene's ids)
    uint32_t mesh;        // mesh index (shading record, emission)
};
static_assert(sizeof(DeviceInstance) == 128, "instance records are 128 bytes");

}  // namespace pt
