// config.h -- compile-time limits shared by host and device code.
#pragma once

// Traversal stack entries per ray.  The reference's ordered DFS needs at most (tree depth + 1)
// entries; pt_scene_create records the depth and calls refuse trees that do not fit.
#define PT_TRAVERSAL_STACK 64
