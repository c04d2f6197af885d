// config.h -- compile-time limits shared by host and device code.
#pragma once

// Traversal stack entries per ray.  The reference's ordered DFS needs at most (tree depth + 1)
// entries; pt_scene_create records the depth and calls refuse trees that do not fit.
#define PT_TRAVERSAL_STACK 64
// Top-level stack entries of a two-level scene (pt_scene_create_two_level refuses deeper trees).
#define PT_TOP_STACK 64

// Warp rounds of the persistent walks (walk_round, traverse.cuh): the lanes of a warp take node
// steps together until this many of them hold a leaf or have ended their walk (32 = every walking
// lane), then test faces together; 0 walks each lane on its own to its next leaf instead (no vote,
// fewer live registers).  One value per kernel: the ray-query kernel, the persistent path kernel
// and the wavefront extend/shadow kernel.  Measured on a B200 (each against the per-lane walk):
// ray queries on the 1.3 M-face microbench 1722 -> 1985 Mrays/s at 16 (12: 1937, 24: slower);
// whole paths on the 6.5 M-face frame 1595 -> 1678 Msamples/s at 12 (8 and 16 slower); the
// wavefront kernel on the 256-scene batch 1806 -> 2024 Mrays/s at 12 with its first 16 stack
// entries in shared memory (16: 1954, 20: 1801; with the stack in local memory the vote lost 17 %
// at this kernel's 64 registers).
#ifndef PT_LEAF_BATCH_TRACE
#define PT_LEAF_BATCH_TRACE 16
#endif
#ifndef PT_LEAF_BATCH_PATHS
#define PT_LEAF_BATCH_PATHS 12
#endif
#ifndef PT_LEAF_BATCH_WAVEFRONT
#define PT_LEAF_BATCH_WAVEFRONT 12
#endif

// Persistent path kernel (wf_path_kernel): lanes whose ray has ended wait until this many lanes of
// the warp can shade together (or no lane still walks), and the resident-block floor given to the
// register allocator (blocks of 128 threads per SM).  With the lighter node steps (the box form
// chosen per warp round, sign-mask child order, paired pushes) 7 blocks (72 registers) overtook 8
// on a B200: the 6.5 M-face frame 1884-1888 against 1800-1805 Msamples/s, the saturated serving mix
// 4624 against 4411 Mrays/s (the 256-scene plain frames 1551 against 1567); 6 blocks (80
// registers) 1847 and 4574; shade batches of 12 or 24 measured 1706 / 1703 (at 8 blocks).
#ifndef PT_SHADE_BATCH_PATHS
#define PT_SHADE_BATCH_PATHS 16
#endif
#ifndef PT_PATH_MIN_BLOCKS
#define PT_PATH_MIN_BLOCKS 7
#endif
