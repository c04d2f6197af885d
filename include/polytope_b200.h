/*
 * polytope_b200.h — C ABI of the B200 (sm_100a) ray/path-tracing hot path.
 *
 * This header is the drop-in boundary for Polytope's CPU render call.  The reference has no
 * plugin/FFI layer; its boundary is a set of C++ classes.  Each entry point below names the
 * reference interface it replaces (paths are relative to the Polytope source tree):
 *
 *   pt_bvh_build      <- poly::bvh::bound + poly::bvh::compact      src/cpu/acceleration/bvh.cpp:36-395, 652-698
 *   pt_scene_create   <- poly::Scene (Shapes, Lights, Skybox, bvh_root) after compact()
 *                                                                   src/cpu/scenes/Scene.h:17-35
 *   pt_trace          <- poly::Scene::intersect -> bvh::intersect_compact -> Mesh::intersect
 *                                                                   src/cpu/scenes/Scene.cpp:12-31,
 *                                                                   src/cpu/acceleration/bvh.cpp:476-523,
 *                                                                   src/cpu/shapes/mesh.cpp:161-355
 *   pt_render         <- spawn N x AbstractRunner::Run + join + Output()
 *                        (TileRunner::Run -> AbstractRunner::Trace -> PathTraceIntegrator::GetSample)
 *                                                                   src/cpu/main.cpp:187-220,
 *                                                                   src/cpu/runners/TileRunner.cpp:77-117,
 *                                                                   src/cpu/runners/AbstractRunner.cpp:11-31,
 *                                                                   src/cpu/integrators/PathTraceIntegrator.cpp:10-135
 *   pt_render_rgba8   <- the same, then Output()'s PNGFilm quantisation src/cpu/films/PNGFilm.cpp:20-45
 *   pt_load_ply / pt_load_obj / pt_load_pbrt, pt_film_to_rgba8 / pt_write_png
 *                     <- the scene readers and the PNG output step (declared below with their citations)
 *
 * Entry points with no counterpart in the reference (one frame per process, no instancing layout,
 * errors end the process): pt_scene_status, pt_render_noalloc, pt_scene_create_two_level,
 * pt_two_level_plan, pt_batch_*, pt_tuning_*, pt_server_* (pt_server_cancel among them).
 *
 * Conventions
 *   - Every function returns PT_OK (0) or a negative PT_E* status and never exits the process
 *     (the reference calls exit(1) from ERROR, src/common/utilities/Common.h:13).  The message of
 *     the last failure on the calling thread is returned by pt_last_error().
 *   - Scene handles are immutable after pt_scene_create; concurrent pt_trace / pt_render calls on
 *     one handle from several host threads (on different streams) are safe.
 *   - `stream` arguments are cudaStream_t values passed as void* (NULL = legacy default stream).
 *   - There is no CPU fallback: without a usable CUDA device every call that launches work
 *     returns PT_ECUDA.
 */
#ifndef POLYTOPE_B200_H
#define POLYTOPE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define PT_OK        0
#define PT_EINVAL   (-1)   /* bad argument, malformed tree, size out of range              */
#define PT_ENOMEM   (-2)   /* host or device allocation failed                             */
#define PT_ETIMEOUT (-3)   /* a bounded device wait ran out                                */
#define PT_ECUDA    (-4)   /* CUDA runtime error or no device                              */
#define PT_ESTACK   (-5)   /* traversal stack capacity exceeded (tree deeper than capacity) */
#define PT_ECANCELED (-6)  /* the served request was cancelled (pt_server_cancel)           */

/* ---- geometry ---------------------------------------------------------------------------- */

/* One compacted BVH node, byte-identical to poly::compact_bvh_node (src/cpu/acceleration/bvh.h:24-53):
 * bounding box p0,p1 (24 B), a union of high_child_offset (interior: the high child sits at
 * this index + offset; the low child at this index + 1) and face_index_offset (leaf: first entry
 * of the leaf-ordered face list), num_faces (0 for interior nodes) and the split axis. */
typedef struct pt_bvh_node {
    float    bb_min[3];
    float    bb_max[3];
    uint32_t offset;
    uint16_t num_faces;
    uint16_t axis;
} pt_bvh_node;

/* Materials (src/cpu/shading/brdf/abstract_brdf.h:15-20 BRDF_TYPE; Lambert = 1, Mirror = 2). */
#define PT_MAT_LAMBERT 1u
#define PT_MAT_MIRROR  2u

/* One mesh instance: poly::Mesh + poly::mesh_geometry (src/cpu/shapes/mesh.h:17-113).
 * Vertices are the *packed* arrays (x_packed...) indexed by fv0/fv1/fv2.  object_to_world is the
 * row-major 4x4 poly::Transform::Matrix; world_to_object its Inverse (used only for vertex
 * normals, src/cpu/structures/Transform.cpp:135-143).  A mesh with is_light != 0 is an area
 * emitter (poly::Mesh::spd, mesh.h:99-109); emission is in the reference's x255 domain. */
typedef struct pt_mesh_desc {
    const float    *x, *y, *z;          /* packed vertex positions, num_vertices each          */
    uint32_t        num_vertices;
    const uint32_t *fv0, *fv1, *fv2;    /* per-face vertex indices, num_faces each             */
    uint32_t        num_faces;
    const float    *nx, *ny, *nz;       /* optional packed vertex normals (NULL if none)        */
    float           object_to_world[16];
    float           world_to_object[16];
    uint32_t        material;           /* PT_MAT_LAMBERT or PT_MAT_MIRROR                      */
    float           albedo[3];          /* Lambert reflectance or mirror Kr                     */
    int32_t         is_light;
    float           emission[3];
} pt_mesh_desc;

/* A scene: meshes in poly::Scene::Shapes order plus an optional constant environment
 * (poly::ColorSkybox, src/cpu/scenes/skyboxes/ColorSkybox.cpp:8-10).  If `nodes` is non-NULL the
 * caller passes the tree its own poly::bvh::compact() produced (nodes + leaf_ordered_indices as
 * (mesh, face) uint32 pairs); otherwise pt_scene_create builds it with pt_bvh_build. */
typedef struct pt_scene_desc {
    const pt_mesh_desc *meshes;
    uint32_t            num_meshes;
    const pt_bvh_node  *nodes;          /* optional */
    uint32_t            num_nodes;
    const uint32_t     *leaf_pairs;     /* optional, 2 * (total faces) entries                  */
    int32_t             has_env;
    float               env[3];
} pt_scene_desc;

typedef struct pt_scene pt_scene;

/* Global primitive ids: the faces of mesh m are numbered prim_base[m] + face, with prim_base the
 * exclusive prefix sum of num_faces in mesh order (the order of poly::bvh::master_indices,
 * bvh.cpp:45-118). */
#define PT_PRIM_NONE 0xFFFFFFFFu

/* Build the reference's SAH BVH (12-bucket binned SAH, BFS, bvh.cpp:36-395) and DFS-compact it
 * (bvh.cpp:652-698) on the host.  The result is node-for-node and byte-for-byte identical to the
 * reference.  nodes_out must hold *num_nodes_out entries on input (query the count first with
 * nodes_out == NULL); leaf_pairs_out must hold 2 * total faces entries.  threads <= 0 = all cores. */
int pt_bvh_build(const pt_mesh_desc *meshes, uint32_t num_meshes, int threads,
                 pt_bvh_node *nodes_out, uint32_t *num_nodes_out, uint32_t *leaf_pairs_out);

/* Upload a scene to the current CUDA device.  The descriptor's arrays are copied; the caller may
 * free them on return. */
int pt_scene_create(const pt_scene_desc *desc, pt_scene **out);
/* Two-level (instanced) scene: an opt-in layout with no counterpart in the reference, which
 * flattens every ObjectInstance into its own world-space mesh and one tree
 * (src/common/parsers/pbrt_parser.cpp:1439-1472, bvh::bound src/cpu/acceleration/bvh.cpp:36-130).
 * Meshes of `desc` whose vertex, face and normal arrays are the same pointers with the same counts
 * share one geometry: it is stored once, in object space, with its own tree (the same SAH build);
 * each mesh becomes an instance with its object_to_world (affine and invertible), and a top-level
 * tree over the instances' world boxes picks the instances a ray reaches.  Rays are carried into
 * object space for the bottom-level tests, so hits are those of the flattened scene up to float
 * rounding: primitive ids agree wherever the first hit is unambiguous, t to about 1e-6 relative,
 * and images agree in RMSE rather than bit for bit.  Shading uses the instance's world vertices
 * computed as pt_scene_create bakes them.  Primitive ids, materials, lights and the environment
 * are the flattened scene's.  The scene works with pt_trace / pt_trace_counted (node counts then
 * include top-level tests), pt_render and pt_render_rgba8 with the fused (default for such scenes)
 * and persistent pipelines (PT_RENDER_WAVEFRONT is rejected), pt_render_noalloc, and batches and
 * servers with PT_PIPELINE_PATHS or PT_PIPELINE_FUSED; every route gives the same film bit for bit.
 * `desc->nodes` must be NULL; the top-level and bottom-level depths together must leave room in
 * the traversal stack (PT_ESTACK otherwise). */
int pt_scene_create_two_level(const pt_scene_desc *desc, pt_scene **out);

/* What pt_scene_create_two_level would build from `desc`, computed on the host alone (no device
 * needed): counts and the device bytes the scene would hold. */
typedef struct pt_two_level_info {
    uint32_t num_instances, num_geometries;
    uint32_t blas_nodes, blas_faces;    /* bottom-level trees and faces, all geometries   */
    uint32_t tlas_nodes;
    uint32_t max_depth, tlas_depth;      /* deepest bottom-level and top-level node         */
    uint32_t num_prims;                  /* faces of the flattened scene (primitive ids)    */
    uint64_t device_bytes;
} pt_two_level_info;
int pt_two_level_plan(const pt_scene_desc *desc, pt_two_level_info *info);

int pt_scene_destroy(pt_scene *scene);

typedef struct pt_scene_info {
    uint32_t num_nodes;
    uint32_t num_prims;
    uint32_t num_meshes;
    uint32_t max_depth;            /* deepest node level (root = 0)                           */
    uint64_t device_bytes;         /* device memory held by the handle                        */
} pt_scene_info;
int pt_scene_get_info(const pt_scene *scene, pt_scene_info *info);

/* ---- ray queries (Scene::intersect) ------------------------------------------------------ */

/* A ray: origin, tmax (poly::Ray::MinT at entry, INFINITY for an unbounded closest-hit query),
 * direction (not required to be normalized) and flags. */
typedef struct pt_ray {
    float    org[3];
    float    tmax;
    float    dir[3];
    uint32_t flags;
} pt_ray;
#define PT_RAY_ANY_HIT 1u   /* stop at the first accepted triangle (shadow query)            */

/* Result: prim = global primitive id of the committed triangle (PT_PRIM_NONE on a miss);
 * t = final poly::Ray::MinT (= tmax on a miss); u, v = the committed barycentrics
 * (poly::Intersection::u, v; mesh.cpp:302-303,338-339).  For an any-hit ray the fields describe
 * the first accepted triangle. */
typedef struct pt_hit {
    uint32_t prim;
    float    t;
    float    u;
    float    v;
} pt_hit;

#define PT_MEM_DEVICE 1u   /* rays/hits (or film) pointers are device pointers               */

/* Trace n rays.  Closest-hit rays reproduce bvh::intersect_compact exactly (same node order, same
 * Wald arithmetic, same tie-breaking); any-hit rays return whether that closest-hit query would
 * have found any hit.  With PT_MEM_DEVICE the call is asynchronous on `stream`; with host
 * pointers it stages through the handle's pinned buffers, overlaps the copies with the kernels
 * and returns when the hits are on the host. */
int pt_trace(pt_scene *scene, const pt_ray *rays, uint64_t n, pt_hit *hits,
             uint32_t mem_flags, void *stream);

/* Same traversal, also writing per-ray counts of node box tests (poly::Intersection::num_bb_hits +
 * num_bb_misses) and triangle tests (num_triangle_isects), bvh.cpp:495,502,520.  Pointers follow
 * mem_flags; counts may be NULL.  Used for the algorithmic-bytes accounting and order checks. */
int pt_trace_counted(pt_scene *scene, const pt_ray *rays, uint64_t n, pt_hit *hits,
                     uint32_t *node_tests, uint32_t *tri_tests, uint32_t mem_flags, void *stream);

/* Launch shape of the ray-query kernel (per scene).  shared_stack: traversal-stack entries per
 * lane kept in shared memory (0, 8, 16, 24 or 32; the rest stays in local memory); queue_chunk: rays a
 * warp takes per fetch (multiple of 32).  Results do not depend on it. */
typedef struct pt_trace_tuning {
    uint32_t shared_stack;
    uint32_t queue_chunk;
} pt_trace_tuning;
int pt_scene_set_trace_tuning(pt_scene *scene, const pt_trace_tuning *tuning);
int pt_scene_get_trace_tuning(const pt_scene *scene, pt_trace_tuning *tuning);
/* Times the candidate shapes on the given device rays (CUDA events, fastest of five launches
 * after a warm-up, one knob at a time), keeps the fastest on the scene and returns it. */
int pt_trace_autotune(pt_scene *scene, const pt_ray *rays_dev, uint64_t n, pt_hit *hits_dev,
                      pt_trace_tuning *best, float *best_ms);

/* ---- rendering (the CPU render call) ----------------------------------------------------- */

/* Pinhole camera as built by the PBRT "LookAt" + "Camera perspective" directives
 * (src/common/parsers/pbrt_parser.cpp:1099-1171, Transform::LookAt Transform.cpp:322-365,
 * PerspectiveCamera.cpp:17-49, left-handed = true). */
typedef struct pt_camera {
    float eye[3];
    float look_at[3];
    float up[3];
    float fov_deg;
} pt_camera;

#define PT_RENDER_NEE        1u   /* area-light next-event estimation with shadow rays       */
#define PT_RENDER_JITTER     2u   /* jittered pixel samples (default: pixel centres, the
                                     reference CenterSampler, samplers.cpp:13-18)             */
#define PT_RENDER_WAVEFRONT  4u   /* queue-based wavefront kernels                             */
#define PT_RENDER_PERSISTENT 8u   /* one persistent path kernel per wave whose lanes take the
                                     next path as soon as theirs ends: the default pipeline     */
#define PT_RENDER_FUSED     16u   /* one thread per path, one launch per wave (the simplest
                                     form); the three pipeline flags exclude each other        */

typedef struct pt_render_desc {
    uint32_t  width, height;
    uint32_t  spp;
    uint32_t  max_depth;          /* PathTraceIntegrator::MaxDepth                           */
    uint64_t  seed;               /* counter-RNG key                                         */
    uint32_t  flags;              /* PT_RENDER_*                                             */
    uint32_t  wave_paths;         /* paths per wave (0 = automatic)                           */
    pt_camera camera;
} pt_render_desc;

/* Render one frame (replaces AbstractRunner::Run on N threads + Output, src/cpu/main.cpp:187-220,
 * AbstractRunner.cpp:11-31).  rgb_out: width*height*3 floats, the box-filtered film (per-sample
 * clamp to 255 then the mean, BoxFilter.cpp:14-71) before PNG quantization.  primary_prim_out
 * (optional): width*height global primitive ids hit by sample 0's camera ray (PT_PRIM_NONE on a
 * miss).  Every pipeline gives the same film bit for bit; without a pipeline flag the persistent
 * path kernel runs.  Pointers follow mem_flags:
 *   - host pointers: the call returns when the film is on the host, and reports PT_ESTACK if one
 *     of its own paths met a traversal guard;
 *   - PT_MEM_DEVICE: the call only queues the work on `stream` (its temporaries return to a
 *     stream-ordered pool behind it) and returns; a guard failure raises the scene's device flag,
 *     which pt_scene_status reports. */
int pt_render(pt_scene *scene, const pt_render_desc *desc, float *rgb_out,
              uint32_t *primary_prim_out, uint32_t mem_flags, void *stream);

/* The render call followed by the reference's PNG output step on the device: the frame of
 * pt_render, quantised as PNGFilm::Output stores it (src/cpu/films/PNGFilm.cpp:20-45; see
 * pt_film_to_rgba8), so only width*height*4 bytes leave the device instead of the 12-byte float
 * film.  rgba_out: width*height*4 bytes; primary_prim_out as in pt_render (optional).  Pointers
 * follow mem_flags with pt_render's semantics (host: returns when the bytes are there and reports
 * its own guard failures; PT_MEM_DEVICE: queued on `stream`, guard failures in pt_scene_status). */
int pt_render_rgba8(pt_scene *scene, const pt_render_desc *desc, uint8_t *rgba_out,
                    uint32_t *primary_prim_out, uint32_t mem_flags, void *stream);

/* Waits for `stream`, then reports (PT_ESTACK) and clears the scene's device error flag: set when
 * a kernel of an asynchronous call on this scene (pt_render or pt_trace with PT_MEM_DEVICE,
 * pt_render_noalloc, pt_batch_run, served requests) met a traversal guard since the last report.
 * Host-memory pt_render / pt_trace calls report their own guard failures and leave it alone.  The
 * guards are a stack deeper than the host checked or a node index outside the tree; a scene built
 * by pt_scene_create (which validates the tree) does not reach them.  No counterpart in the
 * reference (its errors call exit, src/common/utilities/Common.h:13). */
int pt_scene_status(pt_scene *scene, void *stream);

/* Same render as pt_render, for callers that cannot allocate device memory during the call: an
 * application that owns the whole device-memory budget and forbids allocations after start-up,
 * or a per-frame loop that cannot afford the device-wide synchronisation of cudaFree.  No
 * counterpart in the reference.  The scratch (film sums and one wave of path radiance) lives in a
 * fixed 6 MiB device array inside the library instead of being allocated per call.
 *   - rgb_dev (width*height*3 floats) and primary_dev (width*height ids, optional) are DEVICE
 *     pointers owned by the caller; the call is asynchronous on `stream`.
 *   - At most 262,144 pixels (e.g. 512x512) per frame and 262,144 paths per wave (larger frames
 *     run in several waves); larger frames are rejected with PT_EINVAL.  It always runs the fused
 *     pipeline: PT_RENDER_WAVEFRONT and PT_RENDER_PERSISTENT are rejected with PT_EINVAL.
 *   - A traversal guard failure in its kernels raises the scene's device flag, like every
 *     asynchronous call: pt_scene_status (after the frame) reports it.
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 *     that device current; make that first call before any stream capture.  The address is kept
 *     for the life of the process, so cudaDeviceReset must not be called while the library is in
 *     use (it would also free every scene).
 *   - Every call shares the array and it keeps the previous call's contents (the film sums are
 *     cleared at the start of each call): calls that overlap on the GPU (different streams, or
 *     different host threads) race and must be serialised by the caller.
 *   - The call calls no cudaMalloc, cudaFree or allocating library routine. */
int pt_render_noalloc(pt_scene *scene, const pt_render_desc *desc, float *rgb_dev,
                      uint32_t *primary_dev, void *stream);

/* ---- scene ingest ------------------------------------------------------------------------- */

/* A mesh read from a file: packed vertex arrays and faces, the shape pt_mesh_desc takes (and the
 * reference's mesh_geometry x/y/z_packed, nx/ny/nz_packed, u/v_packed, fv0/fv1/fv2, mesh.h:37-62).
 * Arrays are owned by the library; release them with pt_mesh_data_free. */
typedef struct pt_mesh_data {
    float    *x, *y, *z;
    uint32_t  num_vertices;
    uint32_t *fv0, *fv1, *fv2;
    uint32_t  num_faces;
    float    *nx, *ny, *nz;   /* NULL when the file has no vertex normals */
    float    *u, *v;          /* NULL when the file has no vertex uv */
} pt_mesh_data;

/* ply_parser::parse_file (src/common/parsers/mesh_parsers.cpp:336-545): ascii and binary PLY.
 * Header errors and malformed data return PT_EINVAL with the reason. */
int pt_load_ply(const char *path, pt_mesh_data *out);
/* obj_parser::parse_file (src/common/parsers/mesh_parsers.cpp:547-598): Wavefront OBJ as the
 * reference reads it -- every line whose first word starts with 'v' (vn and vt too) adds a vertex,
 * every line starting with 'f' adds one triangle from its first three indices (the leading integer
 * of each word, 1-based); other lines are ignored.  Unreadable numbers and indices outside the
 * vertices return PT_EINVAL with the reason.  Release with pt_mesh_data_free. */
int pt_load_obj(const char *path, pt_mesh_data *out);
void pt_mesh_data_free(pt_mesh_data *mesh);

/* poly::pbrt_parser::parse_file (src/common/parsers/pbrt_parser.cpp:284-1711): a PBRT scene file
 * read into the descriptions pt_scene_create and pt_render take.  Meshes come in the reference's
 * poly::Scene::Shapes order with the transforms, materials and radiances the reference ends up
 * with (including its in-place updates of a scope's transform and area light, the x255 radiance
 * scale, the UV sphere tessellation of Shape "sphere" and ObjectBegin / ObjectInstance); plymesh
 * paths are relative to the scene file.  Defaults as the reference's: 640x360, 8 samples, depth 5,
 * field of view 90.  Supported: Sampler, Film "image", PixelFilter, Camera "perspective" set by at
 * most one LookAt (none: the identity camera, returned as LookAt (0,0,0) (0,0,1) (0,1,0), the same
 * matrix), Integrator "path", AttributeBegin/End, TransformBegin/End, Translate, Scale, Rotate,
 * Transform, Material "matte" / "mirror", MakeNamedMaterial / NamedMaterial, AreaLightSource
 * "diffuse", LightSource "infinite", Shape "plymesh" / "objmesh" / "sphere", ObjectBegin / ObjectEnd /
 * ObjectInstance, Shape "objmesh" (pt_load_obj).  Textures, Material "plastic" and other camera
 * transforms are rejected with PT_EINVAL and the reason; like the reference, other unknown directives are skipped.
 * A shape with neither a material nor an area light comes back with material 0, which
 * pt_scene_create rejects.  The mesh descriptions point into arrays owned by the handle
 * (instances share them) and stay valid until pt_pbrt_free. */
typedef struct pt_pbrt_scene pt_pbrt_scene;
typedef struct pt_pbrt_info {
    uint32_t  num_meshes;
    int32_t   has_env;          /* LightSource "infinite" seen; env = its L x 255               */
    float     env[3];
    uint32_t  width, height;    /* Film "image" xresolution / yresolution                       */
    uint32_t  spp;              /* Sampler pixelsamples                                          */
    uint32_t  max_depth;        /* Integrator "path" maxdepth                                    */
    pt_camera camera;           /* LookAt eye / look-at / up, Camera "perspective" fov           */
} pt_pbrt_info;
int pt_load_pbrt(const char *path, pt_pbrt_scene **out);
int pt_pbrt_get_info(const pt_pbrt_scene *scene, pt_pbrt_info *info);
int pt_pbrt_get_meshes(const pt_pbrt_scene *scene, const pt_mesh_desc **meshes);
void pt_pbrt_free(pt_pbrt_scene *scene);

/* ---- output format ------------------------------------------------------------------------ */

/* The film as the reference's PNG output stores it: RGBA8, row-major, each channel
 * (unsigned char)(v > 255 ? 255 : v) (truncation), alpha 255 -- PNGFilm::Output
 * (src/cpu/films/PNGFilm.cpp:20-45) and OutputPNG::Output (src/cuda/png_output.cpp:29-36).
 * Replaces the float-film download with 4 bytes per pixel.  rgb: width*height*3 floats on the
 * device (a film from pt_render / pt_batch_output with PT_MEM_DEVICE); rgba_out: width*height*4
 * bytes, host (the call returns when they are there) or device with PT_MEM_DEVICE (asynchronous
 * on `stream`).  Films are non-negative; the reference's cast is undefined for negative or NaN
 * values, which map to 0 here. */
int pt_film_to_rgba8(const float *rgb_dev, uint32_t width, uint32_t height, uint8_t *rgba_out,
                     uint32_t mem_flags, void *stream);

/* Writes RGBA8 pixels (host memory) as a PNG file (8-bit RGBA, no interlace, zlib stream of
 * stored blocks).  The decoded pixels equal what lodepng::encode writes for the same data in the
 * reference (PNGFilm.cpp:50); the compressed bytes differ. */
int pt_write_png(const char *path, const uint8_t *rgba, uint32_t width, uint32_t height);

/* ---- batched renders (many uneven scenes in one persistent, graph-captured launch) -------- */

/* One render of a batch.  The batch keeps its own device films; read them with pt_batch_output. */
typedef struct pt_batch_item {
    pt_scene      *scene;
    pt_render_desc desc;              /* no pipeline flags: the batch tuning picks the pipeline  */
} pt_batch_item;

/* Launch shape of a batch (chosen by pt_batch_autotune).
 *   PT_PIPELINE_FUSED:     one persistent kernel; a lane traces every sample of a pixel, then
 *                          takes the next pixel of any render (wave_pixels: pixels per launch).
 *   PT_PIPELINE_WAVEFRONT: waves of paths of all renders; per bounce a persistent extend kernel,
 *                          a shade kernel appending to ray / shadow queues, a persistent shadow
 *                          kernel (wave_pixels: paths per wave).
 *   PT_PIPELINE_PATHS:     waves of paths of all renders as in PT_PIPELINE_WAVEFRONT, but one
 *                          thread runs a whole path (pt_render's fused kernel over several
 *                          renders at once; wave_pixels: paths per wave). */
#define PT_PIPELINE_FUSED     0u
#define PT_PIPELINE_WAVEFRONT 1u
#define PT_PIPELINE_PATHS     2u
typedef struct pt_batch_tuning {
    uint64_t wave_pixels;             /* work per launch / wave; 0 = automatic                    */
    uint32_t threads_per_block;       /* 64, 128 or 256                                           */
    uint32_t stack_depth;             /* traversal stack entries (24/32/48/64; 0 = smallest fit)   */
    uint32_t queue_chunk;             /* pixels or rays a warp takes per fetch (multiple of 32)   */
    uint32_t pipeline;                /* PT_PIPELINE_*                                            */
} pt_batch_tuning;

typedef struct pt_batch_tune_result {
    pt_batch_tuning tuning;
    float           ms;               /* time of one batch replay                                  */
} pt_batch_tune_result;

typedef struct pt_batch pt_batch;

/* Renders several frames of possibly different scenes, resolutions, spp and depths in persistent
 * launches that share the GPU pixel by pixel (a lane traces all samples of one pixel, in sample
 * order, then takes the next pixel of any render).  Every film equals pt_render's bit for bit.
 * The launch sequence is captured once into a CUDA graph; pt_batch_run replays it.  Replaces
 * running the reference's render call once per scene (src/cpu/main.cpp:187-220). */
int pt_batch_default_tuning(pt_batch_tuning *tuning);
int pt_batch_create(const pt_batch_item *items, uint32_t n, const pt_batch_tuning *tuning, pt_batch **out);
/* stream == NULL: run on the batch's own stream and wait; otherwise enqueue on `stream`. */
int pt_batch_run(pt_batch *batch, void *stream);
/* Host copies of item i's film / primary ids (either may be NULL) and the rays traced (camera,
 * bounce and shadow rays) by the last run of the whole batch. */
int pt_batch_output(pt_batch *batch, uint32_t i, float *rgb_out, uint32_t *primary_out, uint64_t *rays_traced);
int pt_batch_destroy(pt_batch *batch);
/* Coordinate descent over threads per block, queue chunk, stack depth and wave size, timing each
 * candidate on the given items (CUDA events, mean of two graph replays after a warm-up).
 * results (optional) receives up to *num_results timed candidates. */
int pt_batch_autotune(const pt_batch_item *items, uint32_t n, pt_batch_tuning *best, double *best_ms,
                      pt_batch_tune_result *results, uint32_t *num_results);

/* ---- autotuner cache (no counterpart in the reference) ------------------------------------ */

/* The class of a batch that a cached tuning is reused for: the device and the workload's scale.
 * Two batches of one class share a tuning; the sizes are bucketed by powers of two. */
typedef struct pt_tuning_class {
    char     device[64];          /* cudaDeviceProp::name, NUL-terminated                       */
    uint32_t sm_count;
    uint32_t compute_capability;  /* major * 10 + minor                                          */
    uint32_t items_log2;          /* floor(log2(number of renders))                              */
    uint32_t pixels_log2;         /* floor(log2(sum of width * height))                          */
    uint32_t samples_log2;        /* floor(log2(sum of width * height * spp))                    */
    uint32_t faces_log2;          /* floor(log2(faces of the distinct scenes))                   */
    uint32_t tree_depth;          /* deepest tree level of the scenes (decides the stacks that fit) */
    uint32_t max_depth;           /* largest path depth                                          */
    uint32_t flags;               /* OR of the renders' PT_RENDER_* flags                        */
} pt_tuning_class;

/* The class of a batch (the scenes' device must be present: PT_ECUDA otherwise). */
int pt_tuning_class_of(const pt_batch_item *items, uint32_t n, pt_tuning_class *cls);
/* Looks a class up in the JSON cache file at `path`: *found = 1 and the stored tuning and time,
 * or *found = 0 (also when the file does not exist).  A file that is not a tuning cache, or holds
 * an entry whose values pt_batch_create would refuse, returns PT_EINVAL with the reason. */
int pt_tuning_cache_get(const char *path, const pt_tuning_class *cls, pt_batch_tuning *tuning, double *ms,
                        int *found);
/* Stores (or replaces) the class's entry.  Safe against concurrent writers in other threads and
 * processes (an exclusive flock on "<path>.lock", then a temporary file renamed over the old one);
 * a file that is not a tuning cache is left untouched and reported with PT_EINVAL. */
int pt_tuning_cache_put(const char *path, const pt_tuning_class *cls, const pt_batch_tuning *tuning, double ms);
/* pt_batch_autotune through the cache: the stored tuning of the batch's class when there is one
 * (*from_cache = 1, no timing runs), otherwise the search, whose result is stored before return.
 * If storing fails, *best is still set and the call returns the file's error. */
int pt_batch_autotune_cached(const pt_batch_item *items, uint32_t n, const char *path, pt_batch_tuning *best,
                             double *best_ms, int *from_cache);

/* ---- serving loop (continuous batching of render requests over resident scenes) ----------- */

/* Wave policies of the serving loop. */
#define PT_SERVE_OLDEST_FIRST 0u  /* each wave is filled from the oldest admitted requests first      */
#define PT_SERVE_FAIR_SHARE   1u  /* each wave gives every admitted request an equal share            */

typedef struct pt_server_config {
    uint32_t        max_inflight;     /* requests admitted at once                                 */
    uint64_t        memory_budget;    /* device bytes for admitted requests' films (0 = 80 % of
                                         the memory free when the server is created)             */
    uint64_t        wave_pixels;      /* work per wave: pixels (PT_PIPELINE_FUSED) or paths (others) */
    pt_batch_tuning tuning;
    uint32_t        policy;           /* PT_SERVE_OLDEST_FIRST or PT_SERVE_FAIR_SHARE              */
    uint64_t        host_budget;      /* pinned host bytes for finished films not yet fetched
                                         (0 = 1 GiB); admission waits while it is full           */
} pt_server_config;

typedef struct pt_server_stats {
    uint64_t waves, completed, rays_traced;
    double   busy_ms;                 /* GPU time of the waves (CUDA events)                       */
    uint64_t pending, active, device_bytes_in_use;
    double   blocked_ms;              /* scheduler time with requests queued but no room to admit
                                         them (in-flight limit, device budget or host arena)    */
    uint64_t host_bytes_in_use;       /* host arena bytes held by finished, unfetched films      */
    double   plan_ms;                 /* scheduler time admitting, planning and enqueueing waves  */
    double   retire_wait_ms;          /* scheduler time waiting for waves and their film copies   */
    uint64_t waves_launched;          /* waves enqueued (waves counts retired ones)               */
    uint64_t cancelled;               /* requests ended by pt_server_cancel                       */
} pt_server_stats;

typedef struct pt_server pt_server;

/* A scheduler thread admits queued requests while max_inflight and the memory budget allow and
 * runs waves that take work from the admitted requests by the configured policy, so requests
 * arriving while others run join the next wave.  Two waves stay queued on the GPU while the host
 * plans the next one and copies finished films out.  Request states: 0 queued, 1 admitted,
 * 2 done, 3 cancelled, < 0 error.  A request's film is identical to pt_render's whether it ran
 * alone or in any mix.  No counterpart in the reference, which renders one frame per process. */
int pt_server_create(const pt_server_config *cfg, pt_server **out);
int pt_server_submit(pt_server *server, pt_scene *scene, const pt_render_desc *desc, uint64_t *ticket);
/* latency_ms: submit to completion (-1 until done). */
int pt_server_poll(pt_server *server, uint64_t ticket, int *state, double *latency_ms);
int pt_server_wait(pt_server *server, uint64_t ticket, uint32_t timeout_ms, int *state);
/* Where a request's latency went, in ms after submission (-1 for a stage not reached yet):
 * admitted (device and host memory taken), first wave enqueued, last wave's kernels done on the
 * GPU, film in host memory (the completion that pt_server_poll's latency reports). */
typedef struct pt_request_timing {
    double admitted_ms, first_wave_ms, last_wave_ms, done_ms;
} pt_request_timing;
int pt_server_timing(pt_server *server, uint64_t ticket, pt_request_timing *timing);
/* Copies a finished request's film (width*height*3 floats) and primary ids, then forgets it.  A
 * failed or cancelled request is forgotten too, and its status (PT_ECANCELED for a cancelled one)
 * is returned. */
int pt_server_fetch(pt_server *server, uint64_t ticket, float *rgb_out, uint32_t *primary_out);
/* Cancels a request.  A queued one ends at once (state 3); an admitted one gets no work in later
 * waves, and ends (state 3, its device memory and host arena space released) once the waves
 * already queued with its work have retired -- at most two, the scheduler's queue depth.  Waiting
 * for it with pt_server_wait then returns state 3.  PT_EINVAL for an unknown ticket or a request
 * that has already finished (done, failed or cancelled). */
int pt_server_cancel(pt_server *server, uint64_t ticket);
int pt_server_get_stats(pt_server *server, pt_server_stats *stats);
int pt_server_destroy(pt_server *server);

/* ---- synthetic workload generators (deterministic, shared by the oracle and the bench) --- */

/* Icosphere: icosahedron subdivided `level` times (20 * 4^level faces, 10 * 4^level + 2
 * vertices) of the given radius, each vertex displaced radially by `noise_amp` times 3-octave
 * seeded value noise.  Writes packed positions and faces; pass NULL to query the counts. */
int pt_gen_icosphere(uint32_t level, float radius, float noise_amp, uint64_t noise_seed,
                     float *x, float *y, float *z, uint32_t *num_vertices,
                     uint32_t *fv0, uint32_t *fv1, uint32_t *fv2, uint32_t *num_faces);

/* The intersection-microbench ray set: origins uniform on a sphere of radius `origin_radius`,
 * directions normalized toward a uniform point in the unit ball; even indices are closest-hit
 * queries (tmax = INFINITY), odd indices any-hit queries with tmax = distance to the target. */
int pt_gen_rays(uint64_t n, float origin_radius, uint64_t seed, pt_ray *rays);

/* ---- misc -------------------------------------------------------------------------------- */
const char *pt_last_error(void);
const char *pt_version(void);

/* ---- exact-arithmetic hooks (no reference counterpart; used by the parity tests) ---------- */

/* (float)((double)a*b - (double)c*d) computed without FP64 instructions, as the kernels do for
 * the Wald test's edge fallback (src/cpu/shapes/mesh.cpp:252-264).  Host build of the same code. */
float pt_host_f64_diff_emulated(float a, float b, float c, float d);

/* Runs a device build of one exact helper over n host inputs: which = 0 f64_diff_emulated
 * (in: 4 floats, out: 1 float per item), 1 sin/cos(2*pi*u) (in: 1 float, out: 2 floats),
 * 2 Philox4x32-10 keyed by seed (in: 4 uint32 counters, out: 4 uint32). */
int pt_selftest_device(int which, const void *in, void *out, uint32_t n, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif /* POLYTOPE_B200_H */
