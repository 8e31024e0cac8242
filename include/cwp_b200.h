/* cwp_b200.h - C ABI of the B200 wavefront path tracer (libcwpb200.so).
 *
 * Every entry point returns CWP_OK (0) or an error code; cwp_last_error() gives the message of the last failure on
 * the calling thread. No entry point exits the process. Handles are not thread-safe: use one handle per host thread
 * (the reference renderer has the same single-thread rule). Device pointers are CUDA global-memory addresses on the
 * handle's device; host pointers are ordinary process memory. All float4 arrays are 16-byte aligned, x y z w.
 *
 * Each declaration names the reference interface it replaces (file:line in YJLi-new/cuda-wavefront-pathtracer).
 */
#ifndef CWP_B200_H
#define CWP_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define CWP_OK 0
#define CWP_ERR_INVALID 1      /* bad argument or malformed buffer */
#define CWP_ERR_CUDA 2         /* CUDA runtime error */
#define CWP_ERR_NOMEM 3        /* device or host allocation failed, or admission refused */
#define CWP_ERR_STATE 4        /* call out of order (e.g. render before init) */
#define CWP_ERR_TRAVERSAL 5    /* a ray hit the traversal stack bound or visit budget (malformed or too deep BVH) */
#define CWP_ERR_IO 6           /* file unreadable / unwritable */

#define CWP_LAYOUT_BVH2 2
#define CWP_LAYOUT_BVH4 4
#define CWP_LAYOUT_CWBVH 8
#define CWP_TRI_MT 0           /* Moller-Trumbore on (v0, e1, e2) */
#define CWP_TRI_WOOP 1         /* Woop unit-triangle rows */
#define CWP_FILTER_TABLE 64

const char* cwp_last_error(void);
int32_t cwp_version(void);

/* ------------------------------------------------------------------------------------------------------------------
 * Meshes and the synthetic box field. Replaces Mesh (scene/mesh.h:9-26), loadMesh/loadOBJ/loadPLY
 * (io/mesh_loader.h:6-8); the box field has no reference counterpart (the reference's synthetic scene is a sphere
 * grid, scene/synthetic.cpp:6-48).
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_mesh cwp_mesh;
typedef struct cwp_mesh_view {
    const float* verts; int64_t n_verts;       /* 3 floats per vertex */
    const int32_t* faces; int64_t n_tris;      /* 3 vertex indices per triangle */
    const int32_t* face_mat;                   /* material id per triangle or NULL */
    const float* normals;                      /* 3 floats per vertex or NULL */
    const float* albedo; int32_t n_albedo;     /* 3 floats per material */
} cwp_mesh_view;

int cwp_mesh_box_field(int32_t n_boxes, uint64_t seed, cwp_mesh** out);
int cwp_mesh_load(const char* path, cwp_mesh** out);
/* The reference's procedural scene, makeSynthetic (scene/synthetic.h:6, synthetic.cpp:6-48), vertex for vertex: a
 * ground of ground x ground quads and grid x grid bumpy spheres of nu x nv quads, five albedos. The reference's CLI
 * uses nu = 200, nv = 100, ground = 200 (app/scene_setup.cpp:93): 2,000,000 triangles at grid = 7.
 * cwp_sphere_grid_c2w replaces syntheticCamera (synthetic.h:8): its row-major camera-to-world matrix. */
int cwp_mesh_sphere_grid(int32_t grid, int32_t nu, int32_t nv, int32_t ground, cwp_mesh** out);
void cwp_sphere_grid_c2w(float c2w[16]);
int cwp_mesh_from_view(const cwp_mesh_view* v, cwp_mesh** out);
int cwp_mesh_view_of(const cwp_mesh* m, cwp_mesh_view* out);
int cwp_mesh_write_ply(const cwp_mesh* m, const char* path);
void cwp_mesh_free(cwp_mesh* m);

/* ------------------------------------------------------------------------------------------------------------------
 * Host BVH construction. Replaces BVHBuilder::build (accel/bvh_builder.cpp:5-68), BVH2Flat/BVH4Flat/BVH8Flat::build
 * (accel/bvh_layouts.cpp:24,57,97), CWBVH::build (accel/bvh_tools.cpp:75), sahCost (bvh_tools.cpp:40),
 * packTriangles / packWoop (accel/tri_pack.cpp:6,18) and the layout step of setupScene (app/scene_setup.cpp:190-222).
 * Output encodings are byte-identical to the reference's at bins = 16.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_build_options {
    int32_t variant;    /* CWP_LAYOUT_* */
    int32_t bins;       /* SAH bins per axis, 2..256 (reference: 16) */
    int32_t leaf;       /* max triangles per leaf (reference --leaf, default 4; CWBVH SAH collapse builds from leaf 1) */
    int32_t collapse;   /* CWBVH: 0 SAH dynamic programme, 1 greedy */
    int32_t threads;    /* host threads, 0 = all */
    float spatial;      /* > 0: spatial splits (SBVH) where the object split's children overlap by more than this
                           fraction of the root's area (1e-5 typical); a spatial split may add at most 30% references
                           to a node. 0: the reference's binned SAH (byte-identical buffers at 16 bins) */
    int32_t builder;    /* 0: host binned SAH (above); 1: the binary tree built on the GPU by H-PLOC, leaves collapsed
                           to the SAH optimum on the host, then the same layouts - the reference's --builder hploc
                           (app/scene_setup.cpp:76-83: hplocBuildHost, hploc.cu:195-209, then treeFromHploc,
                           bvh_tools.cpp:12-38); bins and spatial do not apply; build_ms is then the GPU build time */
    int32_t device;     /* builder 1: CUDA device */
} cwp_build_options;

typedef struct cwp_bvh cwp_bvh;
typedef struct cwp_bvh_data {
    const float* nodes; int64_t n_node_float4; int32_t node_stride;   /* 4 (BVH2), 8 (BVH4) or 5 (CWBVH) float4 per node */
    const int32_t* order; int64_t n_tris;                              /* leaf order of the mesh triangles */
    const float* tris;                                                 /* 3 float4 per triangle, leaf order */
    const float* nrm;                                                  /* 3 float4 per triangle or NULL */
    const float* woop;                                                 /* 3 float4 per triangle */
    int32_t max_depth, max_leaf_tris;
    double sah, build_ms;
    const float* verts;                                                /* 3 float4 per triangle: exact corners v0, v1, v2 */
} cwp_bvh_data;

int cwp_bvh_build(const cwp_mesh* m, const cwp_build_options* opt, cwp_bvh** out);
int cwp_bvh_data_of(const cwp_bvh* b, cwp_bvh_data* out);   /* pointers stay valid until cwp_bvh_free */
void cwp_bvh_free(cwp_bvh* b);

/* ------------------------------------------------------------------------------------------------------------------
 * Device scene + standalone ray batches. Replaces the device traversal trav<V,ANY,TRI> (accel/traverse.cuh:155-160)
 * as used by traceOne / shadowOne (render/wavefront.cu:61-72); the batch entry point itself is new.
 * Rays: o = (ox, oy, oz, tmin), d = (dx, dy, dz, tmax) float4 arrays. Closest hits: float4 (t, u, v, tri bits) with
 * tri = leaf-order triangle index or -1 (t = tmax on a miss). Any-hit: int32 index of the first occluder found or -1.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_scene_buffers {
    const float* nodes; int64_t n_node_float4; int32_t node_stride;
    const float* tris; int64_t n_tris;
    const float* nrm;       /* or NULL */
    const float* woop;      /* or NULL (required for CWP_TRI_WOOP) */
    const float* albedo; int32_t n_albedo;
    const float* verts;     /* exact corners, 3 float4 per triangle, or NULL (required by the precision form) */
} cwp_scene_buffers;

typedef struct cwp_accel cwp_accel;
int cwp_accel_create(const cwp_scene_buffers* s, int32_t tri, int32_t device, cwp_accel** out);
void cwp_accel_destroy(cwp_accel* a);
/* stream: a cudaStream_t or NULL (legacy default stream); asynchronous with respect to the host */
int cwp_trace_closest(cwp_accel* a, const float* d_o, const float* d_d, float* d_hits, int64_t n, void* stream);
int cwp_trace_any(cwp_accel* a, const float* d_o, const float* d_d, int32_t* d_occluder, int64_t n, void* stream);
/* host buffers; copies in, traces, copies out, synchronises; *ms = device time of the whole call (may be NULL). Batches
 * of 512k rays and more are cut into up to 8 chunks over two streams, so copies in, traversal and copies out overlap;
 * from pinned host memory the copies run asynchronously, from pageable memory the driver stages them. */
int cwp_trace_closest_host(cwp_accel* a, const float* o, const float* d, float* hits, int64_t n, float* ms);
int cwp_trace_any_host(cwp_accel* a, const float* o, const float* d, int32_t* occluder, int64_t n, float* ms);
/* traversal status of the calls since the last query (CWP_OK or CWP_ERR_TRAVERSAL); clears it */
int cwp_accel_status(cwp_accel* a);
/* kernel form of the batch calls: 0 auto (persistent refill for CWBVH), 1 refill (BVH2 / CWBVH), 2 one ray per thread */
int cwp_accel_set_traversal(cwp_accel* a, int32_t mode);

/* Precision form (no counterpart in the reference): mode 1 makes the batch calls traverse the CWBVH with f16x2 slab
 * tests over its 8-bit child boxes, rounded outward so that they are conservative, and decide hits with a watertight
 * FP32 triangle test on the exact corners (cwp_scene_buffers.verts) - no hit inside [tmin, tmax] is lost. Mode 0 is the
 * plain path (FP32 slabs, the reference's triangle tests). Hits use the same leaf-order indices. */
int cwp_accel_set_precision(cwp_accel* a, int32_t mode);
/* FP64 traversal of the same CWBVH and exact corners (the precision form's oracle): t in double (tmax on a miss) and
 * the leaf-order triangle (-1 on a miss); any_hit stops at the first occluder. Device buffers, stream-ordered. */
int cwp_trace_fp64(cwp_accel* a, int32_t any_hit, const float* d_o, const float* d_d, double* d_t, int32_t* d_tri, int64_t n, void* stream);

/* ------------------------------------------------------------------------------------------------------------------
 * Wavefront renderer. Replaces class WavefrontRenderer (render/renderer.h:47-93): init (wavefront.cu:469-502),
 * render (wavefront.cu:684-741 legacy loop, 644-680 graph frame), readAccum / accumDevice (renderer.h:58-59),
 * setParams / setMaterials (wavefront.cu:744-752), introspection (renderer.h:69). Params mirrors render/params.h:8-16,
 * RenderOptions renderer.h:11-28, FrameStats renderer.h:45. The accumulation buffer holds w*h float4 radiance sums.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_camera {
    float pos[3], ax[3], ay[3], az[3];   /* camera looks down -az, +ay up (scene/camera.h:7) */
    float fx, fy, px, py;
    int32_t w, h;
    float lens_r, focus_d;
} cwp_camera;

typedef struct cwp_params {
    cwp_camera cam;
    float sun_to[3], sun_e[3], sky[3];
    float sun_cos;                       /* cos of the sun's angular radius */
    int32_t max_b; uint32_t seed;
    float eps, near_clip;
    int32_t has_n, filter_bh;
    float ftab[CWP_FILTER_TABLE + 1];    /* pixel-filter inverse CDF (used when filter_bh) */
} cwp_params;

typedef struct cwp_render_options {
    int32_t variant;      /* CWP_LAYOUT_* of the scene's nodes */
    int32_t tri;          /* CWP_TRI_* */
    int32_t batch;        /* samples per pixel in flight per wavefront pass */
    int32_t bounces;      /* max bounce depth (camera hit = 0) */
    int32_t graph;        /* 1: each frame is one CUDA graph with device-side queue counts; 0: host loop */
    int32_t block;        /* threads per block of the traversal kernels (0 = 128) */
    int32_t device;       /* CUDA device ordinal */
    int32_t profile;      /* 1: CUDA event pair around every kernel launch (also inside the graph), see cwp_renderer_depth_stats */
    int32_t traversal;    /* 0 auto (refill for CWBVH closest-hit), 1 persistent lanes with dynamic refill everywhere, 2 one 32-ray fetch per warp */
    int32_t sort;         /* continuation rays regrouped before each bounce: 0 off, 1 by direction octant, 2 by octant and a 4x4x4 origin cell */
    int32_t stage_levels; /* CWBVH: levels 0..L of the tree copied into every traversal block's shared memory (L = 1..3, at most
                             512 nodes); -1 none; 0 the library's default */
    int32_t reserved;
} cwp_render_options;

typedef struct cwp_frame_stats { double rays, shadow_rays, trace_ms, frame_ms; } cwp_frame_stats;
typedef struct cwp_renderer_info { double vram_mb, tlas_ms; int32_t pt_blocks, n_sm; char gpu_name[256]; } cwp_renderer_info;

typedef struct cwp_renderer cwp_renderer;
int cwp_renderer_create(cwp_renderer** out);
int cwp_renderer_init(cwp_renderer* r, const cwp_params* p, const cwp_scene_buffers* s, const cwp_render_options* o);
int cwp_renderer_render(cwp_renderer* r, int32_t spp, cwp_frame_stats* st, int32_t s_base, int32_t clear);
int cwp_renderer_read_accum(const cwp_renderer* r, float* dst);      /* w*h*4 floats */
const void* cwp_renderer_accum_device(const cwp_renderer* r);
int cwp_renderer_set_params(cwp_renderer* r, const cwp_params* p);
int cwp_renderer_set_materials(cwp_renderer* r, const float* albedo, int32_t n);
int cwp_renderer_info_of(const cwp_renderer* r, cwp_renderer_info* out);
/* Per-depth figures of the last frame, summed over its passes, for d < n_depths = bounces + 2: closest[d] / shadow[d]
 * = rays traced at depth d (queue lengths); trace_ms[d] / shadow_ms[d] = device time of the depth-d trace+shade and
 * shadow kernels (needs options.profile = 1, else zeros). Any pointer may be NULL. (The reference reports these
 * only as frame totals: FrameStats, renderer.h:45, and t_trace_ms from event pairs, wavefront.cu:700-709.) */
int cwp_renderer_depth_stats(const cwp_renderer* r, int64_t* closest, int64_t* shadow, float* trace_ms, float* shadow_ms, int32_t n_depths);
void cwp_renderer_destroy(cwp_renderer* r);

/* ------------------------------------------------------------------------------------------------------------------
 * Rendering without allocation. No counterpart in the reference. For callers that cannot call cudaMalloc - a plugin
 * whose host application owns the GPU's memory budget, a serving loop that must not stall on cudaMalloc / cudaFree
 * (both may synchronise the device), code that must not fail on an allocation mid-frame - this renders the same frame
 * as cwp_renderer_render into the caller's accumulation buffer, with every scratch buffer in a fixed 31.5 MB device
 * array inside the library that each GPU loading the library holds until process exit. Limits: w*h*batch <= 262144
 * paths per pass, bounces <= 62. The scene pointers are device copies of buffers that cwp_bvh_build produced (or that
 * cwp_accel_create would accept); they are not re-validated here. The first call on a device looks up the array's
 * device address (do it before any stream capture on that device). All calls share the array: calls whose work
 * overlaps on the GPU (other streams, other host threads) race and must be serialised by the caller. Launches are
 * stream-ordered on `stream`; when h_rays is not NULL the call waits for the frame and stores the closest and shadow
 * ray totals there (and reports traversal errors). The call runs on the current device: options.device must name
 * it, and every scene pointer and d_accum must be device (or managed) memory of that device, else CWP_ERR_INVALID.
 * Of the options, variant, tri, batch, bounces and device are used; the traversal is always one 32-ray fetch per
 * warp (traversal must be 0 or 2), there is no regrouping (sort must be 0), and graph, block and profile are
 * ignored: the passes are plain stream launches.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_device_scene {
    const float* nodes; const float* tris; const float* woop; const float* nrm;   /* device pointers; woop / nrm may be NULL */
    const float* albedo;                                                          /* device, 3 floats per material */
} cwp_device_scene;
int cwp_render_noalloc(const cwp_params* p, const cwp_device_scene* s, const cwp_render_options* o, int32_t spp, int32_t s_base,
                       int32_t clear, float* d_accum, int64_t* h_rays, void* stream);

/* ------------------------------------------------------------------------------------------------------------------
 * Instances and two-level scenes (the batched form).
 * cwp_instance replaces DevInstance (accel/instance.h:7, 112 B: world->object rows, object->world rows, BLAS root,
 * mesh, det sign); cwp_xform_invert replaces invertXform (scene/instances.cpp:64-79: FP64 adjugate inverse rounded to
 * fp32); cwp_xform_animate replaces instanceXform (scene/instances.cpp:48-62: translate + axis/angle rotation + scale,
 * each with a per-frame velocity, composed in FP64).
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_instance {
    float inv[12];      /* world -> object, 3 rows of (m0 m1 m2 t) */
    float fwd[12];      /* object -> world */
    int32_t root;       /* root node of the instance's BLAS in the traced layout (cwp_batch_download_tlas fills it in) */
    int32_t mesh;       /* BLAS index */
    float det_sign;     /* sign of det(fwd) */
    int32_t pad;
} cwp_instance;

typedef struct cwp_instance_desc {   /* InstanceDesc (scene/instances.h) */
    int32_t mesh;
    float translate[3], translate_per_frame[3];
    float axis[3], angle_deg, angle_deg_per_frame;
    float scale[3], scale_per_frame[3];
} cwp_instance_desc;

int cwp_xform_invert(const float m[12], float inv[12], float* det_sign);
int cwp_xform_animate(const cwp_instance_desc* d, int32_t frame, float m[12]);
/* fills fwd = m, inv and det_sign from cwp_xform_invert, mesh; root = -1 */
int cwp_instance_from_xform(const float m[12], int32_t mesh, cwp_instance* out);

/* ------------------------------------------------------------------------------------------------------------------
 * Batched form: many meshes built on the GPU in one pass, many two-level scenes traced in one persistent launch.
 * Replaces HplocBuilder (accel/hploc.h:18-41: reserve/build/release, one mesh per build) with a builder that takes
 * every BLAS at once; hplocToBVH2 (hploc.h:36) and setInstances (render/renderer.h:53, wavefront.cu:570-581: instance
 * boxes k_inst_boxes, TLAS rebuild) for every scene at once; travInst / StepTrav / persistentTrace
 * (accel/traverse_inst.cuh:10-159, render/wavefront.cu:403-442) for a ray queue whose rays carry a scene id. The
 * autotuner has no reference counterpart.
 * Hits: float4 (t, u, v, tri bits), tri = index into the batch's leaf-order triangle array (its w field of the first
 * float4 is the triangle's index in its mesh), plus the instance index (into the cwp_batch_set_scenes array) or -1.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_batch cwp_batch;
typedef struct cwp_batch_options {
    int32_t device;
    int32_t leaf;           /* max triangles per BVH2 / BVH4 leaf (default 4 when 0); CWBVH leaves hold at most 3 */
    int32_t widths;         /* bit mask of the layouts to emit: 1 << 2 (BVH2), 1 << 4 (BVH4), 1 << 8 (CWBVH); 0 = all */
    int32_t builder;        /* 0: every BLAS on the GPU in one H-PLOC launch; 1: on the host cores (binned SAH, 32 bins,
                               SAH-collapsed CWBVH, spatial splits when `spatial` > 0), for resident scenes */
    float spatial;          /* builder 1: spatial-split overlap threshold (cwp_build_options.spatial) */
    int32_t tlas_width;     /* TLAS nodes the traversal reads: 4 (default when 0; each node holds the grandchildren of the
                               BVH2 TLAS, about half the TLAS node visits) or 2 (the reference's BVH2 TLAS) */
    int32_t reserved[2];
} cwp_batch_options;

typedef struct cwp_batch_tuning {
    int32_t block;          /* threads per block, 64..512 */
    int32_t width;          /* BLAS layout 2, 4 or 8 */
    int32_t fetch;          /* idle lanes of a warp before it fetches new rays, 1..32 */
    int32_t smem_stack;     /* 1: BLAS traversal stack in shared memory, 0: in local memory */
    float ms;               /* autotuner: measured time of the sample (closest + any), else 0 */
    int32_t reserved[3];
} cwp_batch_tuning;

typedef struct cwp_batch_info {
    int32_t n_blas, n_scenes;
    int64_t n_tris, n_instances;
    int64_t node_bytes[3];  /* BVH2, BVH4, CWBVH node arrays (0 if not emitted) */
    double blas_build_ms;   /* GPU time of the BLAS build (bounds, keys, sort, H-PLOC, layouts) */
    double tlas_build_ms;   /* GPU time of the last cwp_batch_set_scenes (instance boxes, H-PLOC, TLAS layout) */
    int32_t blas_hploc_launches;   /* H-PLOC kernel launches of the BLAS build (1) */
    int32_t pad;
} cwp_batch_info;

/* Builds every BLAS on the device: one bounds pass, one key pass, one segmented radix sort and ONE H-PLOC launch
 * over all meshes' triangles, then the BVH2 / BVH4 / CWBVH encodings and Moller-Trumbore triangle records. */
int cwp_batch_create(const cwp_mesh_view* meshes, int32_t n_meshes, const cwp_batch_options* opt, cwp_batch** out);
void cwp_batch_destroy(cwp_batch* b);
/* Scenes: scene s owns instances [scene_first[s], scene_first[s + 1]) of inst (n_scenes + 1 entries). Builds every
 * scene's TLAS (BVH2 over instance world boxes) on the device in one H-PLOC launch; call again each frame when the
 * transforms move. Synchronous. */
int cwp_batch_set_scenes(cwp_batch* b, const cwp_instance* inst, int64_t n_inst, const int32_t* scene_first, int32_t n_scenes);
/* Incremental form for scenes that change one at a time (a serving loop's slots): cwp_batch_reserve_scenes lays out
 * n_scenes empty scenes with room for `cap` instances each (scene s owns instances [s * cap, s * cap + cap)); then
 * cwp_batch_update_scenes replaces the instances of the n listed scenes (distinct) with counts[i] <= cap instances
 * each, taken in order from inst, and rebuilds only their TLAS, in one H-PLOC launch; the other scenes' TLAS stay as
 * they are and traceable. An empty scene's rays miss. Rays of the updated scenes must not be in flight. Synchronous.
 * cwp_batch_set_scenes returns the batch to the packed form. */
int cwp_batch_reserve_scenes(cwp_batch* b, int32_t n_scenes, int32_t cap);
int cwp_batch_update_scenes(cwp_batch* b, const int32_t* scenes, int32_t n, const cwp_instance* inst, const int32_t* counts);
/* One persistent launch over a queue of rays tagged with scene ids (d_scene, int32 per ray). any_hit: d_hits may be
 * NULL and d_inst receives the occluding instance or -1. */
int cwp_batch_trace(cwp_batch* b, int32_t any_hit, const float* d_o, const float* d_d, const int32_t* d_scene, float* d_hits,
                    int32_t* d_inst, int64_t n, void* stream);
/* Times the closest + any-hit trace of the given sample over block size {64, 128, 256, 512}, BLAS width {2, 4, 8},
 * fetch granularity {1, 2, 4, 8, 16, 32} and stack placement {local, shared}, keeps the fastest and returns it.
 * d_hits / d_inst are scratch of n entries. */
int cwp_batch_autotune(cwp_batch* b, const float* d_o, const float* d_d, const int32_t* d_scene, float* d_hits, int32_t* d_inst,
                       int64_t n, cwp_batch_tuning* best);
int cwp_batch_set_tuning(cwp_batch* b, const cwp_batch_tuning* t);
int cwp_batch_get_tuning(const cwp_batch* b, cwp_batch_tuning* t);
int cwp_batch_info_of(const cwp_batch* b, cwp_batch_info* out);
/* Host copies for checking: the node array of one layout (width 2, 4 or 8) and the triangle records. Pass NULL
 * buffers to query the sizes (in float4). */
int cwp_batch_download(const cwp_batch* b, int32_t width, float* nodes, int64_t* n_node_float4, float* tris, int64_t* n_tri_float4);
/* root node of mesh m's BLAS in layout width (instances name their mesh; the traversal looks its root up for the
 * traced width); and the TLAS (BVH2 nodes, root per scene, instances with `root` set for the current tuning's width) */
int cwp_batch_blas_root(const cwp_batch* b, int32_t width, int32_t mesh, int32_t* root);
int cwp_batch_download_tlas(const cwp_batch* b, float* nodes, int64_t* n_node_float4, int32_t* roots, cwp_instance* inst);
/* TLAS form the traversal reads from the next launch on (2 or 4; both are built by every scene update), and thereby
 * the form cwp_batch_download_tlas returns (8 float4 per node for width 4: lo x, hi x, lo y, hi y, lo z, hi z of four
 * children, references, counts; count 1 = an instance, reference -1 = an empty slot) */
int cwp_batch_set_tlas_width(cwp_batch* b, int32_t width);
int cwp_batch_status(cwp_batch* b);   /* synchronises; CWP_ERR_TRAVERSAL if a ray hit a stack bound or the visit budget */

/* ------------------------------------------------------------------------------------------------------------------
 * Serving form: a request loop over the resident scenes of a cwp_batch with continuous batching. Requests (scene,
 * animation frame, camera / resolution, spp, depth, lighting, seed) are admitted while request slots and free device
 * memory allow; every step advances all admitted requests' paths by one bounce in the same launches (new camera
 * paths join at every step), so requests that arrive while others run share the GPU. Each request's image depends only
 * on its own inputs: the sample streams are keyed by (pixel, sample, depth, dimension, seed).
 * Replaces the full integrator for instanced scenes (render/wavefront.cu:223-356 shadeFull<INST>, render/bsdf.h,
 * scene/material.h): OpenPBR-subset materials, next-event estimation with one light sample per vertex over the sun,
 * the emissive triangles (by power) and an environment map (by luminance x sin(theta)), combined with BSDF sampling by
 * the power heuristic, optional Russian roulette; the request loop itself is new.
 * ------------------------------------------------------------------------------------------------------------------ */
typedef struct cwp_material {        /* Material (scene/material.h:12-17), 64 B */
    float base_color[3]; float metallic;
    float specular_color[3]; float roughness;
    float emission[3]; float ior;    /* emission radiance (colour x strength) */
    float specular_weight; float transmission; float pad0, pad1;
} cwp_material;

typedef struct cwp_server cwp_server;
typedef struct cwp_server_options {
    int64_t max_paths;     /* paths in flight over all requests (default 8 Mi) */
    int32_t max_requests;  /* requests admitted at once (default 64; 1 for the plain form) */
    int32_t gd_energy;     /* glossy-diffuse energy compensation (default 1, as the reference's --gd_energy) */
    int64_t hbm_reserve;   /* device bytes that admission leaves free (default 1 GiB) */
    int32_t device;
    int32_t regroup;       /* sort each step's continuations by request before tracing: 1 on, -1 off, 0 default (on) */
    int32_t policy;        /* new camera paths each step: 0 even share of the free path capacity among the requests with
                              samples left (oldest first, the default); 1 oldest first takes all it can use, the later
                              ones fill what is left (a request's drain no longer idles the GPU, big requests keep the
                              plain form's speed) */
    int32_t overlap;       /* 0 (default) or 1: a step returns once its launches are queued, and the next call to
                              cwp_server_step waits for them and takes their results (completions, queue lengths), so
                              the caller's work between steps (submissions, results) overlaps the device; -1: every step
                              waits for its own work before returning */
    int32_t reserved[2];
} cwp_server_options;

typedef struct cwp_request {
    int32_t scene;         /* scene of the batch: its instances are animated to `frame` (cwp_server_set_scenes) */
    int32_t frame;
    cwp_camera cam;        /* pinhole; resolution cam.w x cam.h */
    int32_t spp, max_depth;
    uint32_t seed;
    float sun_to[3], sun_e[3], sky[3];
    float sun_cos, eps;    /* cos of the sun's half angle; ray offset */
    int32_t env;           /* environment map of the server (cwp_server_set_envmaps) lighting the request, or -1: the
                              constant sky (not light-sampled) */
    float env_rot_deg;     /* rotation of the map about +z (the reference's --env_rot) */
    /* Light sampling (RenderOptions, render/renderer.h:21-25). A light sample picks one of the enabled light types with
     * equal probability (render/wavefront.cu:531-533): the sun when luminance(sun_e) > 0, the emissive triangles of
     * the scene at the request's frame when it has any, the map when env >= 0; the latter two not in BSDF mode. */
    int32_t light_mode;    /* CWP_LIGHT_MIS (0, default), CWP_LIGHT_NEE: emitters hit by BSDF samples count nothing,
                              CWP_LIGHT_BSDF: only the sun is light-sampled */
    int32_t rr, rr_depth;  /* Russian roulette from depth rr_depth on (survival max(T) clamped to [0.05, 1]); rr = 0 off */
    int32_t env_uniform;   /* 1: environment light samples uniform on the sphere instead of by luminance */
    int32_t bump_shadow;   /* 1: bump-terminator shadowing of the diffuse lobe where a normal image perturbed the normal
                              (Chiang et al. 2019; the reference's --bump_shadow) */
    /* Camera rays (k_raygen, render/wavefront.cu:42-58): a thin lens when cam.lens_r > 0 (focused at cam.focus_d),
     * tmin = near_clip, pixel filter box or Blackman-Harris of radius 1.5 (the reference's --filter bh, its default) */
    float near_clip;
    int32_t filter_bh;
} cwp_request;
#define CWP_LIGHT_MIS 0
#define CWP_LIGHT_NEE 1
#define CWP_LIGHT_BSDF 2

typedef struct cwp_request_stats {
    double submit_ms, admit_ms, done_ms;    /* on the server's clock (ms since creation) */
    double rays, shadow_rays;
    int32_t w, h, spp, pad;
} cwp_request_stats;

/* Materials: table of n_mats; mesh m's triangles use materials mesh_mat_base[m] + (triangle material id). */
int cwp_server_create(cwp_batch* b, const cwp_material* mats, int32_t n_mats, const int32_t* mesh_mat_base, const cwp_server_options* o, cwp_server** out);
void cwp_server_destroy(cwp_server* s);
/* Scenes: scene k owns instance descriptors [scene_first[k], scene_first[k + 1]) (cwp_xform_animate at the request's
 * frame gives their transforms); replaces the batch's scenes while the server lives. */
int cwp_server_set_scenes(cwp_server* s, const cwp_instance_desc* desc, int64_t n, const int32_t* scene_first, int32_t n_scenes);
/* Instances placed by 3x4 matrices instead of animation parameters (scene files' "transform" and "transforms" keys;
 * instanceXform, scene/instances.cpp:50-51): descriptor i of the scenes uses xforms[first_xf[i] .. first_xf[i] +
 * n_xf[i]) (12 floats each, row-major object to world), frame f taking entry min(f, n_xf[i] - 1); n_xf[i] = 0 keeps
 * its animation parameters. n = the descriptor count of cwp_server_set_scenes; NULL arrays clear the matrices. Only
 * while no request is queued or running. */
int cwp_server_set_instance_xforms(cwp_server* s, const float* xforms, const int32_t* first_xf, const int32_t* n_xf, int64_t n);
int cwp_server_submit(cwp_server* s, const cwp_request* r, int64_t* id);
/* Environment maps the requests may name (cwp_request.env): equirectangular, row 0 = +z, the centre column facing +x
 * (the reference's orientation, scene/environment.h:1-4); rgb = w x h x 3 linear floats scaled by strength. Replaces
 * the server's maps; only while no request is queued or running. Replaces buildEnvMap's use in setupScene
 * (app/scene_setup.cpp:252) for the serving form. */
typedef struct cwp_envmap { const float* rgb; int32_t w, h; float strength; int32_t pad; } cwp_envmap;
int cwp_server_set_envmaps(cwp_server* s, const cwp_envmap* maps, int32_t n);
/* Material textures (glTF metallic-roughness; scene/texture.h:10-24): images are 8-bit RGBA, top row first, looked up
 * at (u, 1 - v) with bilinear filtering (nearest = 1: the nearest texel, the reference's --tex_filter nearest, which it
 * applies to every image) and wrap addressing, colour images (srgb = 1) decoded from sRGB. Material m's
 * factors are multiplied by its bound images: base colour and emission by rgb, metallic and roughness by one channel;
 * a normal image perturbs the shading normal in the tangent frame. mtex has n_mtex entries (material index, as in the
 * server's table; materials beyond n_mtex are untextured). uvs: 2 float4 per triangle of every batch mesh in mesh
 * order, by mesh-local triangle index ((u0, v0, u1, v1), (u2, v2, -, -)); tans: 3 float4 per triangle (corner tangent
 * xyz, handedness sign w) or NULL (normal images then ignored). Replaces the texture set-up of the full integrator
 * (render/wavefront.cu:535-547, packAttributes in app/scene_setup.cpp:255). Only while no request is queued or running. */
typedef struct cwp_texture { const uint8_t* rgba; int32_t w, h; int32_t srgb, nearest; } cwp_texture;
typedef struct cwp_material_textures {
    int32_t base_color, emission, normal, metallic, roughness;   /* texture ids or -1 */
    int32_t metallic_ch, roughness_ch;                          /* channel of the metallic / roughness image (glTF: 2, 1) */
    float normal_scale;
} cwp_material_textures;
int cwp_server_set_textures(cwp_server* s, const cwp_texture* tex, int32_t n_tex, const cwp_material_textures* mtex, int32_t n_mtex,
                            const float* uvs, const float* tans);
/* Texture lookups on the device, for tests of the filtering: n (texture, u, v) -> rgba, with the images of tex bound as
 * cwp_server_set_textures binds them. */
int cwp_texture_sample_batch(const cwp_texture* tex, int32_t n_tex, const int32_t* id, const float* uv, float* rgba, int64_t n);
/* One step: the results of the previous step (completions, queue lengths), admission, new camera paths, one bounce of
 * every admitted request (closest hit + shading, light-sample shadow rays). With options.overlap (the default) the
 * call returns once the bounce's launches are queued and its completions appear at the next call; with overlap -1 it
 * waits for them. *n_active / *n_pending: admitted / waiting requests. A submission prepares the request's host data
 * (instances at its frame, emissive tables), so the step's admission only copies them to the device. */
int cwp_server_step(cwp_server* s, int32_t* n_active, int32_t* n_pending);
/* Completed request ids since the last call (up to cap). */
int cwp_server_poll(cwp_server* s, int64_t* ids, int32_t cap, int32_t* n);
/* The image of a completed request (w * h float4 radiance sums over its spp, may be NULL) and its statistics; the
 * request's device memory is released. */
int cwp_server_result(cwp_server* s, int64_t id, float* accum, cwp_request_stats* st);
double cwp_server_clock_ms(const cwp_server* s);
typedef struct cwp_server_info {
    int64_t steps, rays, shadow_rays, admissions, tlas_rebuilds;
    double closest_ms, shade_ms, shadow_ms, raygen_ms, tlas_ms, step_ms;   /* device time per phase (CUDA events), wall time of the steps */
    double admit_ms;         /* host time of admissions (instance animation, image allocation) */
    double tlas_device_ms;   /* device time of the TLAS updates inside tlas_ms (which is their wall time) */
    double accum_ms;         /* device time of the shadow contributions' accumulation inside shadow_ms */
} cwp_server_info;
int cwp_server_info_of(const cwp_server* s, cwp_server_info* out);
/* Device-side BSDF of a material table for n (material, wo, wi) triples in local frames (wo.z > 0): f (float4) and
 * pdf; and n samples (u, u1, u2 in uvw) -> wi, weight, pdf. nr: an unperturbed normal per triple for the
 * bump-terminator term (bsdfEval's nr, render/bsdf.h:196), or NULL (+z, off). For tests of the device arithmetic. */
int cwp_bsdf_eval_batch(const cwp_material* mats, int32_t n_mats, const int32_t* mat, const float* wo, const float* wi, const float* eta,
                        int32_t gd_energy, const float* ux, float* f, float* pdf, int64_t n, const float* nr);
int cwp_bsdf_sample_batch(const cwp_material* mats, int32_t n_mats, const int32_t* mat, const float* wo, const float* eta, int32_t gd_energy,
                          const float* ux, const float* uvw, float* wi, float* weight, float* pdf, int32_t* ok, int64_t n, const float* nr);

/* ------------------------------------------------------------------------------------------------------------------
 * Headless display transform. Replaces launchDisplay (app/display.cu, display.h:9) without the viewer's graphics
 * interop: d_accum (w * h float4 radiance sums over spp samples) -> d_rgba (w * h RGBA8). Mode 0 = the PNG transform
 * (io/image.cpp tonemapSRGB8: divide by spp, clip, sRGB OETF); 1 = Reinhard; 2 = ACES fit; exposure in EV.
 * ------------------------------------------------------------------------------------------------------------------ */
int cwp_display(const float* d_accum, uint8_t* d_rgba, int64_t n, int32_t spp, float exposure_ev, int32_t mode, void* stream);

/* ------------------------------------------------------------------------------------------------------------------
 * Environment maps on the host. cwp_hdr_load replaces loadHDR (io/hdr_image.cpp:13-45): a Radiance RGBE file
 * (new-style run-length or flat scanlines, '-Y H +X W') into w x h x 3 floats, row 0 = top; rgb = NULL queries the
 * size. cwp_envmap_build replaces buildEnvMap's tables (scene/environment.cpp:7-38): texels = w x h float4 radiance x
 * strength, marg = h + 1 floats (CDF over rows), cond = h rows of w + 1 floats (CDF within each row), texel weight
 * luminance x sin(theta); the same float tables as the reference's for the same input.
 * ------------------------------------------------------------------------------------------------------------------ */
int cwp_hdr_load(const char* path, int32_t* w, int32_t* h, float* rgb);
int cwp_envmap_build(const float* rgb, int32_t w, int32_t h, float strength, float* texels, float* marg, float* cond);

/* ------------------------------------------------------------------------------------------------------------------
 * Emissive triangles of an instanced scene at one frame, as the serving form light-samples them. Replaces the light
 * tables of SceneSetup::frameData (app/scene_setup.cpp:274-299): every instance in order, each emissive triangle of
 * its mesh in mesh order (material = mesh_mat_base[mesh] + face material, emissive when an emission component is
 * > 0), corners transformed by the instance's 3x4 rows (xforms, 12 floats per instance, as cwp_xform_animate gives),
 * power = luminance(emission) x area in double. em_tris: 3 float4 per triangle ((w0, global triangle id), (w1 - w0,
 * material), (w2 - w0, 0)); the global id (mesh's first triangle + face index) addresses the uvs of
 * cwp_server_set_textures. em_cdf: n_em + 1 floats, the CDF of power; mat_pdf: n_mats floats, luminance(emission) /
 * total power = the area density of sampling a point of that material. em_tris = NULL: *n_em only. A scene whose
 * emissive triangles have no area has n_em = 0.
 * ------------------------------------------------------------------------------------------------------------------ */
int cwp_emissive_tables(const cwp_mesh_view* meshes, int32_t n_meshes, const int32_t* mesh_mat_base, const cwp_material* mats, int32_t n_mats,
                        const float* xforms, const int32_t* inst_mesh, int64_t n_inst, float* em_tris, float* em_cdf, float* mat_pdf, int64_t* n_em);

/* ------------------------------------------------------------------------------------------------------------------
 * On-chip read bandwidth of a device, for the traversal kernels' roofline (not in the reference, whose node and
 * triangle reads are served from L2): `bytes` (1..96 MiB, L2-resident) read `reps` times per launch with 16-byte
 * L2-cached loads from every SM; *gbs = the best of five timed launches after a warm-up, in GB/s.
 * ------------------------------------------------------------------------------------------------------------------ */
int cwp_measure_l2_read(int64_t bytes, int32_t reps, int32_t device, double* gbs);

/* ------------------------------------------------------------------------------------------------------------------
 * Camera and parameter helpers. Replace lookAtC2W / focalFromHfov / makeCamera (scene/camera.cpp:7-23) and the
 * Params filling of setupScene (app/scene_setup.cpp:175-185, Lighting defaults scene/lighting.h:7-13).
 * ------------------------------------------------------------------------------------------------------------------ */
int cwp_camera_look_at(const float pos[3], const float target[3], const float up[3], float hfov_deg, int32_t w, int32_t h, cwp_camera* out);
int cwp_camera_from_c2w(const float c2w[16], float fx, float fy, int32_t w, int32_t h, cwp_camera* out);
/* defaults of the reference CLI: sun (0.3,-0.5,0.8) at 3 W/m^2, 0.526 deg, sky 0.3, seed 1000, box filter off */
int cwp_params_defaults(cwp_params* p);
int cwp_params_finish(cwp_params* p, float sun_angle_deg, float eps_scale, float scene_extent);   /* normalises sun_to, fills sun_cos, eps, ftab */

#ifdef __cplusplus
}
#endif
#endif
