/* C-ABI of the B200 beam tracer (libbt_gpu.so).
 *
 * Plain C types only: host pointers and sizes, caller-owned buffers, int
 * status codes (BT_OK = 0, negative = error; bt_gpu_last_error() describes
 * the last failure on the calling thread).  No call aborts the process.
 *
 * The entry points replace the GPU port of joelsalzman/beamtrace2007:
 *   bt_gpu_available        gpuAvailable            cuda/gpu_render.h:24
 *   bt_gpu_create/destroy   GpuRenderer ctor/dtor   cuda/gpu_render.h:28-29,
 *                                                   cuda/gpu_render.cu:489-541
 *   bt_gpu_soft             GpuRenderer::softShadows  cuda/gpu_render.h:36
 *   bt_gpu_soft_points      wfSoftShadows (shading points supplied)
 *                                                   cuda/gpu_common.cuh:148-150
 *   bt_gpu_primary          GpuRenderer::primary    cuda/gpu_render.h:41
 *   bt_gpu_point            GpuRenderer::pointShadows cuda/gpu_render.h:45-46
 *   bt_gpu_raster           rasterize (aa = 1)      src/render/render.h:29
 * and the host-side preparation the GPU path needs:
 *   bt_scene_finalize       Scene::finalize         src/scene/scene.cpp:89-118
 *   bt_kd_build             KdTree::build           src/accel/kdtree.h:36
 *   bt_kd_build_gpu         KdTree::build on the GPU (the same tree)
 *   bt_camera_make          Camera::make            src/render/render_types.h:24
 * and scene ingest (configs, OBJ/PLY meshes, procedural scenes):
 *   bt_scene_load_config    loadConfig + buildScene src/scene/scene.h:58-61
 *   bt_scene_parse_config   parseConfig + buildScene src/scene/scene.h:60-61
 * Batching and serving (no counterpart in the reference): bt_gpu_batch_soft,
 * bt_gpu_add_scene, bt_gpu_serve_start, bt_gpu_submit, bt_gpu_poll,
 * bt_gpu_serve_stats.
 */
#ifndef BT_GPU_H
#define BT_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BT_API __attribute__((visibility("default")))
#else
#define BT_API
#endif

enum {
  BT_OK = 0,
  BT_ERR_INVALID = -1,     /* bad argument */
  BT_ERR_CUDA = -2,        /* a CUDA call failed (message in bt_gpu_last_error) */
  BT_ERR_NOMEM = -3,       /* host or device allocation failed */
  BT_ERR_CAPACITY = -4,    /* a root needs more live sub-beams than the queues hold */
  BT_ERR_TIMEOUT = -5,     /* the round limit was reached */
  BT_ERR_NODEVICE = -6,    /* no usable CUDA device */
  BT_ERR_BUSY = -7,        /* serving: no free slot / memory budget for the request */
  BT_ERR_TOO_LARGE = -8    /* a size exceeds a fixed limit of the entry point */
};

/* Camera (render_types.h:15-39): image plane at distance 1 along fwd,
 * q in [-half_w, half_w] x [-half_h, half_h], ray dir = fwd + right qx + down qy. */
typedef struct {
  float eye[3], fwd[3], right[3], down[3];
  float half_w, half_h;
  int32_t W, H;
} bt_camera;

/* Square/parallelogram area light (soft_core.h:10-14): centre and full edge
 * vectors; emits along normalize(U x V). */
typedef struct {
  float c[3], U[3], V[3];
} bt_area_light;

/* Finalised scene (see bt_scene_finalize): vertex positions, triangles and
 * unit normals; bounds = lo xyz, hi xyz of the triangles' vertices. */
typedef struct {
  const float* pos;
  int64_t num_verts;
  const uint32_t* tris;
  const float* tri_normals;
  int64_t num_tris;
  float bounds[6];
} bt_scene_desc;

/* kd-tree in structure-of-arrays form (KdNode split/data/offset, parent
 * links, node boxes lo xyz hi xyz, leaf triangle lists, root box). */
typedef struct {
  const float* split;
  const uint32_t* data;
  const uint32_t* offset;
  const uint32_t* parent;
  const float* node_box;
  int64_t num_nodes;
  const uint32_t* tri_indices;
  int64_t num_refs;
  float bounds[6];
} bt_kd_desc;

typedef struct {
  float cost_traverse, cost_intersect, empty_bonus;
  int32_t max_depth, bin_threshold, bins, clip_bounds, single_leaf;
} bt_kd_params;

typedef struct bt_kd_tree bt_kd_tree;

typedef struct {
  char name[256];
  int32_t sm_count;
  double mem_gb;
  int32_t cc_major, cc_minor;
} bt_gpu_info;

/* Engine tunables (GpuRenderer public fields, gpu_render.h:50-58). */
typedef struct {
  int32_t device;           /* CUDA device ordinal */
  int32_t budget;           /* live sub-beams per soft/point root before it is abandoned and retried with 16x
                               (wfBudget; default 2048, the reference's 128 x 16) */
  int32_t primary_budget;   /* live sub-beams per primary tile (wfPrimaryBudget; default 4096).  A root
                               reserves min(budget, 128) queue slots when admitted and takes more from the
                               queues' free capacity as it grows; past its budget, or when the queues
                               cannot cover it, it is abandoned and retried with 16x the budget; the last
                               retry pass (max_retries) reserves each root's whole budget, at most a queue */
  int64_t capacity;         /* sub-beam records per spill queue (wfCapacity); 0 = 2^25, at most a tenth of
                               the free device memory over the three queues */
  int32_t blocks_per_sm;    /* persistent CTAs per SM; 0 = occupancy */
  int32_t kernel_timing;    /* nonzero: CUDA events around the trace kernels fill ms_kernel_trace */
  int32_t max_retries;      /* budget x16 retries before BT_ERR_CAPACITY */
  int64_t tail_records;     /* tail rounds (one fused trace-and-clip kernel) below this many queued
                               records once every root is admitted; 0 = a sixth of the trace grid's lanes, < 0 = never */
  int32_t eps_stats;        /* nonzero: trace kernels that also count the edge votes in the fuzzy band
                               and their FP64 re-evaluation (eps_band_corners, eps_fp64_flips); results
                               are the same, the kernels are slower */
  int32_t yield_pct;        /* once a round's trace queue is drained and this percentage of the trace
                               warps has exited, the records still in flight go on in the next round
                               instead of holding the round (results are the same); 0 = 50, < 0 = never */
  int32_t fuse_primary;     /* nonzero: bt_gpu_soft(_device) trace each pixel's eye ray in the admission of
                               its shadow root instead of a separate primary-ray pass (same results) */
  int32_t eps_fp64;         /* nonzero (soft shadows): beam corners whose float distance to a triangle edge
                               line falls inside the fuzzy band are re-decided with the edge line in FP64
                               (from the same float vertices) in the votes and the clip, before a split;
                               results then differ from the reference's float build (eps_band_corners and
                               eps_fp64_flips count the band corners and the re-decided ones) */
  int32_t graph_rounds;     /* nonzero (default): each batch of rounds (the admit / trace / clip /
                               bookkeeping launches between two looks at the counters) is replayed as one
                               CUDA graph, captured again only when the launch parameters change (the
                               executable graph updated in place); same results.  Off with kernel_timing */
  int32_t trace_ctas;       /* CTAs per SM of the full-round trace kernel: 3 (up to 170 registers a
                               thread) or 4 (128, a few spills, more warps to hide latency); 0 = 4 for
                               scenes up to 16 MB on the device, else 3; same results */
} bt_gpu_config;

typedef struct {
  int32_t exact;            /* Lambert's formula over the visible light (E) instead of eq. 2 */
  float offset;             /* apex offset along the normal; <= 0: |scene diagonal| * 2e-5 */
} bt_soft_opts;

/* Counters (TraceStats, src/util/stats.h:8-42) and engine figures of the last call. */
typedef struct {
  uint64_t kd_steps, leaf_visits, tri_tests, hits, splits, beams, root_beams, presplit_beams, five_splits, climbs;
  double dropped_area;
  uint64_t eps_band_corners;  /* eps_stats: edge-vote corners inside the fuzzy band (traced records) */
  uint64_t eps_fp64_flips;    /* of those, corners whose FP64 re-evaluation lies outside the band */
  double ms_primary, ms_trace, ms_total;
  double ms_round;            /* summed device time of the persistent round kernels */
  int32_t launches;           /* kernels launched by the call */
  int32_t round_launches;     /* of those, persistent round kernels */
  int32_t passes, retried_roots, max_spill;
  int64_t roots;
  int32_t rounds;             /* rounds run (each: admit, trace, clip, bookkeeping launches) */
  int32_t tail_rounds;        /* of those, tail rounds (fused trace and clip, bookkeeping) */
  /* summed device time of the trace launches (kernel_timing only, else 0); admit and clip reserved (0) */
  double ms_kernel_admit, ms_kernel_trace, ms_kernel_clip;
  int64_t yields;             /* records handed on unfinished to the next round (yield_pct) */
  int64_t overflow_roots;     /* roots over budget in their first pass: the reference recomputes these on
                                 the CPU (lastOverflowPixels), here they are retried on the GPU */
} bt_run_info;

/* Beam cross-sections on a query plane (OutBeam, beam_types.h:68-73):
 * x/y hold 4 corners per polygon (the last corner repeated when n = 3). */
typedef struct {
  float* x;
  float* y;
  int32_t* n;
  int32_t* tri;
  float* area;
  int32_t* root;  /* index of the root (tile / hit beam) it came from; may be NULL */
  int64_t cap;
} bt_polys;

typedef struct bt_gpu_ctx bt_gpu_ctx;

BT_API const char* bt_gpu_last_error(void);
BT_API void bt_gpu_config_default(bt_gpu_config* cfg);

/* ---- host-side scene preparation ---- */
BT_API int64_t bt_scene_finalize(const float* pos, int64_t num_verts, const uint32_t* tris_in, int64_t num_tris_in,
                                 uint32_t* tris_out, float* tri_normals, float* tri_area, float* bounds);
BT_API void bt_kd_params_default(bt_kd_params* p);
BT_API int bt_kd_build(const float* pos, const uint32_t* tris, const float* tri_area, int64_t num_tris,
                       const float* scene_bounds, const bt_kd_params* params, bt_kd_tree** out);
BT_API void bt_kd_sizes(const bt_kd_tree* t, int64_t* num_nodes, int64_t* num_refs, int32_t* num_leaves,
                        int32_t* max_depth);
BT_API void bt_kd_view(const bt_kd_tree* t, bt_kd_desc* d);
BT_API void bt_kd_free(bt_kd_tree* t);
/* The same tree, node for node, built on CUDA device `device` (level by
 * level: binned SAH histograms and exact event sweeps per node, partition
 * with clipping, leaf sorting on the device; the host numbers the nodes).
 * num_verts bounds the triangle indices.  *ms (may be NULL): wall-clock time
 * of the call.  Free the tree with bt_kd_free. */
BT_API int bt_kd_build_gpu(const float* pos, int64_t num_verts, const uint32_t* tris, const float* tri_area,
                           int64_t num_tris, const float* scene_bounds, const bt_kd_params* params, int32_t device,
                           bt_kd_tree** out, double* ms);
BT_API void bt_camera_make(const float* eye, const float* target, float fov_y, const float* up, int32_t W, int32_t H,
                           bt_camera* cam);

/* ---- scene ingest (SceneConfig and Scene, src/scene/scene.h:13-61) ----
 * A config is lines of `key values` (# comments): name, mesh (obj PATH |
 * ply PATH | procedural NAME [key=value ...], with optional `scale s`,
 * `translate x y z`, `color r g b`), cull_backfaces, up, view (eye target
 * fov), orbit, walk, point_light, area_light (centre and full edge
 * vectors), light_intensity, background.  Mesh paths are taken as written
 * (relative ones from the working directory).  The scene is the one the
 * reference builds from the same config, float for float, with its
 * degenerate triangles removed (bt_scene_finalize's rule).  Errors:
 * BT_ERR_INVALID with the reason in bt_gpu_last_error(). */
typedef struct bt_scene_file bt_scene_file;
typedef struct {
  char name[128];
  int64_t num_verts, num_tris, num_materials, num_views;
  int32_t cull_backfaces, has_point_light, has_area_light;
  float up[3];
  float point_light[3];
  float light_c[3], light_u[3], light_v[3];
  float light_intensity;
  float background[3];
} bt_scene_file_info;
BT_API int bt_scene_load_config(const char* path, bt_scene_file** out);
BT_API int bt_scene_parse_config(const char* text, bt_scene_file** out);
BT_API void bt_scene_file_info_get(const bt_scene_file* f, bt_scene_file_info* info);
/* pos: 3 x num_verts; tris: 3 x num_tris; tri_mat: num_tris; mat_color:
 * 3 x num_materials; views: 7 x num_views (eye, target, fov in degrees).
 * Any pointer may be NULL. */
BT_API void bt_scene_file_arrays(const bt_scene_file* f, float* pos, uint32_t* tris, uint16_t* tri_mat,
                                 float* mat_color, float* views);
BT_API void bt_scene_file_free(bt_scene_file* f);

/* ---- device ---- */
BT_API int bt_gpu_available(bt_gpu_info* info);
BT_API int bt_gpu_create(const bt_scene_desc* scene, const bt_kd_desc* kd, const bt_gpu_config* cfg,
                         bt_gpu_ctx** out);
BT_API int bt_gpu_destroy(bt_gpu_ctx* ctx);

/* Adds another finalised scene and its kd-tree to the context's scene pool
 * (no counterpart in the reference); *scene_id names it in batch jobs.  The
 * scene of bt_gpu_create is id 0 and stays the one the single-image entry
 * points render. */
BT_API int bt_gpu_add_scene(bt_gpu_ctx* ctx, const bt_scene_desc* scene, const bt_kd_desc* kd, int32_t* scene_id);

/* Exact soft shadows of a W x H image: GPU primary rays (tri, shading point,
 * normal per pixel centre), then one shadow-beam root per covered pixel.
 * Outputs (host, W*H each, any may be NULL): tri (-1 background), vis
 * (visible light fraction; -1 background, 0 below the horizon), E
 * (exact: Lambert integral over the visible light; else A*G0*V), Eu (A*G0). */
BT_API int bt_gpu_soft(bt_gpu_ctx* ctx, const bt_camera* cam, const bt_area_light* light, const bt_soft_opts* opts,
                       int32_t* tri, float* vis, float* E, float* Eu, bt_run_info* info);

/* Soft shadows for n supplied shading points (host arrays: tri[n], X[3n],
 * N[3n]; tri < 0 = nothing to shade). */
BT_API int bt_gpu_soft_points(bt_gpu_ctx* ctx, const bt_area_light* light, const bt_soft_opts* opts, int64_t n,
                              const int32_t* tri, const float* X, const float* N, float* vis, float* E, float* Eu,
                              bt_run_info* info);

/* The same on device-resident buffers (device pointers).  The work runs on
 * the context's own stream, which does not wait for other streams: the
 * inputs must be complete when the call is made (synchronise the stream
 * that wrote them first); the call returns when the outputs are written. */
BT_API int bt_gpu_soft_points_device(bt_gpu_ctx* ctx, const bt_area_light* light, const bt_soft_opts* opts, int64_t n,
                                     const int32_t* d_tri, const float* d_X, const float* d_N, float* d_vis,
                                     float* d_E, float* d_Eu, bt_run_info* info);

/* Size of the device scratch array inside this library that
 * bt_gpu_soft_points_noalloc works in: 64 MiB, held on every GPU that has
 * loaded the library until the process exits. */
#define BT_NOALLOC_SCRATCH_BYTES (64ll << 20)

/* bt_gpu_soft_points_device for callers that cannot allocate device memory.
 * No counterpart in the reference.
 *
 * Who needs it: a host application whose own allocator owns the GPU's
 * memory (a renderer's or a framework's memory pool) and hands this library
 * buffers from that pool.  cudaMalloc beside such a pool fails once the pool
 * holds the memory, and cudaFree stalls every stream on the device while the
 * application is mid-frame.  This call allocates nothing and needs no
 * bt_gpu_ctx: the caller passes the scene and the shading points in its own
 * device buffers; everything else comes from one fixed scratch array inside
 * the library.
 *
 * Inputs: d_scene and d_kd are the finalised scene and its kd-tree as
 * bt_scene_finalize and bt_kd_build produce them, with every pointer member
 * a device address on the current device (counts and bounds are host
 * values); d_tri[n], d_X[3n], d_N[3n] the shading points as for
 * bt_gpu_soft_points_device.  Outputs d_vis, d_E, d_Eu (n each, any may be
 * NULL) are device buffers.  Results equal bt_gpu_soft_points_device's on
 * the same inputs.
 *
 * Limit: the scene in the engine's layout (44 bytes per kd node, 64 per
 * reference, 32 per triangle), 168 bytes per point and three sub-beam queues
 * of at least 8192 64-byte records must fit in BT_NOALLOC_SCRATCH_BYTES
 * (each section rounded up to 256 bytes); larger calls return
 * BT_ERR_TOO_LARGE before any GPU work.  A kd-tree whose indices are out of
 * range or out of order returns BT_ERR_INVALID, as do triangle references
 * or vertex indices out of range.
 *
 * BT_ERR_CAPACITY can come back here where bt_gpu_soft_points_device
 * succeeds: the queues get what the fixed array leaves over (at most about
 * 349,000 records each, against 2^25 on a context).  Roots take queue slots
 * from that pool as they grow; a root over its budget (2048 live
 * sub-beams) or one the pool cannot cover is abandoned and retried with
 * 16 times the budget, and the last of four retries admits roots one queue
 * at a time: the call fails, with a message that names the queue size,
 * only for a root that needs more live sub-beams than one queue of the
 * pool holds, and takes longer the more roots the small pool squeezes.
 *
 * Runs on the current device's legacy default stream and returns when the
 * results are complete.  That stream waits for all work already queued on
 * the device's blocking streams and holds back their later work until this
 * call's kernels finish: a caller that keeps its own streams running
 * alongside should create them with cudaStreamNonBlocking, and must itself
 * finish the work that writes the inputs before the call (synchronise the
 * stream that wrote them).  The first call on a device sets up (looks up the
 * scratch array's device address, creates two timing events): make it
 * before any stream capture.  All calls on a device share the scratch array,
 * which keeps the last call's contents; each call clears what must start at
 * zero.  Calls whose GPU work overlaps race on the array: this library
 * serialises its own calls per device within a process, so do not run this
 * entry point on the same device from another library copy or module at the
 * same time. */
BT_API int bt_gpu_soft_points_noalloc(const bt_scene_desc* d_scene, const bt_kd_desc* d_kd,
                                      const bt_area_light* light, const bt_soft_opts* opts, int64_t n,
                                      const int32_t* d_tri, const float* d_X, const float* d_N, float* d_vis,
                                      float* d_E, float* d_Eu, bt_run_info* info);

/* bt_gpu_soft on device buffers (W*H each; d_vis/d_E/d_Eu may be NULL):
 * everything stays in device memory.  Runs on the context's stream and
 * returns when the results are complete. */
BT_API int bt_gpu_soft_device(bt_gpu_ctx* ctx, const bt_camera* cam, const bt_area_light* light,
                              const bt_soft_opts* opts, int32_t* d_tri, float* d_vis, float* d_E, float* d_Eu,
                              bt_run_info* info);

/* One soft-shadow job of a batch: an image W x H from cam of one scene of
 * the context's pool, its light and options, and its outputs in device
 * memory (W*H each; any may be NULL; tri ids are the scene's own). */
typedef struct {
  bt_camera cam;
  bt_area_light light;
  bt_soft_opts opts;
  int32_t* d_tri;
  float* d_vis;
  float* d_E;
  float* d_Eu;
  int32_t scene;            /* 0: the context's own scene; else an id from bt_gpu_add_scene */
} bt_soft_job;

/* bt_gpu_soft_device for num_jobs images of the context's scene in one
 * run of the engine: the shadow-beam roots of all jobs share the rounds,
 * so one job's tail overlaps the others' work.  Each job's outputs equal
 * what bt_gpu_soft_device gives for it alone.  Returns when all are done. */
BT_API int bt_gpu_batch_soft(bt_gpu_ctx* ctx, int32_t num_jobs, const bt_soft_job* jobs, bt_run_info* info);

/* GPU primary rays only (primaryKernel, cuda/gpu_render.cu:222-244): per
 * pixel centre the nearest triangle (-1 none), hit point X (3 floats) and
 * normal N facing the eye.  Host buffers (_device: device buffers). */
BT_API int bt_gpu_primary_rays(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t* tri, float* X, float* N);
BT_API int bt_gpu_primary_rays_device(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t* d_tri, float* d_X, float* d_N);

/* Primary visibility, one root per tile x tile pixels: the visible
 * polygons (image plane) in `out`; *count = number produced (may exceed
 * out->cap: then only cap were written and the call should be repeated
 * with a larger buffer). */
BT_API int bt_gpu_primary(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t cull, int32_t tile, bt_polys* out,
                          int64_t* count, bt_run_info* info);

/* Point-light shadows for `hits` (primary hit polygons, image plane), one
 * root per polygon: the shadowed image-plane polygons are written to out
 * (root = index into hits). */
BT_API int bt_gpu_point(bt_gpu_ctx* ctx, const bt_camera* cam, const bt_polys* hits, int64_t num_hits,
                        const float* light, bt_polys* out, int64_t* count, bt_run_info* info);

/* The polygons of the last bt_gpu_primary / bt_gpu_point call on ctx
 * again, into a (larger) buffer: when a call reports more polygons than
 * out->cap held, fetch them with this instead of repeating the call.  They
 * stay on the device until the context's next engine call (BT_ERR_INVALID
 * after it).  Serves the retry loops of GpuRenderer::primary / pointShadows
 * (cuda/gpu_render.h:41-46), which the reference sizes on the host. */
BT_API int bt_gpu_last_polys(bt_gpu_ctx* ctx, bt_polys* out, int64_t* count);

/* Primary visibility to per-pixel hit-triangle ids (-1 background) with the
 * polygons kept in device memory: the engine's tile roots, then the pixel-
 * centre raster of the final polygons on the GPU (rasterize,
 * render.cpp:49-95, at aa = 1; a pixel centre on a shared edge takes the
 * larger id).  Host output (W*H) / device output (_device). */
BT_API int bt_gpu_primary_ids(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t cull, int32_t tile, int32_t* tri,
                              bt_run_info* info);
BT_API int bt_gpu_primary_ids_device(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t cull, int32_t tile,
                                     int32_t* d_tri, bt_run_info* info);

/* Point-light shadow mask (1 = in shadow) of the primary hits, all in device
 * memory: primary roots, their final hit polygons as point-shadow roots,
 * the shadowed polygons rasterised at pixel centres; optionally the ids
 * too (tri / d_tri may be NULL).  Host outputs (W*H) / device (_device). */
BT_API int bt_gpu_point_mask(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t cull, int32_t tile, const float* light,
                             int32_t* tri, uint8_t* mask, bt_run_info* info);
BT_API int bt_gpu_point_mask_device(bt_gpu_ctx* ctx, const bt_camera* cam, int32_t cull, int32_t tile,
                                    const float* light, int32_t* d_tri, uint8_t* d_mask, bt_run_info* info);

/* Rasterises polygons at pixel centres (rasterize, render.cpp:49-95, aa = 1)
 * on the GPU: prim polygons write tri ids (-1 elsewhere), shadow polygons
 * set flag = 1.  tri and flag are host buffers of W*H. */
BT_API int bt_gpu_raster(bt_gpu_ctx* ctx, const bt_camera* cam, const bt_polys* prim, int64_t num_prim,
                         const bt_polys* shadow, int64_t num_shadow, int32_t* tri, uint8_t* flag);

/* ---- serving: continuous batching behind submit / poll ----
 *
 * The batched and served variants of the entry points above (no counterpart
 * in the reference, whose GpuRenderer calls are synchronous, one image at a
 * time: cuda/gpu_render.h:26-46).  Requests name a scene of the context's
 * pool and carry host output buffers; bt_gpu_submit queues one and returns
 * at once, bt_gpu_poll hands back finished ones.  Behind them, serving
 * threads keep the scenes resident and run requests on lanes -- engine
 * buffers and a stream of their own on the context's device, so that
 * requests overlap on the GPU:
 *  - soft-shadow requests go to the soft lane, whose engine run folds in
 *    requests that arrive while it goes on: their roots join the rounds
 *    already in flight (for fold_ms after the run started), and each request
 *    is handed back as soon as its own roots are done;
 *  - primary-id and point-shadow-mask requests go to `vis_lanes` lanes, one
 *    request per lane at a time.
 * Each result equals what bt_gpu_soft / bt_gpu_primary_ids / bt_gpu_point_mask
 * give for the request alone.  Admission: a request is refused with
 * BT_ERR_BUSY while the resident scenes, the lanes' sub-beam queue high-water
 * mark and the requests already admitted would exceed memory_budget. */
enum { BT_REQ_SOFT = 0, BT_REQ_PRIMARY_IDS = 1, BT_REQ_POINT_MASK = 2 };

typedef struct {
  int32_t kind;              /* BT_REQ_* */
  int32_t scene;             /* scene id of the context's pool (0: the context's own) */
  bt_camera cam;
  bt_area_light light;       /* BT_REQ_SOFT */
  bt_soft_opts opts;         /* BT_REQ_SOFT */
  float point_light[3];      /* BT_REQ_POINT_MASK */
  int32_t cull, tile;        /* BT_REQ_PRIMARY_IDS / BT_REQ_POINT_MASK (tile 0: 16) */
  /* host outputs, W*H each, any may be NULL: ids (the scene's own, -1
   * background), visibility, E, Eu (soft), mask (point) */
  int32_t* tri;
  float* vis;
  float* E;
  float* Eu;
  uint8_t* mask;
  uint64_t user;             /* handed back with the completion */
} bt_request;

typedef struct {
  uint64_t ticket, user;
  int32_t kind, status;      /* status: BT_OK or the request's error code */
  double ms_queued;          /* submit to start (soft: to joining a run) */
  double ms_total;           /* submit to hand-back */
  char error[160];
} bt_completion;

typedef struct {
  int32_t vis_lanes;         /* lanes for primary ids and point masks (0: 4) */
  int32_t soft_jobs;         /* requests one soft run holds at most (0: 256) */
  int64_t soft_pixels;       /* pixels one soft run holds at most (0: 8M) */
  int64_t capacity;          /* sub-beam records per queue of each lane (0: the context's) */
  double fold_ms;            /* soft requests join a running soft run this long after it starts (0: 100) */
  int64_t memory_budget;     /* bytes (0: no limit) */
  int32_t soft_blocks_per_sm;  /* CTAs per SM of the soft lane's persistent kernels (<= 0: as many as
                                  fit).  Fewer leave room on every SM for the visibility lanes' kernels
                                  beside a running soft run; measured, 1 or 2 made both kinds slower */
} bt_serve_config;

typedef struct {
  int64_t submitted, completed, refused, queued, running;
  int64_t soft_runs;         /* streaming soft runs so far */
  int64_t soft_folded;       /* soft requests that joined a run after it had started */
  int64_t scene_bytes;       /* the resident scene pool */
  int64_t lane_bytes;        /* the lanes' engine buffers as allocated */
  int64_t queue_high_water;  /* bytes of sub-beam records the lanes have needed at most */
  int64_t admitted_bytes;    /* the requests in flight, as admission charges them */
} bt_serve_stats;

/* Starts serving with `cfg` (NULL: defaults); bt_gpu_submit starts it with
 * defaults if this was not called.  BT_ERR_INVALID if already started. */
BT_API int bt_gpu_serve_start(bt_gpu_ctx* ctx, const bt_serve_config* cfg);
/* Queues a request; *ticket names it in its completion.  BT_ERR_BUSY: over
 * the memory budget now (submit again later); BT_ERR_INVALID: bad request.
 * The output buffers must stay valid until the request is handed back. */
BT_API int bt_gpu_submit(bt_gpu_ctx* ctx, const bt_request* req, uint64_t* ticket);
/* Hands back up to `cap` finished requests (in the order they finished),
 * waiting up to wait_ms for the first (0: no wait, < 0: until one
 * finishes or nothing is in flight). */
BT_API int bt_gpu_poll(bt_gpu_ctx* ctx, bt_completion* out, int32_t cap, int32_t* count, int32_t wait_ms);
BT_API int bt_gpu_serve_stats(bt_gpu_ctx* ctx, bt_serve_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* BT_GPU_H */
