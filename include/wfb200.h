/*
 * wfb200 -- C ABI of the B200 path-tracing engine (libwfb200.so).
 *
 * Plain pointers, sizes and opaque handles; no C++ types, no exceptions across the boundary.
 * Every function returns a status (WFB_OK = 0) unless stated otherwise; the message of the last
 * failure on the calling thread is returned by wfb_last_error().
 *
 * Each entry point names the reference interface it replaces (paths inside the reference
 * project us-llm-engineer/graphics-book-tutorials, WVM = wavefront-vs-megakernel-path-tracing).
 * Host array layouts are the reference's public structs (WVM/include/wf/scene.hpp:12-100):
 *   sphere 32 B {float center[3], radius; int material, pad[3]}
 *   vertex 12 B {float x, y, z}
 *   triangle 16 B {int i0, i1, i2, material}
 *   material 48 B {int type; float ior, pad0, pad1; float albedo[3], pad2; float emission[3], pad3}
 *   BVH node 48 B {float lo[3]; int skip; float hi[3]; int prim_start, prim_count, pad[3]}
 *   light 16 B {int prim; float area, pad[2]}
 */
#ifndef WFB200_H
#define WFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WFB_ABI_VERSION 1

/* Status codes. */
#define WFB_OK 0
#define WFB_ERR_INVALID_ARGUMENT 1 /* bad handle, size, index or parameter */
#define WFB_ERR_CUDA 2             /* a CUDA runtime call failed (message has the CUDA string) */
#define WFB_ERR_OUT_OF_MEMORY 3    /* device allocation failed or a memory budget is exceeded */
#define WFB_ERR_NOT_FINALIZED 4    /* scene has no BVH nodes (reference: std::runtime_error) */
#define WFB_ERR_UNSUPPORTED 5      /* valid input outside this engine's packed limits */
#define WFB_ERR_TIMEOUT 6          /* a host-side wait ended before completion */
#define WFB_ERR_DEVICE_WAIT 7      /* a bounded device-side wait gave up (kernel returned early) */
#define WFB_ERR_INTERNAL 8

#define WFB_MODE_MEGAKERNEL 0 /* wf::GpuMode::Megakernel */
#define WFB_MODE_WAVEFRONT 1  /* wf::GpuMode::Wavefront */

typedef struct wfb_scene* wfb_scene_t;
typedef struct wfb_renderer* wfb_renderer_t;

/* Library */
int wfb_abi_version(void);
const char* wfb_last_error(void);
/* Writes the CUDA device name; replaces wf::GpuRenderer::device_name (WVM/src/gpu/gpu_renderer.cu:379-390). */
int wfb_device_name(char* buf, int len);
/* Facts of the current CUDA device; replaces wf::query_cuda_device (WVM/src/gpu/gpu_renderer.cu:13-56). */
typedef struct {
    char name[256];
    int driver_version;  /* cudaDriverGetVersion, e.g. 12090 */
    int runtime_version; /* cudaRuntimeGetVersion of this library */
    int cc_major, cc_minor;
    int sm_count;
    uint64_t total_memory_bytes, free_memory_bytes;
    /* L2 (no reference counterpart): size, the largest persisting set-aside, the largest
     * access-policy window, and the largest wavefront pool (paths) that fits the set-aside */
    uint64_t l2_bytes, persisting_l2_max_bytes, access_window_max_bytes;
    int wavefront_l2_resident_paths;
    int wavefront_slot_bytes;
    uint64_t persisting_l2_set_aside_bytes; /* this process's current set-aside (0 when no pool holds a window) */
} wfb_device_facts;
int wfb_device_facts_get(wfb_device_facts* out);

/* ---- scenes ---------------------------------------------------------------------------------
 * Host description of a scene in the reference layouts. n_nodes == 0 means "not finalized". */
typedef struct {
    const void* spheres;     int n_spheres;
    const float* vertices;   int n_vertices;
    const int* triangles;    int n_triangles;
    const void* materials;   int n_materials;
    const void* nodes;       int n_nodes;
    const int* prim_order;   int n_prim_order;
    const void* lights;      int n_lights;
    float env[3];
    float cam_position[3];
    float cam_look_at[3];
    float cam_up[3];
    float cam_vfov_deg;
    int width, height;
} wfb_scene_desc;

typedef struct {
    int n_spheres, n_vertices, n_triangles, n_materials, n_nodes, n_prim_order, n_lights;
    int width, height;
    float env[3];
    float cam_position[3], cam_look_at[3], cam_up[3], cam_vfov_deg;
} wfb_scene_info;

/* Copies the description. finalize_bins == 0: the scene must already be finalized (its nodes,
 * prim_order and lights are used as given, like wf::GpuRenderer's constructor,
 * WVM/src/gpu/gpu_renderer.cu:100-104); finalize_bins > 0: validate, collect lights and build the
 * BVH with that many SAH bins, like wf::finalize_scene (WVM/src/scene.cpp:58-104; 8 bins reproduces
 * the reference tree). The scene is uploaded to the current device on first use. */
int wfb_scene_create(const wfb_scene_desc* desc, int finalize_bins, wfb_scene_t* out);
/* Procedural benchmark scene "cornell36", "icospheres" or "heightfield" (no reference
 * counterpart: the reference's make_scene, WVM/src/scenes.cpp:29, has other scenes). */
int wfb_scene_generate(const char* name, int width, int height, uint32_t seed, int sah_bins,
                       wfb_scene_t* out);
int wfb_scene_info_get(wfb_scene_t scene, wfb_scene_info* info);
/* *nested = 1 when the scene's BVH is a properly nested preorder tree (every node's box inside the
 * box of each node whose subtree -- the nodes before its skip link -- holds it): the condition for
 * exact speculative closest-hit traversal (wfb_renderer_set_speculation). Host only. */
int wfb_scene_boxes_nested(wfb_scene_t scene, int* nested);
/* Copies the finalized host arrays into caller buffers sized from wfb_scene_info (any pointer
 * may be NULL to skip that array). */
int wfb_scene_export(wfb_scene_t scene, void* spheres, float* vertices, int* triangles,
                     void* materials, void* nodes, int* prim_order, void* lights);
/* Replaces wf::scene_hash (WVM/src/scene.cpp:107-160). */
uint64_t wfb_scene_hash(wfb_scene_t scene);
/* Rebuilds the BVH of a scene not yet uploaded, with SAH knobs: bins (8 = reference-compatible
 * policy), leaves of at most max_leaf primitives (1..15), traversal_cost relative to one
 * primitive test. Replaces wf::build_bvh (WVM/src/bvh_build.cpp:228-251) for tuning; the tree
 * stays in the preorder skip-link layout. Subtrees are built on `threads` host threads (0: all
 * cores); the tree is the same for every thread count. */
int wfb_scene_rebuild_bvh(wfb_scene_t scene, int bins, int max_leaf, float traversal_cost, int threads);
/* Replaces wf::validate_bvh (WVM/src/bvh_build.cpp:253-323): writes "" when valid. */
int wfb_scene_validate_bvh(wfb_scene_t scene, char* msg, int len);
/* Releases the caller's reference; device arrays live until the last renderer using them is gone. */
int wfb_scene_destroy(wfb_scene_t scene);
/* Device bytes of the resident (uploaded) scene; 0 before the first upload. */
uint64_t wfb_scene_device_bytes(wfb_scene_t scene);

/* ---- renderer: the wf::GpuRenderer class (WVM/include/wf/renderer.hpp:44-67) ----------------- */
typedef struct {
    int spp;
    uint32_t seed;
    int max_depth;
    int count_rays;
    int stage_timing;
    int queue_capacity;
} wfb_render_params; /* wf::RenderParams (WVM/include/wf/renderer.hpp:11-21) */

typedef struct {
    double render_ms;
    double total_ms;
    uint64_t extension_rays, shadow_rays;
    int64_t queue_high_water[5];
    int64_t queue_overflows;
    int64_t invalid_hits;
    uint64_t peak_vram_bytes;
    double stage_ms[8]; /* extend, classify, lambert, metal, dielectric, shadow, compact, other */
    uint64_t node_visits; /* megakernel, with count_rays: BVH nodes visited (box tests) */
    uint64_t prim_tests;  /* megakernel, with count_rays: primitive intersection tests */
    uint64_t kernel_launches; /* kernels of this library launched by the call */
    double kernel_ms;         /* device time of the main kernel launches alone (persistent megakernel or
                                 wavefront kernel; CUDA events on the launching stream) */
} wfb_render_stats; /* wf::RenderStats (WVM/include/wf/renderer.hpp:23-37) plus traversal counts */

/* GpuRenderer(const Scene&, GpuMode) (WVM/src/gpu/gpu_renderer.cu:100-238). */
int wfb_renderer_create(wfb_scene_t scene, int mode, wfb_renderer_t* out);
/* Camera and resolution of the scene by default; this overrides them (film is reallocated and
 * zeroed). No reference counterpart (the reference binds the camera to the Scene). */
int wfb_renderer_set_camera(wfb_renderer_t r, const float position[3], const float look_at[3],
                            const float up[3], float vfov_deg, int width, int height);
/* GpuRenderer::reset (WVM/src/gpu/gpu_renderer.cu:242-252). */
int wfb_renderer_reset(wfb_renderer_t r);
/* GpuRenderer::run_passes (WVM/src/gpu/gpu_renderer.cu:254-304): adds samples
 * [first_sample, first_sample + count) to the film. stats may be NULL. */
int wfb_renderer_run_passes(wfb_renderer_t r, int first_sample, int count,
                            const wfb_render_params* p, wfb_render_stats* stats);
/* GpuRenderer::download (WVM/src/gpu/gpu_renderer.cu:306-341): rgb = sum * (1/spp) in float,
 * lum_var = max(0, E[l^2] - E[l]^2) in double. rgb: 3*w*h floats, lum_var: w*h (may be NULL). */
int wfb_renderer_download(wfb_renderer_t r, int spp_done, float* rgb, float* lum_var);
/* GpuRenderer::download_mean (WVM/src/gpu/gpu_renderer.cu:343-353). */
int wfb_renderer_download_mean(wfb_renderer_t r, int spp_done, float* rgb);
/* Raw film sums (rgb 3*w*h, lum w*h, lum2 w*h), the bit-exact comparison surface. */
int wfb_renderer_download_sums(wfb_renderer_t r, float* rgb_sum, float* lum_sum, float* lum2_sum);
/* GpuRenderer::render (WVM/src/gpu/gpu_renderer.cu:355-364): reset, run_passes(0, spp), download. */
int wfb_renderer_render(wfb_renderer_t r, const wfb_render_params* p, wfb_render_stats* stats,
                        float* rgb, float* lum_var);
/* GpuRenderer::device_bytes (WVM/src/gpu/gpu_renderer.cu:366-377). */
uint64_t wfb_renderer_device_bytes(wfb_renderer_t r);
/* Launch configuration knobs (no reference counterpart; set by the autotuner). Any value < 0
 * keeps the current setting. Megakernel: block 64/128/256 threads, CTAs per SM (0: all that fit),
 * the minimum number of traversing lanes per warp before shading runs (1..32), work units per
 * pixel (0: automatic), occupancy target (block 128: 0 none, 6, 8 or 10 CTAs per SM by a register
 * cap), and leaf_batch (1..32): a warp runs a round of primitive tests once this many of its
 * lanes hold a pending leaf (or they outnumber the lanes testing boxes). Wavefront: paths in
 * flight, min_active, leaf_batch and occupancy (0, 6, 8 or 10 CTAs of 128 threads per SM). */
int wfb_renderer_configure(wfb_renderer_t r, int block, int blocks_per_sm, int min_active,
                           int split_chunks, int paths_in_flight, int occupancy, int leaf_batch);
/* Wavefront path pool resident in L2 (no reference counterpart; the reference's pool is W*H paths
 * in plain device memory, WVM/src/gpu/wavefront.cu:11-26): every wavefront launch carries a
 * persisting access-policy window over the pool, backed by the context's persisting-L2 set-aside.
 * mode -1 (default): when the pool fits the device's persisting set-aside; 0: never; 1: always
 * (a larger pool gets a window with a hit ratio below 1). Megakernel renderers ignore it. */
int wfb_renderer_set_l2_residency(wfb_renderer_t r, int mode);
/* Bytes of the wavefront pool under the persisting window (0: none). */
uint64_t wfb_renderer_l2_window_bytes(wfb_renderer_t r);
/* Speculative traversal in both arms (no reference counterpart; on by default): a lane whose ray
 * holds a leaf still to test goes on with box tests, and the next leaf it reaches is tested again
 * once the first is done, so leaves are still entered in the reference's order and films are the
 * same bits either way (WVM/include/wf/bvh.hpp:91-116). Closest-hit rays speculate only on a BVH
 * whose boxes nest (wfb_scene_boxes_nested) and whose direction has no zero component. */
int wfb_renderer_set_speculation(wfb_renderer_t r, int on);
int wfb_renderer_width(wfb_renderer_t r);
int wfb_renderer_height(wfb_renderer_t r);
/* ~GpuRenderer. */
int wfb_renderer_destroy(wfb_renderer_t r);

/* ---- autotuner (no reference counterpart) ------------------------------------------------------
 * Measures launch configurations of both arms on `scene` (its camera) at width x height for
 * probe_spp samples: the faster arm (mode), the best megakernel block / occupancy target /
 * min_active / leaf_batch and the best wavefront paths in flight / min_active (0 when the
 * wavefront was not tried). Cached per scene content and size. */
typedef struct {
    int mode;
    int block, occupancy, min_active, leaf_batch;
    int paths_in_flight, wf_min_active;
    double msamples_s, megakernel_msamples_s, wavefront_msamples_s;
    int candidates;
    int wf_occupancy; /* wavefront register cap: 0, 6, 8 or 10 CTAs of 128 threads per SM */
} wfb_tune_result;
int wfb_autotune(wfb_scene_t scene, int width, int height, int probe_spp, int max_depth, int try_wavefront,
                 wfb_tune_result* out);
/* Applies the knobs of a tuning result that belong to the renderer's arm. */
int wfb_renderer_apply_tuning(wfb_renderer_t r, const wfb_tune_result* t);

/* ---- batched rendering (no reference counterpart: one scene/camera/job per GpuRenderer) -------
 * Many jobs of uneven size rendered in ONE persistent launch of either arm: the megakernel
 * (replayed through a CUDA graph captured once per launch shape) or the wavefront (the paths of
 * every job in one pool, each slot carrying its job). Every job's film is bit-identical to the same
 * job rendered alone by wfb_renderer_render. */
typedef struct {
    int mode;            /* WFB_MODE_MEGAKERNEL or WFB_MODE_WAVEFRONT */
    int use_graph;       /* megakernel: replay one captured CUDA graph per launch shape */
    int block;           /* megakernel: 64, 128 or 256 threads; <= 0: 128 */
    int occupancy;       /* register cap for 0, 6, 8 or 10 CTAs per SM: megakernel (block 128) and
                            wavefront (128-thread blocks); < 0: 10 */
    int min_active;      /* 1..32; <= 0: default (megakernel batches and servers 12) */
    int leaf_batch;      /* 1..32; <= 0: default (see wfb_renderer_configure) */
    int paths_in_flight; /* wavefront pool slots; <= 0: 16M */
    int split_chunks;    /* megakernel: work units per pixel of each job; <= 0: automatic (one
                            sample per unit while the job's per-sample buffer fits) */
} wfb_launch_config;
typedef struct wfb_batch* wfb_batch_t;
typedef struct {
    float cam_position[3], cam_look_at[3], cam_up[3];
    float cam_vfov_deg;
    int width, height;
    int spp;
    uint32_t seed;
    int max_depth;
} wfb_job_desc;
/* cfg NULL: megakernel with graph replay and default knobs. */
int wfb_batch_create(int max_jobs, const wfb_launch_config* cfg, wfb_batch_t* out);
int wfb_batch_add(wfb_batch_t b, wfb_scene_t scene, const wfb_job_desc* job, int* job_id);
int wfb_batch_clear(wfb_batch_t b);
/* Zeroes all films, renders every job in one launch, waits; stats may be NULL. */
int wfb_batch_run(wfb_batch_t b, int count_rays, wfb_render_stats* stats);
/* GPU-arm download convention of job `job_id` (rgb 3*w*h, lum_var w*h, either may be NULL). */
int wfb_batch_download(wfb_batch_t b, int job_id, float* rgb, float* lum_var);
int wfb_batch_download_sums(wfb_batch_t b, int job_id, float* rgb_sum, float* lum_sum, float* lum2_sum);
int wfb_batch_destroy(wfb_batch_t b);

/* ---- render server (no reference counterpart) -------------------------------------------------
 * Continuous batching: a worker thread admits queued jobs while their device bytes fit the budget,
 * and every launch advances all admitted jobs by a slice of samples sized to take about
 * launch_target_ms, so requests arriving during a launch join the next one. Latency is measured
 * from wfb_server_submit to the film being ready on the host. one_job_per_launch = 1 gives the
 * sequential baseline (FIFO, one launch per whole job). */
typedef struct wfb_server* wfb_server_t;
typedef struct {
    uint64_t budget_bytes;   /* 0: 40 GiB */
    int max_jobs;            /* per launch; 0: 256 */
    double launch_target_ms; /* 0: 20 */
    int fixed_slice;         /* > 0: samples per job per launch */
    int one_job_per_launch;
    wfb_launch_config launch; /* arm and knobs of every launch (split_chunks <= 0: 4 for servers) */
    int schedule;            /* continuous batching: WFB_SCHEDULE_EXPRESS (0) or WFB_SCHEDULE_SHARED */
} wfb_server_config;
/* Schedules: EXPRESS -- jobs whose remaining work fits a quarter of a launch ride in the next launch
 * whole; large jobs take the rest in arrival order (the oldest always at least a quarter).
 * SHARED -- every admitted job advances by the same number of samples per launch. */
#define WFB_SCHEDULE_EXPRESS 0
#define WFB_SCHEDULE_SHARED 1
typedef struct {
    uint64_t submitted, completed, cancelled, failed, launches, samples_done;
    double busy_ms, wall_s;
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;
    uint64_t bytes_in_use, peak_bytes;
    int queued, active;
} wfb_server_stats;
#define WFB_JOB_QUEUED 0
#define WFB_JOB_ACTIVE 1
#define WFB_JOB_DONE 2
#define WFB_JOB_CANCELLED 3
#define WFB_JOB_FAILED 4
int wfb_server_create(const wfb_server_config* cfg, wfb_server_t* out);
/* Thread-safe. The scene must stay alive until the job is finished. */
int wfb_server_submit(wfb_server_t s, wfb_scene_t scene, const wfb_job_desc* job, uint64_t* ticket);
int wfb_server_poll(wfb_server_t s, uint64_t ticket, int* state);
/* WFB_ERR_TIMEOUT when the job is not finished after timeout_ms (< 0: wait forever). */
int wfb_server_wait(wfb_server_t s, uint64_t ticket, int timeout_ms);
/* Film of a finished job (GPU-arm convention) and its latency; releases the job. */
int wfb_server_result(wfb_server_t s, uint64_t ticket, float* rgb, float* lum_var, double* latency_ms);
/* Drops a queued or running job (running jobs leave at the next launch boundary). */
int wfb_server_cancel(wfb_server_t s, uint64_t ticket);
int wfb_server_stats_get(wfb_server_t s, wfb_server_stats* out);
/* Clears latency samples and counters (keeps jobs in flight). */
int wfb_server_reset_stats(wfb_server_t s);
int wfb_server_destroy(wfb_server_t s);

/* ---- queue primitives (WVM/src/gpu/queues.cuh:30-55) ------------------------------------------
 * Device pointers in, stream-ordered, no host synchronisation. Status 1 (WFB_ERR_INVALID_ARGUMENT,
 * the value of cudaErrorInvalidValue the reference returns) for n > capacity, with nothing enqueued.
 * `stream` is a cudaStream_t (NULL = default stream). */
typedef struct wfb_scan_workspace* wfb_scan_workspace_t;
/* scan_workspace_create (WVM/src/gpu/queues.cu:99-111): look-back status for up to `capacity` items. */
int wfb_scan_workspace_create(int capacity, wfb_scan_workspace_t* out);
/* scan_workspace_destroy (WVM/src/gpu/queues.cu:113-119). */
int wfb_scan_workspace_destroy(wfb_scan_workspace_t ws);
/* scan_exclusive_u32 (WVM/src/gpu/queues.cu:175-196): out[i] = sum(in[0..i-1]), in may equal out,
 * *d_total = sum (d_total may be NULL). Single pass (decoupled look-back). */
int wfb_scan_exclusive_u32(const uint32_t* d_in, uint32_t* d_out, int n, uint32_t* d_total,
                           wfb_scan_workspace_t ws, void* stream);
/* compact_u32 (WVM/src/gpu/queues.cu:214-234): stable; out[k] = values[i] for the k-th i with
 * flags[i] != 0, *d_count = number selected. d_scratch is accepted for signature compatibility and
 * not used (the single-pass kernel needs no indicator array). */
int wfb_compact_u32(const uint32_t* d_values, const uint32_t* d_flags, uint32_t* d_out, uint32_t* d_count,
                    uint32_t* d_scratch, int n, wfb_scan_workspace_t ws, void* stream);
/* test_queue_push (WVM/src/gpu/queues.cu:247-252): lanes i < n with flags[i] != 0 push i through the
 * warp-aggregated queue_push with the given capacity; *d_counter and *d_overflow must be zeroed by
 * the caller. Order inside the queue is unspecified. */
int wfb_test_queue_push(const uint32_t* d_flags, int n, uint32_t* d_items, uint32_t capacity, uint32_t* d_counter,
                        uint32_t* d_overflow, void* stream);
/* Waits for `stream`; WFB_ERR_DEVICE_WAIT if a bounded look-back wait of this workspace gave up
 * (no reference counterpart: the reference's scan has no device-side waits). */
int wfb_scan_workspace_check(wfb_scan_workspace_t ws, void* stream);

/* Test hook for the bounded device-side waits (no reference counterpart: the reference's GPU arms
 * have no device-side waits; its failure suite drives the wavefront's error path through
 * queue_capacity instead, WVM/tests/catch/wavefront_failure.cu:92-114). Sets the limit of every
 * bounded wait -- wavefront grid barriers and scan look-backs -- to limit_ns for later launches
 * (0 restores the 2 s default). With unsatisfiable != 0, the NEXT wavefront launch or scan waits
 * for something that never happens (a barrier expects one CTA more than the launch has; no CTA
 * claims the first scan tile): its waits run out after limit_ns, the kernel returns, and the call
 * reports WFB_ERR_DEVICE_WAIT (renders) or wfb_scan_workspace_check does. Process-wide. */
int wfb_test_bounded_wait(uint64_t limit_ns, int unsatisfiable);
/* Host-side check of the traversal steps (no reference counterpart; needs no GPU): the device's box
 * and primitive steps, compiled for the host, run in simulated 32-lane warps with the megakernel's
 * round choice -- a primitive round once leaf_batch lanes hold a pending leaf, else up to box_steps
 * box steps per lane -- with speculation on or off. rays: n x {o[3], tmin, d[3], tmax} floats (tmin
 * is taken as 1e-4, as every traced ray has it); hits: n x {t, prim (int bits), u, v}. The result
 * equals preorder traversal (WVM/include/wf/bvh.hpp:91-116) whatever the knobs. */
int wfb_test_traverse(wfb_scene_t scene, const void* rays, int n, int anyhit, int speculate, int box_steps,
                      int leaf_batch, void* hits);
/* Host model of a 4-wide traversal over the same tree (no reference counterpart; needs no GPU): the
 * grandchildren of a node are box-tested together against the current tmax and stacked in preorder
 * with that tmax; a node popped after tmax moved is tested again. Rays and hits as in
 * wfb_test_traverse; counts[4]: wide fetches, pops, re-tests, binary box steps of the same rays. */
int wfb_test_traverse_wide(wfb_scene_t scene, const void* rays, int n, int anyhit, void* hits, int64_t* counts);

/* ---- allocation-free rendering ---------------------------------------------------------------
 * No counterpart in the reference. For callers that must not allocate device memory on their
 * render path: a host that owns all device memory through its own pool and does not let plugins
 * allocate, or a real-time loop where an allocation (which can synchronise the device) would
 * break the frame budget.
 *
 * Adds samples [first_sample, first_sample + count) of `scene` -- its own camera and resolution
 * w x h -- to caller-owned DEVICE film sums (rgb_sum 3*w*h floats, lum_sum w*h, lum2_sum w*h),
 * exactly as wfb_renderer_run_passes adds them to a renderer's film (same bits). Enqueued on
 * `stream` (a cudaStream_t; NULL = default stream); the call returns without waiting. The scene
 * may be destroyed as soon as the call returns: its device memory is released only after the
 * queued work.
 * Allocates nothing: its scratch is one static device array of about 12 MB that every GPU which
 * loads the library holds until the process exits, and that all calls share. Calls that overlap
 * on the GPU therefore race: serialise them (one stream, or wait between calls). The first call
 * on a device (and the first after that device's context was reset) looks up the array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture. The scene must already
 * be resident on the current device (creating a renderer on it uploads it). Rejects
 * w * h * count > WFB_NOALLOC_MAX_SAMPLES with WFB_ERR_INVALID_ARGUMENT; render larger requests
 * in passes of fewer samples. */
#define WFB_NOALLOC_MAX_SAMPLES 1048576
int wfb_render_passes_noalloc(wfb_scene_t scene, int first_sample, int count, uint32_t seed, int max_depth,
                              float* rgb_sum, float* lum_sum, float* lum2_sum, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WFB200_H */
