// Engine internals shared by the kernels' host launchers, the renderer and the C ABI.
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "dev_scene.cuh"
#include "wf/renderer.hpp"
#include "wf/scene.hpp"

namespace wfb {

// Error carrying one of the C ABI status codes (include/wfb200.h).
struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

void cuda_check(cudaError_t e, const char* what);  // throws Error(WFB_ERR_CUDA or OOM)

// Bounded device-side waits (wavefront grid barriers, scan look-backs): a wait longer than
// device_wait_limit_ns() gives up and the call reports WFB_ERR_DEVICE_WAIT (queues.cu).
uint64_t device_wait_limit_ns();
// Test hook: sets the limit (0: the 2 s default) and, with unsatisfiable_next, makes the next
// wavefront launch or scan wait for something that never happens (a CTA the launch does not have,
// a tile no CTA claims), so that its wait runs out.
void set_device_wait_test(uint64_t limit_ns, bool unsatisfiable_next);
// Consumes the pending unsatisfiable-wait request, if any.
bool take_unsatisfiable_wait();

// Scene uploaded once in the packed device layout; shared (reference-counted) by every renderer
// and batch job that draws it, so a BVH stays resident across renders.
struct ResidentScene {
    DevScene dev{};  // device pointers into `arena`; camera/resolution are the host defaults
    void* arena = nullptr;
    uint64_t bytes = 0;
    uint64_t content_key = 0;   // hash of the packed arena, environment and default camera
    int device = -1;
    // Recorded after work that reads the arena on a caller's stream and returns without waiting
    // (the allocation-free entry); the arena's release waits for it.
    cudaEvent_t last_use = nullptr;
    ~ResidentScene();
};

// Validates and repacks a finalized scene into the device layout (see dev_scene.cuh).
std::shared_ptr<ResidentScene> upload_scene(const wf::Scene& host);

// Folds `bytes` of `data` into the key `h` (multiply-xorshift over 8-byte words).
uint64_t mix_key(uint64_t h, const void* data, size_t bytes);

// 1 when speculative closest-hit traversal is exact on this BVH (nested boxes; device_scene.cu).
int check_boxes_nested(const std::vector<wf::BvhNode>& nodes);
// Packed records (dev_scene.cuh layout) of node i (2 float4) and prim_order entry j (3 float4);
// throw on what the traversal cannot use.
void pack_node(const wf::Scene& host, int i, float4* out);
void pack_prim(const wf::Scene& host, int j, float4* out);
// Wide records for a 4-wide traversal of the same tree: one per internal node, 8 float4 (128 B):
// slot k = {lo, node id} {hi, code} for up to 4 candidates -- the node's grandchildren in preorder,
// a leaf child standing for itself -- code = the candidate's leaf encoding (>= 0) or ~(its wide
// record index) (< 0); an empty slot has node id -1. `code_of` gets each node's code. Returns false
// (and leaves the outputs empty) when some internal node has more than 4 candidates.
bool pack_wide(const wf::Scene& host, std::vector<float4>* records, std::vector<int>* code_of);
// Host run of the traversal steps in simulated 32-lane warps with the megakernel's round policy
// (trav_check.cu): rays are {o, tmin, d, tmax} (tmin taken as kRayEps), hits {t, prim, u, v}.
void traverse_check(const wf::Scene& host, const float* rays, int n, bool anyhit, bool speculate, int box_steps,
                    int leaf_batch, float* hits);
// Host model of a 4-wide traversal with re-tested speculation over the same tree (trav_check.cu);
// counts[4]: wide fetches, pops, re-tests after a tmax change, binary box steps of the same rays.
void traverse_wide_check(const wf::Scene& host, const float* rays, int n, bool anyhit, float* hits,
                         long long* counts);

// Film download in the GPU-arm convention (mean rgb, luminance variance), resolved on the device;
// shared by renderers, batches and the server. Ordered after the work already queued on `stream`
// (null: the calling thread's own stream, for a film whose writers have finished); returns once
// the host buffers hold the result. rgb or lum_var may be null.
void film_download(const DevFilm& film, int spp_done, float* rgb, float* lum_var, cudaStream_t stream);
// The same result converted on the host: only copy engines work on the device, so it never waits
// for SMs held by a persistent kernel of another stream (the server's download thread uses it).
// Reusable pinned host memory for film_download_host (owned and freed by its caller).
struct PinnedStaging {
    void* ptr = nullptr;
    size_t bytes = 0;
};
void film_download_host(const DevFilm& film, int spp_done, float* rgb, float* lum_var, cudaStream_t stream,
                        PinnedStaging* staging = nullptr);

// Same scene view with another camera / resolution (batch jobs and orbit cameras).
DevScene with_camera(const DevScene& s, const wf::Camera& cam, int width, int height);

// Per-call render controls (mirror of wf::RenderParams without the CPU-only fields).
struct PassParams {
    int first_sample = 0;
    int sample_count = 0;
    uint32_t seed = 1234;
    int max_depth = 8;
    bool count_rays = false;
    bool stage_timing = false;
    int queue_capacity = 0;
};

// ---- megakernel (megakernel.cu) ----
struct MegakernelConfig {
    int block = 128;        // threads per CTA (64, 128 or 256)
    int blocks_per_sm = 0;  // 0: as many as fit
    int min_active = 16;    // traverse on while at least this many lanes of a warp traverse
    int split_chunks = 0;   // work units per pixel; 0: one sample per unit while its buffer fits
    int occupancy = 10;     // block 128 only: 6, 8 or 10 caps registers for that many CTAs per SM (0: none)
    int leaf_batch = 12;    // a warp tests primitives once this many lanes hold a pending leaf
    bool speculate = true;  // lanes holding a pending leaf go on with box steps (box_step)
};
// Split mode keeps each path's radiance (3 floats) per (pixel, sample) until the ordered commit;
// automatic splitting keeps that buffer under kSplitBufferBytes (renders above it run in sub-passes).
constexpr uint64_t kSplitBufferBytes = 2ull << 30;
inline uint64_t split_buffer_bytes(long long pixels, long long samples) {
    return 3ull * sizeof(float) * (uint64_t)pixels * (uint64_t)samples;
}
// Resident threads of the persistent megakernel for this configuration.
int megakernel_resident_threads(const MegakernelConfig& cfg);
// Work units per pixel (1 = direct film accumulation; > 1 needs a per-sample buffer).
int megakernel_split_chunks(int pixels, int sample_count, const MegakernelConfig& cfg);

// CUDA-event timing of a render's main kernel launches (the persistent megakernel or wavefront
// kernel alone: no memsets, pool init, counter folds or film commits), summed over the launches of
// one render. Events are created on first use and reused.
class KernelTimer {
public:
    KernelTimer() = default;
    KernelTimer(const KernelTimer&) = delete;
    KernelTimer& operator=(const KernelTimer&) = delete;
    ~KernelTimer();
    void reset() { used_ = 0; }
    void begin(cudaStream_t stream);  // records before a main launch
    void end(cudaStream_t stream);    // records after it
    double total_ms() const;          // once the stream has passed the last end()
private:
    std::vector<cudaEvent_t> ev_;
    int used_ = 0;
};
// Adds samples [first, first + count) of every pixel to `film`. With chunks > 1, `lbuf` must hold
// 3 * pixels * count floats (per-sample radiance, committed in sample order after the kernel).
// Returns the number of kernels launched.
int launch_megakernel(const DevScene& s, const DevFilm& film, DevCounters* counters,
                       unsigned int* work_counter, float* lbuf, const PassParams& p,
                      const MegakernelConfig& cfg, int chunks, cudaStream_t stream, KernelTimer* timer = nullptr);

// Adds per-(pixel, sample) radiance slots (3 floats, sample-major: sample_slot) to the
// film sums in ascending sample order (megakernel.cu).
void launch_film_commit(const DevFilm& film, const float* lbuf, int count, cudaStream_t stream);

// One render job inside a launch: scene + camera (in `s`), film, sample range, split mode.
// Its work units are [unit_begin, unit_begin + units) of the launch; unit u covers pixel
// (u - unit_begin) mod pixels and chunk (u - unit_begin) div pixels of `chunk` samples.
struct JobDesc {
    DevScene s;
    DevFilm film;
    float* lbuf;  // chunks > 1: 3 floats per (pixel, sample - first_sample)
    int first_sample, sample_count, chunk, chunks;
    uint32_t seed;
    int max_depth;
    unsigned unit_begin, units;
};

// Device-resident size of a batch launch, so a captured graph can be replayed for any batch.
struct BatchHeader {
    unsigned n_jobs;
    unsigned total_units;
    unsigned pad[62];
};

JobDesc make_job(const DevScene& s, const DevFilm& film, float* lbuf, int first_sample, int sample_count,
                 int chunks, uint32_t seed, int max_depth);

#if defined(__CUDACC__)
// Job owning work unit `u` of a batch: the last job whose first unit is <= u (unit_begin ascends).
__device__ __forceinline__ int job_of_unit(const JobDesc* jobs, int n_jobs, unsigned u) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].unit_begin <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
#endif

// Split-mode commits of every job of a batch (jobs with chunks > 1), in sample order.
void launch_film_commit_jobs(const JobDesc* d_jobs, const BatchHeader* d_hdr, int max_jobs, cudaStream_t stream);
// Persistent megakernel over a device job table (unit_begin must be the running sum of units)
// followed by the split-mode commits of its jobs; max_jobs bounds the job count of any batch
// replayed through the same launch; all_split: every job has chunks > 1 (the leaner kernel variant).
// Stream-ordered, no host synchronisation, capturable.
void launch_megakernel_batch(const JobDesc* d_jobs, const BatchHeader* d_hdr, int max_jobs, DevCounters* counters,
                             unsigned int* work_counter, bool count_rays, const MegakernelConfig& cfg,
                             bool all_split, cudaStream_t stream);

// ---- wavefront (wavefront.cu) ----
struct WavefrontConfig {
    int paths_in_flight = 0;  // path-pool slots; 0: 16M (capped at 64 x pixels)
    int l2_persist = -1;      // pool under a persisting L2 window: -1 when it fits the set-aside, 0 never, 1 always
    int occupancy = 10;       // register cap for 6, 8 or 10 CTAs of 128 threads per SM (0: none)
    bool suspend_stragglers = true;  // carry the last extension rays of a bounce over to the next
    int min_active = 24;      // traverse on while at least this many lanes of a warp traverse
    int leaf_batch = 8;       // a warp tests primitives once this many lanes hold a pending leaf
    bool speculate = true;    // lanes holding a pending leaf go on with box steps (box_step)
};

// Launch configuration of a batch or a server: the arm and its knobs.
struct LaunchConfig {
    wf::GpuMode mode = wf::GpuMode::Megakernel;
    // Batch launches (many jobs of several scenes, shading state parked like a single render's)
    // traverse best with a lower min_active than one render of one scene: on the 64-job mix on a
    // B200, 10 CTAs per SM and min_active 12 took 1,168 ms against 1,206 at 8 CTAs and 16.
    MegakernelConfig mk = [] {
        MegakernelConfig c;
        c.min_active = 12;
        return c;
    }();
    WavefrontConfig wf{};
    bool use_graph = true;  // megakernel: replay one captured graph per launch shape
};

// ---- GPU renderer (renderer.cu): one scene, one camera, one film ----
class Renderer {
public:
    Renderer(std::shared_ptr<ResidentScene> scene, wf::GpuMode mode);
    ~Renderer();
    Renderer(const Renderer&) = delete;
    Renderer& operator=(const Renderer&) = delete;

    void set_camera(const wf::Camera& cam, int width, int height);
    void reset();
    void run_passes(const PassParams& p, wf::RenderStats* stats);
    // Traversal counts of the last run_passes with count_rays (megakernel only).
    uint64_t last_node_visits() const { return last_node_visits_; }
    uint64_t last_prim_tests() const { return last_prim_tests_; }
    // Kernels of this library launched by the last run_passes.
    int last_kernel_launches() const { return last_launches_; }
    double last_kernel_ms() const { return last_kernel_ms_; }  // main kernel launches of the last pass
    // Reference download convention (WVM/src/gpu/gpu_renderer.cu:306-341).
    void download(int spp_done, float* rgb, float* lum_var);
    void download_mean(int spp_done, float* rgb);
    void download_sums(float* rgb_sum, float* lum_sum, float* lum2_sum);
    uint64_t device_bytes() const;
    int width() const { return width_; }
    int height() const { return height_; }
    int pixels() const { return width_ * height_; }
    wf::GpuMode mode() const { return mode_; }
    void set_megakernel_config(const MegakernelConfig& c) { mk_cfg_ = c; }
    const MegakernelConfig& megakernel_config() const { return mk_cfg_; }
    // Values < 0 keep the current setting (block and min_active also keep on 0).
    void configure(int block, int blocks_per_sm, int min_active, int split_chunks, int paths_in_flight,
                   int occupancy, int leaf_batch = -1);
    // Wavefront pool under a persisting L2 window: -1 when it fits the set-aside, 0 never, 1 always.
    void set_l2_residency(int mode);
    // Bytes of the wavefront pool under the window (0: none, or a megakernel renderer).
    uint64_t l2_window_bytes() const;
    // Speculative traversal in both arms (box_step): films are the same bits either way.
    void set_speculation(bool on);

private:
    void alloc_film();
    void free_film();
    std::shared_ptr<ResidentScene> scene_;
    DevScene view_{};
    wf::GpuMode mode_;
    int width_ = 0, height_ = 0;
    DevFilm film_{};
    DevCounters* counters_ = nullptr;
    unsigned int* work_ = nullptr;
    float* lbuf_ = nullptr;  // split-mode per-sample radiance
    size_t lbuf_floats_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    MegakernelConfig mk_cfg_{};
    WavefrontConfig wf_cfg_{};
    uint64_t last_node_visits_ = 0, last_prim_tests_ = 0;
    int last_launches_ = 0;
    double last_kernel_ms_ = 0.0;
    KernelTimer ktimer_;
    struct Wavefront;
    std::unique_ptr<Wavefront> wf_;
};

}  // namespace wfb
