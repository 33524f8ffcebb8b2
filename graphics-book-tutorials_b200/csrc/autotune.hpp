// Per-scene autotuner (autotune.cpp).
#pragma once
#include <memory>
#include "engine.hpp"

namespace wfb {

struct TuneResult {
    int mode = 0;  // the faster arm: WFB_MODE_MEGAKERNEL or WFB_MODE_WAVEFRONT
    // Best megakernel knobs.
    int block = 128, occupancy = 0, min_active = 16, leaf_batch = 8;
    // Best wavefront knobs (0: not tried, library defaults).
    int paths_in_flight = 0, wf_min_active = 0, wf_occupancy = -1;
    double msamples_s = 0.0;             // the winner's measured rate
    double megakernel_msamples_s = 0.0;  // best megakernel candidate
    double wavefront_msamples_s = 0.0;   // best wavefront candidate (0 if not tried)
    int candidates = 0;
};

// Measures candidate configurations of both arms on the scene with camera `cam` at width x height
// for probe_spp samples and returns the fastest (cached per scene content and size).
TuneResult autotune(const std::shared_ptr<ResidentScene>& scene, const wf::Camera& cam, int width, int height,
                    int probe_spp, int max_depth, bool try_wavefront);
// Applies the knobs of `t` that belong to the renderer's arm (whichever arm won).
void apply_tuning(Renderer& r, const TuneResult& t);

}  // namespace wfb
