// Persistent-threads wavefront engine (implementation in progress).
#include "wavefront.hpp"
#include "../../include/wfb200.h"

namespace wfb {

WavefrontEngine::WavefrontEngine(int pixels, const WavefrontConfig& cfg) : pixels_(pixels), cfg_(cfg) {
    throw Error(WFB_ERR_UNSUPPORTED, "wavefront mode is not built yet");
}

WavefrontEngine::~WavefrontEngine() {
    if (arena_) cudaFree(arena_);
}

void WavefrontEngine::run(const DevScene&, const DevFilm&, DevCounters*, const PassParams&, wf::StageTimes*,
                          cudaStream_t) {
    throw Error(WFB_ERR_UNSUPPORTED, "wavefront mode is not built yet");
}

}  // namespace wfb
