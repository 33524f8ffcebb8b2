// Procedural benchmark scenes (see scene_gen.cpp for their definitions).
#pragma once
#include <cstdint>
#include <string>
#include "wf/scene.hpp"

namespace wfb {

// Builds and finalizes "cornell36", "icospheres" or "heightfield" at the given resolution.
// Throws std::invalid_argument for an unknown name or a non-positive resolution.
wf::Scene make_config_scene(const std::string& name, int width, int height, uint32_t seed,
                            int sah_bins);

// Camera on the orbit of the scene's default camera around its look-at point.
wf::Camera orbit_camera(const wf::Scene& scene, float azimuth_deg, float elevation_deg);

}  // namespace wfb
