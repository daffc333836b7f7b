// Helper of the C++ drop-in (render_gpu.cpp) for other host programs linked with it.
#pragma once
#include "cr_gpu.h"
#include "render.h"

namespace cr {
// Uploads a finalized scene, the caller's own BVH node array and the environment to `device`
// (cr_gpu_scene_create); throws std::runtime_error (std::bad_alloc when out of memory).
cr_gpu_scene* uploadToGpu(const Scene& scene, const Bvh& bvh, const Environment& environment, int device);
}  // namespace cr
