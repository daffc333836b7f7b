// Host-side preparation shared by the C ABI (cr_host.cpp) and the device driver
// (cr_render.cu). Everything here runs on the CPU once per scene or per render.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <functional>
#include <utility>
#include <vector>
#include "cr_gpu.h"
#include "cr_internal.h"

namespace crh {

// Typed failures carry the cr_status they map to, and the reference's message text.
struct Error : std::runtime_error {
    cr_status status;
    Error(cr_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

cr_status set_last_error(cr_status status, const std::string& message);
const std::string& last_error_text();  // this thread's last message

// Memory blocks the library has requested (device and page-locked host): every allocation
// site calls count_allocation(); cr_gpu_allocation_count reports the total.
void count_allocation();
uint64_t allocation_count();
// Fault injection for tests: the nth device allocation from now (0: the next) made through
// crd::DevAlloc fails as if the device were out of memory; a negative nth disarms it.
void inject_allocation_failure(int64_t nth);
bool injected_allocation_failure();  // consumes one allocation of the countdown

void validate_options(const cr_render_options& o);                           // render.cpp:97-104

// Scene::finalize (geometry.cpp:296-397) on a triangle vector.
void finalize(std::vector<cr_triangle>& triangles, const cr_material* materials, uint32_t materialCount,
              const cr_image* images, uint32_t imageCount, const cr_texture* textures, uint32_t textureCount,
              std::vector<std::string>& warnings);

// Bvh::build (geometry.cpp:463-550).
void build_bvh(const cr_triangle* triangles, uint64_t count, std::vector<cr_bvh_node>& nodes,
               std::vector<uint32_t>& indices);

// Environment tables (render.cpp:12-42, 67-94).
struct EnvTables {
    bool hasImage = false;
    float constant[3] = {0, 0, 0};
    int width = 0, height = 0;
    float rotation = 0, intensity = 1;
    double integral = 0, weightSum = 0;
    std::vector<double> cdf;
    std::vector<float> pdf;       // per texel density
    std::vector<float> rowCos;    // cos(pi*y/H) for y = 0..H
    std::vector<uint32_t> coarse; // bracket table for the CDF search
    // alias-table sampling (built on demand): per column the threshold on the 48-bit residual
    // below which the column's own texel is taken, its alias, and every texel's density under
    // this sampler (its realised probability, exact, over the texel's solid angle)
    std::vector<uint64_t> aliasThreshold;
    std::vector<uint32_t> aliasIndex;
    std::vector<float> aliasPdf;
};
void build_environment(const cr_environment_desc& e, EnvTables& out, bool alias = false);
// Walker/Vose alias table over the same texel probabilities (built on demand).
void build_alias(EnvTables& t);
// The alias sampler's realised probability of every texel, in units of 2^-48 (for checks).
std::vector<uint64_t> alias_masses(const EnvTables& t);

// Runs fn(begin, end) over [0, n) split across the host's hardware threads.
void parallel_for(uint64_t n, const std::function<void(uint64_t, uint64_t)>& fn, uint64_t grain = 65536);

// Lights (render.cpp:131-160).
struct LightTables {
    std::vector<crg::LightEntry> entries;
    std::vector<float> triangleProbability;
    float environmentProbability = 0;
};
// The triangle half of the light table (the scene's bounding radius and the emitters' weights,
// per part in triangle order), which needs no environment: a scene upload computes it while
// the environment tables are still being built.
struct LightScan {
    uint64_t count = 0;
    double radius2 = 1;
    std::vector<std::vector<std::pair<uint32_t, double>>> emitters;
};
LightScan scan_lights(const cr_triangle* triangles, uint64_t count, const cr_material* materials);
void build_lights(const LightScan& scan, const cr_punctual_light* lights, uint32_t lightCount, double envIntegral,
                  LightTables& out);
void build_lights(const cr_triangle* triangles, uint64_t count, const cr_material* materials,
                  const cr_punctual_light* lights, uint32_t lightCount, double envIntegral, LightTables& out);

// Camera::generate's per-render part (geometry.cpp:214-224). Throws Error with the
// reference's invalid_argument text when the camera cannot produce rays.
void camera_setup(const cr_camera& c, int width, int height, crg::DevCamera& out);

// Per-sample failure text, "Pixel (x,y), sample s: <cause>" (render.cpp:437-438).
std::string sample_error_message(const crg::DevError& e);

// ---- output encoding (src/io/image.cpp, src/io/file.h) -----------------------------------------
// detail::imagePixels (file.h:84-89): positive, <= 16384 per axis, <= 16777216 pixels.
void check_image_dims(int width, int height, const std::string& label);
// The display mapping of io::writePng (image.cpp:116-124, 193-201) is a non-decreasing step
// function of the linear value at a fixed exposure, so it is fully described by the least
// value reaching each output byte: out[k] (k = 1..255) is the smallest non-negative float v
// with displayChannel(v) >= k (+inf when none), out[0] = 0. Throws the reference's error for
// an exposure outside [-100, 100] stops.
void display_thresholds(float exposure, float out[256]);
// The reference's display mapping itself, for checks of the table.
unsigned char display_channel(float value, double exposure_scale);
// The text stb_image_write 1.16 (the codec io::writeHdr uses) writes before the scanlines.
std::string hdr_header(int width, int height);

}  // namespace crh
