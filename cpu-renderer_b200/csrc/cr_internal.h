// Internal layouts shared by the host driver (cr_host.cpp) and the kernels (cr_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "cr_gpu.h"

namespace crg {

// Two sibling BVH nodes in one 64-byte record, read as four 128-bit loads. The
// reference allocates children adjacently (geometry.cpp:544-547), so the pair
// (first, first+1) of every interior node is stored together; pair p holds nodes
// 2p+1 and 2p+2. For each child, d.{x,z} is a leaf's first index-slot (count > 0) or
// the pair index of its own children (count == 0); d.{y,w} is the count.
struct __align__(64) NodePair {
    float4 a;  // c0.lo.x c0.lo.y c0.lo.z c0.hi.x
    float4 b;  // c0.hi.y c0.hi.z c1.lo.x c1.lo.y
    float4 c;  // c1.lo.z c1.hi.x c1.hi.y c1.hi.z
    uint4 d;   // c0.ref c0.count c1.ref c1.count
};

// Light-selection CDF entry (render.cpp:122).
struct LightEntry {
    double cdf;
    uint32_t type;   // 0 punctual, 1 triangle, 2 environment
    uint32_t index;
    float probability;
    uint32_t pad;
};
enum : uint32_t { kLightPunctual = 0, kLightTriangle = 1, kLightEnvironment = 2 };

// Triangle flags in tri_pos[3*slot+1].w and tri_ng[triangle].w. kTriNeeNull marks materials
// whose BSDF value is zero for every direction (smooth, and metallic 1 or transmission 1, no
// texture that could change that): their next-event estimation only consumes random draws.
// kTriConductor marks rough GGX conductors (metallic exactly 1, transmission exactly 0, no
// texture that could change either), which the conductor shading kernel takes.
enum : uint32_t { kTriCull = 1u, kTriAlphaMask = 2u, kTriNeeNull = 4u, kTriConductor = 8u };

// Shading classes, one queue each, filled by the traversal kernel.
enum : int { kShadeMiss = 0, kShadeNeeNull = 1, kShadeGeneric = 2, kShadeConductor = 3, kShadeClasses = 4 };

struct DevImage { int32_t width, height; const float4* pixels; };

// Punctual light with its cone cosines evaluated on the host (render.cpp:203, std::cos).
struct DevPunctual {
    int32_t type;
    float position[3], direction[3], color[3];
    float intensity, range, cos_outer, cos_inner;
};

// Everything the kernels read, by value in the kernel parameters.
struct DevScene {
    // geometry
    const float4* tri_pos;        // [3*slot+k] leaf order; [0].w = triangle index bits, [1].w = flags
    const float4* tri_ng;         // [triangle] geometric normal (cull test), w = flags bits
    const cr_triangle* tris;      // [triangle] full finalized data
    const NodePair* pairs;
    uint64_t triangle_count;
    uint32_t has_root;
    float root_lo[3], root_hi[3];
    uint32_t root_ref, root_count;
    // materials and textures
    const cr_material* materials;
    uint32_t material_count;
    const double2* slot_trig;     // [5*material + slot] cos, sin of the slot rotation (double)
    const DevImage* images;
    const cr_texture* textures;
    uint32_t image_count, texture_count;
    uint32_t any_alpha_mask;
    uint32_t nee_skip;            // kTriNeeNull surfaces may skip the light-sample arithmetic
    uint32_t conductor_class;     // kTriConductor surfaces go to the conductor shading kernel
                                  // (set per render by the launchers that run that kernel)
    // lights (render.cpp:120-229)
    const LightEntry* light_entries;
    uint32_t light_entry_count;
    const float* tri_light_probability;   // [triangle]
    float env_probability;
    const DevPunctual* punctual;
    uint32_t punctual_count;
    // environment (render.h:8-28, render.cpp:10-94)
    uint32_t env_has_image;
    float env_constant[3];
    int32_t env_width, env_height;
    const float4* env_pixels;
    const double* env_cdf;        // [w*h]
    const float* env_pdf;         // [w*h] density of each texel, as Environment::pdf computes it
    const float* env_row_cos;     // [h+1] cos(pi*row/h) in float, as Environment::sample computes it
    const uint32_t* env_coarse;   // upper_bound bracket table over env_cdf
    uint32_t env_coarse_count;    // entries in env_coarse (a power of two)
    double env_weight_sum;
    float env_rotation, env_intensity;
    // alias-table sampling (optional; a render that asks for it also points env_pdf at the
    // alias sampler's own texel densities)
    const unsigned long long* alias_threshold;  // [column] 48-bit residual threshold
    const uint32_t* alias_index;                // [column] alias texel
};

// Per-render constants (camera basis from Camera::generate, geometry.cpp:219-224).
struct DevCamera {
    float position[3];
    float f[3], r[3], u[3];
    double ratio, halfHeight;
    float nearClip, farClip;
};

struct RenderParams {
    int32_t width, height, samples, bounces;
    uint64_t seed;
    int32_t nee, rr;
    int32_t env_alias;
    int32_t exact_traversal;
    DevCamera camera;
};

// Guided renders only (all null otherwise): the per-path guiding state of cr_guide.cuh.
struct GuidePathRefs {
    const float* mixture = nullptr;          // [path][40] network outputs for the path's current vertex
    float* hitT = nullptr;                   // [path] closest-hit distance
    void* records = nullptr;                 // GuideRecord [path][kGuideRecords]
    uint32_t* count = nullptr;               // [path] records in use
    void* samples = nullptr;                 // GuideSample [sampleCapacity]: training samples collected
    unsigned long long* sampleCount = nullptr;
    uint64_t sampleCapacity = 0;
    float lo[3] = {0, 0, 0}, inv[3] = {0, 0, 0};  // position features = (p - lo) * inv
    float guideProbability = 0;              // one-sample MIS: share of directions from the network
    int32_t record = 0;                      // collect training samples
};

// Diagnostic record of every traced ray (cr_gpu_render_trace_dump); null otherwise. Only the
// counting traversal kernels write it.
struct TraceDump {
    cr_traced_ray* rays = nullptr;
    unsigned long long* count = nullptr;
    uint64_t capacity = 0;
};

// Path state, structure of arrays over path slots.
struct PathSoA {
    float4* ray_o;        // origin, tmin
    float4* ray_d;        // direction, tmax
    float4* ray_lo;       // originLow (precise replay only)
    uint32_t* hit_tri;    // closest-hit output (kNoTriangle = miss)
    float4* thr;          // throughput, etaScale
    float4* rad;          // radiance, lastPdf
    float4* last_pos;     // lastPosition
    uint32_t* flags;      // kPath* bits
    float4* absorb;       // absorption, medium (int bits)
    uint64_t* rng;
    uint32_t* prev_tri;
    uint32_t* pixel;
    uint32_t* sample;
    uint32_t* depth;
    // shadow rays
    float4* sh_o;         // origin, tmin(0)
    float4* sh_d;         // direction, tmax
    float4* sh_lo;        // originLow
    float4* sh_c;         // contribution, ignore-triangle bits
    // per-sample radiance of the current chunk, indexed by sample id - chunk start
    float4* out;
    GuidePathRefs guide;  // zero unless the render is guided
    TraceDump dump;       // zero unless the render records its rays
};
// bits of PathSoA::flags
// kPathNull (alone): a multi-job pool slot whose camera sample failed; it only returns to the ring.
enum : uint32_t { kPathLastDelta = 1u, kPathPrecise = 2u, kPathDead = 4u, kPathShadow = 8u, kPathNull = 16u };

// Index queues of the path pool, each a ping-pong pair indexed by iteration parity.
struct Queues {
    uint32_t* extend[2];  // live paths awaiting a closest hit
    uint32_t* shadow[2];  // paths with a queued shadow ray
    uint32_t* free[2];    // finished slots awaiting a new camera sample
    uint32_t* shade[kShadeClasses];  // traced paths by shading class
    uint32_t* counts;     // kCount* words
};
// kCountTraceWork0/1: queue entries k_trace has handed out (indexed by iteration parity);
// kCountShadeWork0 + class: the same for each k_shade instantiation.
enum { kCountExtend0 = 0, kCountExtend1 = 1, kCountShadow0 = 2, kCountShadow1 = 3, kCountFree0 = 4, kCountFree1 = 5,
       kCountShade0 = 6, kCountTraceWork0 = kCountShade0 + kShadeClasses, kCountShadeWork0 = kCountTraceWork0 + 2,
       kCountWords = kCountShadeWork0 + kShadeClasses };
static_assert(kCountWords == 16, "queue counter words");

// Device error record; the host reports the one with the smallest key, which is the
// order a single reference worker would meet them (tiles, rows, columns, samples).
struct DevError {
    uint64_t key;
    int32_t code;         // ErrorCode
    int32_t x, y, sample;
    int32_t depth;
    uint32_t triangle, material;
    double t;
    float point[3], origin[3], direction[3];
};
enum ErrorCode : int32_t {
    kErrNone = 0,
    kErrNonFiniteThroughput = 1,
    kErrNonFiniteRadiance = 2,
    kErrNestedVolume = 3,
    kErrExitWithoutEntry = 4,
    kErrInvalidSecondaryRay = 5,
    kErrOffsetOverflow = 6,
    kErrUnrepresentableCameraRay = 7,
    kErrStackOverflow = 8,
    kErrInvalidSurfaceHit = 9,
    kErrTextureCoordinates = 10,
};
constexpr int kMaxErrors = 64;

constexpr int kStackSize = 64;

}  // namespace crg
