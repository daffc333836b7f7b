/*
 * cr_gpu.h — C ABI of the B200 path-tracing backend.
 *
 * This is the drop-in boundary for CPU-Renderer's per-path radiance loop. It replaces,
 * behind a plain C interface (no C++ or torch types), these reference entry points:
 *
 *   cr::render(scene, bvh, camera, environment, options, progress)   src/render.h:53
 *   cr::Bvh::intersect(scene, ray, hit, any, ignoreTriangle)          src/scene.h:126-127
 *   cr::RenderOptions::validate()                                     src/render.h:38, render.cpp:97-104
 *   cr::Bvh::build(scene)  (host restatement, same node array)        src/scene.h:123, geometry.cpp:463-550
 *   cr::Scene::finalize()  (host restatement)                         src/scene.h:232, geometry.cpp:296-397
 *   cr::Camera::generate(...)                                         src/scene.h:206, geometry.cpp:213-234
 *
 * All structs below are plain data. The first five mirror the reference's value types
 * field for field, so a C++ caller holding cr::Triangle / cr::Ray / cr::Hit arrays can
 * pass them without conversion (the C++ drop-in shim static_asserts the layouts).
 *
 * Ownership: the library never retains a caller pointer past the call that received it.
 * A cr_gpu_scene owns device copies of everything it needs.
 *
 * Errors: every entry point returns a cr_status. The text of the most recent failure on
 * the calling thread is available from cr_gpu_last_error(); for a failed sample it has
 * the reference's form "Pixel (x,y), sample s: <cause>" (render.cpp:437-438).
 */
#ifndef CR_GPU_H
#define CR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CR_GPU_ABI_VERSION 1

typedef enum cr_status {
    CR_OK = 0,
    CR_ERR_INVALID_ARGUMENT = 1, /* bad options/scene/camera: std::runtime_error / invalid_argument */
    CR_ERR_RENDER = 2,           /* a camera sample failed; message carries pixel and sample   */
    CR_ERR_OUT_OF_RANGE = 3,     /* index outside its table (std::out_of_range)               */
    CR_ERR_LENGTH = 4,           /* too many triangles for 32-bit node indices (length_error) */
    CR_ERR_LOGIC = 5,            /* traversal stack exhausted (std::logic_error)              */
    CR_ERR_OUT_OF_MEMORY = 6,    /* device or host allocation failed                          */
    CR_ERR_DEVICE_TIMEOUT = 7,   /* a bounded device loop gave up                              */
    CR_ERR_CUDA = 8,             /* CUDA runtime failure                                      */
    CR_ERR_UNSUPPORTED = 9       /* input uses a feature this build does not implement        */
} cr_status;

/* cr::Vertex (scene.h:155): position, normal, tangent (w = handedness), two UV sets. 56 bytes. */
typedef struct cr_vertex {
    float position[3];
    float normal[3];
    float tangent[4];
    float uv[2][2];
} cr_vertex;

/* cr::Triangle (scene.h:158-163) after Scene::finalize(): world-space vertices, material
 * index, outward geometric normal and area. 188 bytes. */
typedef struct cr_triangle {
    cr_vertex v[3];
    uint32_t material;
    float geometric_normal[3];
    float area;
} cr_triangle;

/* cr::Ray (scene.h:139-143): origin + origin_low + t*direction on [tmin, tmax]. 44 bytes. */
typedef struct cr_ray {
    float origin[3];
    float direction[3];
    float tmin, tmax;
    float origin_low[3];
} cr_ray;

/* cr::Hit (scene.h:166): double t, u, v and the triangle index. 32 bytes. */
typedef struct cr_hit {
    double t, u, v;
    uint32_t triangle;
    uint32_t reserved_;
} cr_hit;

/* Bvh::Node (scene.h:261): bounds, then first/count; count > 0 is a leaf over
 * indices[first, first+count), count == 0 an interior node whose children are the two
 * adjacent nodes first and first+1. 32 bytes. */
typedef struct cr_bvh_node {
    float lo[3];
    float hi[3];
    uint32_t first;
    uint32_t count;
} cr_bvh_node;

/* cr::TextureSlot (scene.h:179-182). texture == -1 means "no map". */
typedef struct cr_texture_slot {
    int32_t texture;
    int32_t texcoord;
    float offset[2];
    float scale[2];
    float rotation;
} cr_texture_slot;

enum { CR_WRAP_REPEAT = 0, CR_WRAP_CLAMP = 1, CR_WRAP_MIRROR = 2 };
enum { CR_ALPHA_OPAQUE = 0, CR_ALPHA_MASK = 1 };

/* cr::Material (scene.h:187-199) without its name. */
typedef struct cr_material {
    float base_color[4];
    float metallic, roughness;
    float emission[3];
    float transmission, ior;
    float thickness, attenuation_distance;
    float attenuation_color[3];
    int32_t double_sided;
    int32_t alpha_mode;
    float alpha_cutoff, normal_scale;
    cr_texture_slot base_color_texture;
    cr_texture_slot metallic_roughness_texture;
    cr_texture_slot normal_texture;
    cr_texture_slot emissive_texture;
    cr_texture_slot transmission_texture;
} cr_material;

/* cr::Image (scene.h:176): width*height RGBA float texels, row-major, top row first. */
typedef struct cr_image {
    int32_t width, height;
    const float* pixels;
} cr_image;

/* cr::Texture (scene.h:177). */
typedef struct cr_texture {
    int32_t image;
    int32_t wrap_s, wrap_t;
    int32_t linear;
} cr_texture;

enum { CR_LIGHT_POINT = 0, CR_LIGHT_DIRECTIONAL = 1, CR_LIGHT_SPOT = 2 };

/* cr::PunctualLight (scene.h:211-215). */
typedef struct cr_punctual_light {
    int32_t type;
    float position[3];
    float direction[3];
    float color[3];
    float intensity, range, inner_cone, outer_cone;
} cr_punctual_light;

/* cr::Camera (scene.h:202-207) without its name. */
typedef struct cr_camera {
    float position[3];
    float forward[3];
    float right[3];
    float up[3];
    float yfov, aspect, near_clip, far_clip;
} cr_camera;

/* cr::RenderOptions (render.h:31-39). */
typedef struct cr_render_options {
    int32_t width, height, samples, bounces, threads;
    uint64_t seed;
    int32_t next_event_estimation, russian_roulette;
} cr_render_options;

/* Everything a scene upload needs. triangles must already be finalized (Scene::finalize()).
 * bvh_nodes/bvh_indices may be NULL, in which case the library builds the reference's
 * binned-SAH tree itself (cr_bvh_build). */
typedef struct cr_scene_desc {
    const cr_triangle* triangles;
    uint64_t triangle_count;
    const cr_material* materials;
    uint32_t material_count;
    const cr_punctual_light* lights;
    uint32_t light_count;
    const cr_image* images;
    uint32_t image_count;
    const cr_texture* textures;
    uint32_t texture_count;
    const cr_bvh_node* bvh_nodes;
    uint64_t bvh_node_count;
    const uint32_t* bvh_indices;
    uint64_t bvh_index_count;
} cr_scene_desc;

/* cr::Environment (render.h:8-28). With pixels == NULL it is the constant radiance
 * `constant`. Otherwise a width*height RGBA equirect image; rotation_radians is the
 * already-reduced yaw the reference stores (fmod(degrees,360)*pi/180, render.cpp:24;
 * cr_environment_rotation() computes it). cdf may be NULL (the library rebuilds the
 * reference's FP64 CDF, render.cpp:28-41) or the caller's copy of it. */
typedef struct cr_environment_desc {
    float constant[3];
    const float* pixels;
    int32_t width, height;
    float rotation_radians;
    float intensity;
    const double* cdf;
} cr_environment_desc;

/* Per-render report; mirrors cr::RenderResult (render.h:41-48) plus device figures. */
typedef struct cr_render_stats {
    double seconds;             /* wall time of the call, like RenderResult::seconds    */
    double device_ms;           /* CUDA-event time of all render kernels                 */
    double trace_ms;            /* CUDA-event time of the traversal launches (closest and
                                   any hit share one launch per iteration)              */
    double shade_ms;            /* CUDA-event time of the shading launches              */
    double regen_ms;            /* CUDA-event time of the camera-sample launches        */
    int32_t workers;            /* the reference's worker-count formula (render.cpp:363) */
    int32_t chunks;             /* chunks of sample ids (each accumulated in order)      */
    uint64_t camera_samples;    /* width*height*samples                                  */
    uint64_t boundary_retries;  /* precision replays (render.cpp:409)                    */
    uint64_t extend_rays;       /* closest-hit rays traced                               */
    uint64_t shadow_rays;       /* any-hit rays traced                                   */
    uint64_t kernel_launches;   /* kernels launched by this call                         */
    uint64_t extend_pairs;      /* node pairs fetched by closest-hit (count_traversal)    */
    uint64_t extend_triangles;  /* triangles tested by closest-hit (count_traversal)      */
    uint64_t shadow_pairs;      /* node pairs fetched by any-hit (count_traversal)        */
    uint64_t shadow_triangles;  /* triangles tested by any-hit (count_traversal)          */
    uint64_t iterations;        /* pool iterations (regen, trace, shade)                  */
} cr_render_stats;

typedef void (*cr_progress_fn)(uint64_t complete, uint64_t total, double seconds, void* user);

/* Render-time switches that have no counterpart in cr::RenderOptions. Zero-initialise for
 * the defaults. */
typedef struct cr_gpu_tuning {
    int32_t exact_traversal;   /* 1: FP64 box tests in the reference's order for every ray */
    int32_t env_alias;         /* 1: alias-table environment sampling (different streams)   */
    int32_t paths_per_wave;    /* 0: automatic                                             */
    int32_t chunk_log2;        /* 0: automatic; n in [16, 28]: 2^n sample ids per chunk     */
    int32_t generic_shading;   /* 1: every hit through the generic shading kernel (no
                                  NEE-null class; diagnostic: the films are identical)    */
    int32_t time_phases;       /* 1: CUDA-event time every extend/shade/shadow launch      */
    int32_t count_traversal;   /* 1: count node pairs and triangles visited by closest-hit */
} cr_gpu_tuning;

typedef struct cr_gpu_scene cr_gpu_scene;

/* ---- library ---------------------------------------------------------------------- */
int cr_gpu_abi_version(void);
/* Copies the last error text of this thread into buf (always NUL-terminated when n>0);
 * returns its full length. */
size_t cr_gpu_last_error(char* buf, size_t n);
cr_status cr_gpu_device_count(int* count);

/* ---- host-side restatements of the reference's preparation steps ------------------- */
/* RenderOptions::validate (render.cpp:97-104). */
cr_status cr_options_validate(const cr_render_options* options);
/* Scene::finalize (geometry.cpp:296-397) over the triangle array in place: validates,
 * drops zero-area triangles (compacting the array and renumbering), fixes normals and
 * tangents. *triangle_count is updated. Warnings are joined with '\n' into warnings
 * (may be NULL). */
cr_status cr_scene_finalize(cr_triangle* triangles, uint64_t* triangle_count,
                            const cr_material* materials, uint32_t material_count,
                            const cr_image* images, uint32_t image_count,
                            const cr_texture* textures, uint32_t texture_count,
                            char* warnings, size_t warnings_size);
/* Bvh::build (geometry.cpp:463-550): nodes must hold 2*triangle_count-1 entries (at least
 * one), indices triangle_count entries. *node_count receives the node count. */
cr_status cr_bvh_build(const cr_triangle* triangles, uint64_t triangle_count,
                       cr_bvh_node* nodes, uint64_t* node_count, uint32_t* indices);
/* fmod(degrees, 360) * pi / 180 in float, as Environment's constructor stores it. */
float cr_environment_rotation(float degrees);
/* Environment's importance table (render.cpp:28-41) as the device uses it: cdf receives
 * width*height doubles (may be NULL), weight_sum_integral the weight sum and the luminance
 * integral. A constant environment yields only the integral (4*pi*luminance). */
cr_status cr_environment_tables(const cr_environment_desc* environment, double* cdf,
                                double* weight_sum_integral);

/* ---- device scene ------------------------------------------------------------------ */
cr_status cr_gpu_scene_create(const cr_scene_desc* scene, const cr_environment_desc* environment,
                              int device, cr_gpu_scene** out);
cr_status cr_gpu_scene_destroy(cr_gpu_scene* scene);
/* Device bytes held by the scene (geometry, BVH, environment, work buffers). */
cr_status cr_gpu_scene_bytes(const cr_gpu_scene* scene, uint64_t* bytes);

/* Bvh::intersect over a batch (scene.h:126-127): hits is read as the incoming Hit (its t
 * is the upper bound, geometry.cpp:557) and overwritten where found[i] = 1; rays that
 * find nothing keep their input hit, as the reference leaves Hit untouched. */
cr_status cr_gpu_intersect(cr_gpu_scene* scene, const cr_ray* rays, uint64_t count, int any,
                           uint32_t ignore_triangle, cr_hit* hits, uint8_t* found,
                           const cr_gpu_tuning* tuning);

/* Camera::generate for every pixel of one sample index, with the render's own jitter
 * (two draws of the sample's stream, render.cpp:396-398). rays holds width*height. */
cr_status cr_gpu_camera_rays(cr_gpu_scene* scene, const cr_camera* camera,
                             const cr_render_options* options, uint32_t sample, cr_ray* rays);

/* cr::render (render.cpp:352-456): film_rgb receives width*height linear RGB floats.
 * progress may be NULL; it is called on this thread between sample waves, at most every
 * two seconds, and once at the end. tuning may be NULL. */
cr_status cr_gpu_render(cr_gpu_scene* scene, const cr_camera* camera,
                        const cr_render_options* options, cr_progress_fn progress, void* user,
                        float* film_rgb, cr_render_stats* stats, const cr_gpu_tuning* tuning);

/* As cr_gpu_render, but the film stays in device memory (see cr_gpu_film_download).
 * per_sample_rgb, when not NULL, receives samples*width*height*3 floats: the radiance of
 * every camera sample (sample-major), for stream-level comparisons. */
cr_status cr_gpu_render_resident(cr_gpu_scene* scene, const cr_camera* camera,
                                 const cr_render_options* options, cr_render_stats* stats,
                                 const cr_gpu_tuning* tuning, float* per_sample_rgb);
cr_status cr_gpu_film_download(cr_gpu_scene* scene, float* film_rgb, uint64_t floats);

/* Environment samples (diagnostic; no counterpart in the reference): the texel and density of
 * `count` samples of the environment image, sample i from the stream
 * Rng(sampleSeed(seed, i, 0)), by the reference's CDF search (Environment::sample,
 * render.cpp:67-84; alias = 0) or by the alias table (alias = 1), whose densities are its own
 * realised texel probabilities over the texel's solid angle. For checks of the sampler's
 * distribution. */
cr_status cr_gpu_environment_sample(cr_gpu_scene* scene, int alias, uint64_t seed, uint64_t count,
                                    uint32_t* texels, float* densities);

/* One ray a render traced and the traversal's answer (diagnostic; no counterpart in the
 * reference, whose trace() calls Bvh::intersect, geometry.cpp:554-639, with exactly these
 * arguments: render.cpp:241 for kind 0, render.cpp:284-285 for kind 1). */
typedef struct cr_traced_ray {
    cr_ray ray;
    uint32_t ignore;    /* the query's ignoreTriangle                                        */
    uint32_t kind;      /* 0: closest hit (any = false), 1: shadow ray (any = true)          */
    uint32_t depth;     /* the path's bounce when the ray was traced                         */
    uint32_t found;     /* the traversal's return value                                      */
    uint32_t launch;    /* the pool iteration (traversal launch) of the render that traced it */
    cr_hit hit;         /* kind 0 and found: t, u, v, triangle as the traversal returned them */
} cr_traced_ray;

/* As cr_gpu_render_resident (counting traversal kernels, no per-sample output), and every ray
 * the render traces is recorded: the first `capacity` of them (in no particular order) go to
 * rays, *count receives how many were traced. For parity checks of the traversal on the rays
 * a real render produces, bounce by bounce. */
cr_status cr_gpu_render_trace_dump(cr_gpu_scene* scene, const cr_camera* camera,
                                   const cr_render_options* options, const cr_gpu_tuning* tuning,
                                   cr_traced_ray* rays, uint64_t capacity, uint64_t* count);

/* cr_gpu_render without any allocation (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory while rendering: hosts that hand out GPU
 * memory only at start-up (fixed budgets or their own pools), request paths that must not
 * block on cudaMalloc/cudaFree (both may synchronise the device and can fail under memory
 * pressure mid-request), and code that must not fragment a shared device. Everything the
 * render needs besides the scene (created earlier with cr_gpu_scene_create) comes from one
 * fixed 32 MiB array in device memory that every GPU loading this library holds until the
 * process exits; film_rgb (host memory, width*height*3 floats) receives the same film
 * cr_gpu_render produces.
 *
 * Limits: width*height <= 262144 (512x512); any sample and bounce counts cr::RenderOptions
 * accepts. Larger images fail with CR_ERR_INVALID_ARGUMENT before any work.
 *
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) and
 * creates two timing events, so make that first call before any stream capture. Under the CUDA
 * runtime's lazy module loading (the default since CUDA 12.2) the array is committed on a device
 * when this library's render module first loads there, which can be that first call: make one
 * small call at start-up, while memory is still to be had, and the later calls reserve nothing.
 * stats, when not NULL, is filled as cr_gpu_render fills it, except trace_ms, shade_ms and
 * regen_ms, which stay 0. All calls on a device share the array and
 * it keeps the last call's contents (each call clears what must start at zero); calls that
 * overlap on the GPU — from different threads or scenes on one device — race on it and must
 * be serialised by the caller. */
cr_status cr_gpu_render_noalloc(cr_gpu_scene* scene, const cr_camera* camera,
                                const cr_render_options* options, float* film_rgb,
                                cr_render_stats* stats);

/* Diagnostic (no counterpart in the reference): the number of memory blocks this library has
 * requested since it was loaded, device blocks (cudaMalloc or its own block cache) and
 * page-locked host blocks alike. A call that allocates nothing leaves it unchanged. */
cr_status cr_gpu_allocation_count(uint64_t* count);

/* Fault injection for tests (no counterpart in the reference, which has none): the nth device
 * allocation from now (0: the next one) that goes through the library's device allocator fails
 * as if the device were out of memory, and the call that made it returns CR_ERR_OUT_OF_MEMORY
 * with "device allocation (injected failure)" in its message; a negative nth disarms it. That
 * allocator holds scenes (geometry, sky, alias tables), render workspaces, films, guided-render
 * buffers and the engine's job buffers; the encoder's buffers and page-locked staging do not go
 * through it. Process-wide: allocations made on other threads count too. A failed call leaves
 * every object usable: the same call made again after disarming returns what it would have
 * returned without the failure. */
cr_status cr_gpu_debug_fail_allocation(int64_t nth);

/* ---- output encoding on the device ----------------------------------------------------------
 * Replaces the per-pixel work of io::writePng / io::writeHdr (src/io/image.cpp:100-124,
 * 193-230; scene.h:144-146), which the reference runs on the CPU after cr::render.
 *   CR_ENCODE_SRGB8     width*height*3 bytes: exactly the 8-bit pixels io::writePng passes to
 *                       its PNG codec (exposure in stops, filmic curve, sRGB, rounding).
 *   CR_ENCODE_RGBE      width*height*4 bytes: the shared-exponent quads of the Radiance codec
 *                       io::writeHdr uses (stb_image_write 1.16).
 *   CR_ENCODE_HDR_FILE  the complete .hdr file io::writeHdr writes, byte for byte (header and
 *                       run-length coded scanlines).
 * Pixels are checked as the reference checks them (finite, non-negative; below 2^127 for the
 * HDR forms; exposure within [-100, 100] for SRGB8) and fail with CR_ERR_INVALID_ARGUMENT and
 * the reference's message. `*size` receives the encoded size. With out == NULL nothing is
 * copied; with capacity below the size nothing is copied and CR_ERR_OUT_OF_RANGE returns. */
typedef enum cr_encode_format {
    CR_ENCODE_SRGB8 = 0,
    CR_ENCODE_RGBE = 1,
    CR_ENCODE_HDR_FILE = 2
} cr_encode_format;

/* Host-only. The table the SRGB8 encoder uses: out[k] (k = 1..255) is the least non-negative
 * float whose display byte (io::writePng's mapping at `exposure` stops) is at least k, +inf
 * when none is; out[0] = 0. The mapping is non-decreasing in the linear value, so a pixel's
 * byte is the largest k with out[k] <= value. */
cr_status cr_display_thresholds(float exposure, float* out256);

/* Encodes the film of the scene's last cr_gpu_render / cr_gpu_render_resident /
 * cr_gpu_render_progressive (the film cr_gpu_film_download returns) where it lies. */
cr_status cr_gpu_film_encode(cr_gpu_scene* scene, int format, float exposure, void* out,
                             uint64_t capacity, uint64_t* size);

/* Encodes a caller's film (host memory, width*height*3 floats) on device `device`. */
cr_status cr_gpu_encode(const float* film_rgb, int width, int height, int format, float exposure,
                        int device, void* out, uint64_t capacity, uint64_t* size);

/* Progressive output: cr::render's film after every `every_samples` samples per pixel.
 * on_frame(samples_done, frame, size, user) is called on this thread with the encoded film
 * (format and exposure as cr_gpu_film_encode) at samples_done = every_samples,
 * 2*every_samples, ... and options->samples. Each frame is exactly the film a render with
 * samples = samples_done would return (the per-pixel sums run in sample order). The frame
 * buffer is valid during the call only. Requires every_samples*width*height <= 2^28.
 * film_rgb and stats as cr_gpu_render (film_rgb may be NULL). No counterpart in the
 * reference, whose render returns only the final film. */
typedef void (*cr_frame_fn)(uint32_t samples_done, const void* frame, uint64_t size, void* user);
cr_status cr_gpu_render_progressive(cr_gpu_scene* scene, const cr_camera* camera,
                                    const cr_render_options* options, uint32_t every_samples,
                                    int format, float exposure, cr_frame_fn on_frame, void* user,
                                    float* film_rgb, cr_render_stats* stats,
                                    const cr_gpu_tuning* tuning);

/* ---- phase benchmark -----------------------------------------------------------------------
 * tests/benchmark.cpp:18-62 on the device: camera (count rays at raster positions drawn from
 * Rng(seed) for a width x height image, the reference's rays), closest-hit and occlusion
 * traversal of those rays, surfaceAt for every hit, BSDF sampling and evaluation at every hit,
 * environment sample + radiance + pdf (count calls; the scene's own environment). Each phase
 * is one kernel over all its calls, run once untimed and once timed with CUDA events.
 * out[CR_PHASE_*] receive seconds, calls and the reference's checksum term of each phase
 * (hit t for closest hit, 1 per blocked ray for occlusion, pdfs for the BSDF phases,
 * luminance + pdf for the environment; 0 for camera and surface). The BSDF and environment
 * phases draw call i from its own stream Rng(sampleSeed(seed, i, phase)), where the
 * reference continues one sequential stream. */
enum { CR_PHASE_CAMERA = 0, CR_PHASE_CLOSEST_HIT, CR_PHASE_OCCLUSION, CR_PHASE_SURFACE, CR_PHASE_BSDF_SAMPLE,
       CR_PHASE_BSDF_EVAL, CR_PHASE_ENVIRONMENT, CR_PHASE_COUNT };
typedef struct cr_phase_timing {
    double seconds;
    uint64_t calls;
    double checksum;
} cr_phase_timing;
cr_status cr_gpu_phase_benchmark(cr_gpu_scene* scene, const cr_camera* camera, int32_t width, int32_t height,
                                 uint32_t count, uint64_t seed, cr_phase_timing* out);

/* ---- learned path guiding -----------------------------------------------------------------------
 * No counterpart in the reference. A cr_guide is a small network on one device: 4 dense layers
 * 64 wide map a shading point (position scaled to the scene bounds, outgoing direction,
 * geometric normal; 9 features plus sin/cos of 8 octaves of the position, 64 inputs) to a mixture of 8 von Mises-Fisher
 * lobes (40 outputs: per lobe the mixture logit, log kappa and the unnormalised mean). Its
 * weights are FP32 masters (trained by Adam) with an FP16 copy used by inference on the tensor
 * cores (FP32 accumulation). cr_gpu_render_guided trains it online on the tracer's own radiance
 * samples and samples directions from it, mixed with BSDF sampling by one-sample MIS. */
typedef struct cr_guide cr_guide;
cr_status cr_guide_create(int device, uint64_t seed, cr_guide** out);
cr_status cr_guide_destroy(cr_guide* guide);
uint32_t cr_guide_parameter_count(void);
cr_status cr_guide_get_parameters(cr_guide* guide, float* out);       /* FP32 masters */
cr_status cr_guide_set_parameters(cr_guide* guide, const float* in);  /* also refreshes the FP16 copy */
/* features: n x 9 floats; out: n x 40 network outputs (tensor-core inference). */
cr_status cr_guide_evaluate(cr_guide* guide, const float* features, uint64_t n, float* out);
/* samples: n x 13 floats (features 9, direction 3, weight w). grad (parameter count floats)
 * receives d/dparams of sum_i w_i * -log q_i(direction_i), *loss that sum, with the FP16-rounded
 * weights inference uses. */
cr_status cr_guide_gradients(cr_guide* guide, const float* samples, uint64_t n, float* grad, double* loss);
/* `steps` Adam steps (learning rate lr) over mini-batches of `batch` of the samples, weights
 * normalised by their mean; *loss receives the last batch's loss. */
cr_status cr_guide_train(cr_guide* guide, const float* samples, uint64_t n, uint32_t steps, uint32_t batch, float lr,
                         float* loss);

/* Guided render: cr::render's estimator with the directions at rough, opaque surfaces drawn by
 * one-sample MIS from the guide's mixture (probability guide_probability) and the BSDF, the
 * combined density used in both MIS weights of trace(), so the film stays unbiased. During the
 * first train_samples samples per pixel the render runs one sample per pixel at a time and,
 * after each, trains the guide (Adam, lr 1e-3, `epochs` passes in mini-batches of `batch`) on
 * the light that arrived along each guided direction. The guide keeps its trained weights.
 * gopt may be NULL: train 32 samples, probability 0.5, batch 16384, 4 epochs. */
typedef struct cr_guide_options {
    uint32_t train_samples;
    float guide_probability;
    uint32_t batch;
    uint32_t epochs;
} cr_guide_options;
cr_status cr_gpu_render_guided(cr_gpu_scene* scene, const cr_camera* camera, const cr_render_options* options,
                               cr_guide* guide, const cr_guide_options* gopt, float* film_rgb,
                               cr_render_stats* stats, const cr_gpu_tuning* tuning);

/* ---- many renders in one path pool ------------------------------------------------------------
 * No counterpart in the reference, which renders one image per cr::render call. The engine
 * runs the paths of many jobs (scene, camera, options) in one shared pool on one device: free
 * path slots take the next samples of whichever jobs have samples left, so small and large
 * jobs keep the GPU full together. Each job's samples run on its own streams and its pixel
 * sums are added in sample order, so every job's film is exactly the film cr_gpu_render
 * returns for it alone, whatever else shares the pool. */
typedef struct cr_job {
    /* inputs */
    cr_gpu_scene* scene;          /* every job of one batch or server on the same device     */
    cr_camera camera;
    cr_render_options options;
    float* film_rgb;              /* host, width*height*3 floats, or NULL                     */
    uint32_t every_samples;       /* > 0: on_frame after every N samples per pixel            */
    int32_t format;               /* cr_encode_format of the frames                           */
    float exposure;               /* of CR_ENCODE_SRGB8 frames                                */
    cr_frame_fn on_frame;         /* called on the engine's thread; may be NULL               */
    void* user;
    /* results, written when the job ends */
    cr_status status;
    cr_render_stats stats;        /* camera_samples, boundary_retries, workers, chunks, seconds */
    double submitted_at;          /* seconds on the engine's clock                            */
    double started_at;            /* admitted: buffers allocated, samples may start           */
    double first_frame_at;        /* first progressive frame (0 without frames)               */
    double finished_at;
    char error[256];              /* the failure text, as cr_gpu_last_error would give it     */
} cr_job;

typedef struct cr_engine_tuning {
    uint32_t pool_paths;          /* path slots; 0: 2^24                                      */
    uint32_t range_samples;       /* most samples per issue range; 0: 2^22                    */
    uint32_t refill_interval;     /* iterations between refills of freed slots; 0: 1          */
    uint32_t iterations_per_step; /* iterations between host checks (even); 0: 8              */
    int32_t use_graphs;           /* 1: launch each step as one captured CUDA graph           */
    int32_t issue_policy;         /* 0: automatic (batch: 1, server: 2); 1: jobs in order, each
                                     fed to the end before the next starts (the pool's paths
                                     stay on few scenes: throughput); 2: the job with the fewest
                                     samples per pixel issued first (a new job's first frame
                                     goes ahead: latency)                                      */
    uint64_t memory_budget;       /* bytes of job buffers admitted at once; 0: 150 GB          */
    uint32_t refill_free_percent; /* refill only when at least this share of the pool is free
                                     (new paths then start together, as one wave); 0: always   */
    uint32_t solo_samples_log2;   /* cr_gpu_render_batch: a job with at least 2^n camera
                                     samples between two drains (the whole job; for a
                                     progressive job, every_samples x pixels) fills the device
                                     on its own and renders alone (the single-render path) on a
                                     helper thread beside the pool, which takes the rest;
                                     0: n = 22; 64 or more: every job shares the pool. Servers
                                     ignore it                                                 */
    uint32_t block_size;          /* threads per block of the pool's traversal and shading
                                     kernels: 64, 128 or 256; 0: 128                          */
    uint32_t reserved;            /* must be 0                                                */
} cr_engine_tuning;

typedef struct cr_engine_stats {
    double seconds;               /* wall time the engine was working                         */
    uint64_t camera_samples;      /* of finished jobs                                         */
    uint64_t iterations, launches, extend_rays, shadow_rays;
    uint32_t jobs_done, jobs_failed, peak_jobs, graph_steps;
} cr_engine_stats;

/* Renders every job in one shared pool and returns when all have ended. The call's status is
 * CR_OK when every job succeeded; each job's own status and error say how it ended. */
cr_status cr_gpu_render_batch(cr_job* jobs, uint32_t count, const cr_engine_tuning* tuning,
                              cr_engine_stats* stats);

/* The engine's own autotuner (no counterpart in the reference): picks the pool's queue depth
 * (pool_paths), its regroup interval (iterations_per_step: iterations between the host's
 * regrouping of finished ranges and new issue ranges), its refill threshold and the kernels'
 * block size by timing short trial renders (the jobs that share the pool, at 1 sample per
 * pixel), one dimension after another starting from *tuning, each keeping the fastest value.
 * The jobs are not modified. */
cr_status cr_gpu_autotune_batch(const cr_job* jobs, uint32_t count, cr_engine_tuning* tuning);

/* One trial of the autotuner: the settings and the wall time of its trial batch. */
typedef struct cr_autotune_trial {
    uint32_t pool_paths, iterations_per_step, refill_free_percent, block_size;
    double seconds;
} cr_autotune_trial;
/* As cr_gpu_autotune_batch, and the trials it ran: the first `capacity` go to trials,
 * *trial_count receives how many ran. */
cr_status cr_gpu_autotune_batch_trials(const cr_job* jobs, uint32_t count, cr_engine_tuning* tuning,
                                       cr_autotune_trial* trials, uint32_t capacity,
                                       uint32_t* trial_count);

/* Continuous batching: a server owns an engine thread on `device`. Jobs submitted while
 * others run join the pool as soon as the memory budget admits them; their samples share the
 * pool with the jobs already running. A submitted cr_job must stay valid until it has ended
 * (cr_server_wait returned for it, or the server was destroyed). */
typedef struct cr_server cr_server;
cr_status cr_server_create(int device, const cr_engine_tuning* tuning, cr_server** out);
cr_status cr_server_submit(cr_server* server, cr_job* job, uint64_t* ticket);
/* Waits until the job has ended (returns its status) or timeout_seconds pass
 * (CR_ERR_DEVICE_TIMEOUT, the job keeps running). timeout < 0 waits without limit. */
cr_status cr_server_wait(cr_server* server, uint64_t ticket, double timeout_seconds);
cr_status cr_server_stats(cr_server* server, cr_engine_stats* stats);
double cr_server_clock(cr_server* server);  /* seconds on the engine's clock */
/* Finishes the submitted jobs, stops the thread and frees the engine. */
cr_status cr_server_destroy(cr_server* server);

#ifdef __cplusplus
}
#endif

#endif /* CR_GPU_H */
