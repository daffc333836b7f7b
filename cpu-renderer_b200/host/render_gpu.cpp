// GPU drop-in for CPU-Renderer's cr::render (src/render.h:53, src/render.cpp:352-456).
//
// Build the reference's `renderer` library as usual, with src/render.cpp compiled under
// -Drender=<another name> (the token `render` names only that function there and in
// render.h:53), add this file and link libcr_b200.so. The reference's own object then still
// provides cr::Environment (render.h:8-28) and cr::RenderOptions::validate (render.h:38),
// which the CPU side keeps using for its sample/pdf/radiance queries, and this file provides
// the one definition of cr::render: it uploads the scene, the caller's own BVH node array and
// the environment to the GPU, renders with the wavefront tracer and returns the film.
//
// Errors keep the reference's types and texts: validation throws std::runtime_error before
// any allocation, and a failing sample throws std::runtime_error("Pixel (x,y), sample s: ...").
// Progress is called on the calling thread between sample waves, at most every two seconds,
// and once at the end (render.cpp:419-427, 454). RenderResult::workers reports the worker
// count the CPU renderer would have used (render.cpp:363), so callers that check it see the
// same value; the GPU ignores it.
//
// The private members of cr::Bvh and cr::Environment are read through the explicit-
// instantiation access rule (member pointers named in an explicit template instantiation are
// exempt from access checks), so the reference's headers stay unmodified.
#include "render.h"
#include "cr_gpu.h"
#include "render_gpu.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {
template <typename Tag, auto Member>
struct Access { friend auto get(Tag) { return Member; } };
struct BvhNodes { friend auto get(BvhNodes); };
struct BvhIndices { friend auto get(BvhIndices); };
struct EnvImage { friend auto get(EnvImage); };
struct EnvConstant { friend auto get(EnvConstant); };
struct EnvRotation { friend auto get(EnvRotation); };
struct EnvIntensity { friend auto get(EnvIntensity); };
struct EnvCdf { friend auto get(EnvCdf); };
}  // namespace
template struct Access<BvhNodes, &cr::Bvh::nodes_>;
template struct Access<BvhIndices, &cr::Bvh::indices_>;
template struct Access<EnvImage, &cr::Environment::image_>;
template struct Access<EnvConstant, &cr::Environment::constant_>;
template struct Access<EnvRotation, &cr::Environment::rotation_>;
template struct Access<EnvIntensity, &cr::Environment::intensity_>;
template struct Access<EnvCdf, &cr::Environment::cdf_>;

static_assert(sizeof(cr::Triangle) == sizeof(cr_triangle), "cr_triangle mirrors cr::Triangle");

namespace cr {

namespace {
std::string lastError() {
    char buf[4096];
    cr_gpu_last_error(buf, sizeof(buf));
    return buf;
}
[[noreturn]] void raise(cr_status s) {
    const std::string m = lastError();
    if (s == CR_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
    throw std::runtime_error(m);
}
cr_texture_slot slot(const TextureSlot& s) {
    return {s.texture, s.texcoord, {s.offset.x, s.offset.y}, {s.scale.x, s.scale.y}, s.rotation};
}
struct ProgressThunk {
    const Progress* fn;
    static void call(uint64_t done, uint64_t total, double seconds, void* user) {
        (*static_cast<ProgressThunk*>(user)->fn)(done, total, seconds);
    }
};
struct SceneGuard {
    cr_gpu_scene* s = nullptr;
    ~SceneGuard() { if (s) cr_gpu_scene_destroy(s); }
};
}  // namespace

// ---- scene upload (shared with the drop-in phase benchmark) ---------------------------------------
cr_gpu_scene* uploadToGpu(const Scene& scene, const Bvh& bvh, const Environment& environment, int device) {
    // Scene arrays: triangles are binary-compatible; materials lose their names.
    std::vector<cr_material> materials(scene.materials.size());
    for (std::size_t i = 0; i < materials.size(); ++i) {
        const Material& m = scene.materials[i];
        cr_material& o = materials[i];
        std::memcpy(o.base_color, &m.baseColor, sizeof(o.base_color));
        o.metallic = m.metallic; o.roughness = m.roughness;
        o.emission[0] = m.emission.x; o.emission[1] = m.emission.y; o.emission[2] = m.emission.z;
        o.transmission = m.transmission; o.ior = m.ior; o.thickness = m.thickness;
        o.attenuation_distance = m.attenuationDistance;
        o.attenuation_color[0] = m.attenuationColor.x; o.attenuation_color[1] = m.attenuationColor.y; o.attenuation_color[2] = m.attenuationColor.z;
        o.double_sided = m.doubleSided; o.alpha_mode = m.alphaMode == AlphaMode::Mask ? CR_ALPHA_MASK : CR_ALPHA_OPAQUE;
        o.alpha_cutoff = m.alphaCutoff; o.normal_scale = m.normalScale;
        o.base_color_texture = slot(m.baseColorTexture); o.metallic_roughness_texture = slot(m.metallicRoughnessTexture);
        o.normal_texture = slot(m.normalTexture); o.emissive_texture = slot(m.emissiveTexture);
        o.transmission_texture = slot(m.transmissionTexture);
    }
    std::vector<cr_punctual_light> lights(scene.lights.size());
    for (std::size_t i = 0; i < lights.size(); ++i) {
        const PunctualLight& l = scene.lights[i];
        cr_punctual_light& o = lights[i];
        o.type = l.type == LightType::Directional ? CR_LIGHT_DIRECTIONAL : l.type == LightType::Spot ? CR_LIGHT_SPOT : CR_LIGHT_POINT;
        std::memcpy(o.position, &l.position, 12); std::memcpy(o.direction, &l.direction, 12); std::memcpy(o.color, &l.color, 12);
        o.intensity = l.intensity; o.range = l.range; o.inner_cone = l.innerCone; o.outer_cone = l.outerCone;
    }
    std::vector<cr_image> images(scene.images.size());
    for (std::size_t i = 0; i < images.size(); ++i)
        images[i] = {scene.images[i].width, scene.images[i].height, reinterpret_cast<const float*>(scene.images[i].pixels.data())};
    std::vector<cr_texture> textures(scene.textures.size());
    for (std::size_t i = 0; i < textures.size(); ++i) {
        const Texture& t = scene.textures[i];
        auto w = [](Wrap x) { return x == Wrap::Clamp ? CR_WRAP_CLAMP : x == Wrap::Mirror ? CR_WRAP_MIRROR : CR_WRAP_REPEAT; };
        textures[i] = {t.image, w(t.wrapS), w(t.wrapT), t.linear ? 1 : 0};
    }
    // The caller's own BVH, node for node (Bvh::Node has cr_bvh_node's layout).
    const auto& nodes = bvh.*get(BvhNodes{});
    const auto& indices = bvh.*get(BvhIndices{});
    std::vector<cr_bvh_node> flat(nodes.size());
    for (std::size_t i = 0; i < nodes.size(); ++i) {
        std::memcpy(flat[i].lo, &nodes[i].box.lo, 12);
        std::memcpy(flat[i].hi, &nodes[i].box.hi, 12);
        flat[i].first = nodes[i].first;
        flat[i].count = nodes[i].count;
    }
    cr_scene_desc d{};
    d.triangles = reinterpret_cast<const cr_triangle*>(scene.triangles.data());
    d.triangle_count = scene.triangles.size();
    d.materials = materials.data(); d.material_count = static_cast<uint32_t>(materials.size());
    d.lights = lights.data(); d.light_count = static_cast<uint32_t>(lights.size());
    d.images = images.data(); d.image_count = static_cast<uint32_t>(images.size());
    d.textures = textures.data(); d.texture_count = static_cast<uint32_t>(textures.size());
    d.bvh_nodes = flat.data(); d.bvh_node_count = flat.size();
    d.bvh_indices = indices.data(); d.bvh_index_count = indices.size();
    const Image& image = environment.*get(EnvImage{});
    const Vec3 constant = environment.*get(EnvConstant{});
    cr_environment_desc e{};
    e.constant[0] = constant.x; e.constant[1] = constant.y; e.constant[2] = constant.z;
    if (!image.pixels.empty()) {
        e.pixels = reinterpret_cast<const float*>(image.pixels.data());
        e.width = image.width; e.height = image.height;
        e.cdf = (environment.*get(EnvCdf{})).data();
    }
    e.rotation_radians = environment.*get(EnvRotation{});
    e.intensity = environment.*get(EnvIntensity{});

    cr_gpu_scene* handle = nullptr;
    const cr_status st = cr_gpu_scene_create(&d, &e, device, &handle);
    if (st != CR_OK) raise(st);
    return handle;
}

// ---- render (render.cpp:352-456) ----------------------------------------------------------------
RenderResult render(const Scene& scene, const Bvh& bvh, const Camera& camera, const Environment& environment,
                    const RenderOptions& options, Progress progress) {
    options.validate();
    SceneGuard g;
    g.s = uploadToGpu(scene, bvh, environment, 0);
    cr_status st = CR_OK;
    cr_camera c{};
    std::memcpy(c.position, &camera.position, 12); std::memcpy(c.forward, &camera.forward, 12);
    std::memcpy(c.right, &camera.right, 12); std::memcpy(c.up, &camera.up, 12);
    c.yfov = camera.yfov; c.aspect = camera.aspect; c.near_clip = camera.nearClip; c.far_clip = camera.farClip;
    cr_render_options o{options.width, options.height, options.samples, options.bounces, options.threads, options.seed,
                        options.nextEventEstimation, options.russianRoulette};
    RenderResult result;
    result.pixels.resize(static_cast<std::size_t>(options.width) * options.height);
    cr_render_stats stats{};
    ProgressThunk thunk{&progress};
    st = cr_gpu_render(g.s, &c, &o, progress ? &ProgressThunk::call : nullptr, &thunk,
                       reinterpret_cast<float*>(result.pixels.data()), &stats, nullptr);
    if (st != CR_OK) raise(st);
    result.seconds = stats.seconds;
    result.workers = stats.workers;
    result.cameraSamples = stats.camera_samples;
    result.boundaryRetries = stats.boundary_retries;
    return result;
}

}  // namespace cr
