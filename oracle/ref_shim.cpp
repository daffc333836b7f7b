// C ABI over the UNMODIFIED reference (CPU-Renderer src/geometry.cpp, src/bsdf.cpp,
// src/render.cpp), compiled from the reference's own source files into
// oracle/_ref/libcr_ref.so by oracle/Makefile. This file is test infrastructure: it is
// the checker that pins the oracle restatement and the GPU backend, and the CPU arm of the
// benchmark. Nothing in the product links it.
//
// The cr_* plain structs of include/cr_gpu.h mirror the reference's value types, so the
// conversions below are field copies. Private members of cr::Bvh and cr::Environment are
// read through the explicit-instantiation access rule (member pointers named in an
// explicit template instantiation are exempt from access checking), which lets the tests
// compare node arrays and CDFs without changing a line of the reference.
#include "render.h"
#include "cr_gpu.h"

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <typeinfo>
#include <vector>

namespace {
template <typename Tag, auto Member>
struct Steal {
    friend auto get(Tag) { return Member; }
};
struct BvhNodesTag { friend auto get(BvhNodesTag); };
struct BvhIndicesTag { friend auto get(BvhIndicesTag); };
struct EnvImageTag { friend auto get(EnvImageTag); };
struct EnvCdfTag { friend auto get(EnvCdfTag); };
struct EnvRotationTag { friend auto get(EnvRotationTag); };
struct EnvIntensityTag { friend auto get(EnvIntensityTag); };
struct EnvWeightSumTag { friend auto get(EnvWeightSumTag); };
}  // namespace
template struct Steal<BvhNodesTag, &cr::Bvh::nodes_>;
template struct Steal<BvhIndicesTag, &cr::Bvh::indices_>;
template struct Steal<EnvImageTag, &cr::Environment::image_>;
template struct Steal<EnvCdfTag, &cr::Environment::cdf_>;
template struct Steal<EnvRotationTag, &cr::Environment::rotation_>;
template struct Steal<EnvIntensityTag, &cr::Environment::intensity_>;
template struct Steal<EnvWeightSumTag, &cr::Environment::weightSum_>;

static_assert(sizeof(cr::Triangle) == sizeof(cr_triangle), "cr_triangle mirrors cr::Triangle");
static_assert(sizeof(cr::Ray) == sizeof(cr_ray), "cr_ray mirrors cr::Ray");
static_assert(sizeof(cr::Hit) == sizeof(cr_hit), "cr_hit mirrors cr::Hit");

namespace {
thread_local std::string lastError;

// Exceptions become (code, text); the type name is kept so tests can check it.
int fail(const std::exception& e) {
    lastError = e.what();
    if (dynamic_cast<const std::invalid_argument*>(&e)) return 1;
    if (dynamic_cast<const std::out_of_range*>(&e)) return 3;
    if (dynamic_cast<const std::length_error*>(&e)) return 4;
    if (dynamic_cast<const std::logic_error*>(&e)) return 5;
    if (dynamic_cast<const std::bad_alloc*>(&e)) return 6;
    if (dynamic_cast<const std::overflow_error*>(&e)) return 10;
    return 2;  // std::runtime_error and anything else
}

cr::Vec3 v3(const float* p) { return {p[0], p[1], p[2]}; }
void put3(float* out, cr::Vec3 v) { out[0] = v.x; out[1] = v.y; out[2] = v.z; }

cr::TextureSlot slot(const cr_texture_slot& s) {
    cr::TextureSlot out;
    out.texture = s.texture; out.texcoord = s.texcoord;
    out.offset = {s.offset[0], s.offset[1]}; out.scale = {s.scale[0], s.scale[1]};
    out.rotation = s.rotation;
    return out;
}

cr::Material material(const cr_material& m) {
    cr::Material out;
    out.baseColor = {m.base_color[0], m.base_color[1], m.base_color[2], m.base_color[3]};
    out.metallic = m.metallic; out.roughness = m.roughness;
    out.emission = v3(m.emission);
    out.transmission = m.transmission; out.ior = m.ior;
    out.thickness = m.thickness; out.attenuationDistance = m.attenuation_distance;
    out.attenuationColor = v3(m.attenuation_color);
    out.doubleSided = m.double_sided != 0;
    out.alphaMode = m.alpha_mode == CR_ALPHA_MASK ? cr::AlphaMode::Mask : cr::AlphaMode::Opaque;
    out.alphaCutoff = m.alpha_cutoff; out.normalScale = m.normal_scale;
    out.baseColorTexture = slot(m.base_color_texture);
    out.metallicRoughnessTexture = slot(m.metallic_roughness_texture);
    out.normalTexture = slot(m.normal_texture);
    out.emissiveTexture = slot(m.emissive_texture);
    out.transmissionTexture = slot(m.transmission_texture);
    return out;
}

cr::Ray ray(const cr_ray& r) {
    cr::Ray out;
    std::memcpy(&out, &r, sizeof(out));
    return out;
}

cr::Camera camera(const cr_camera& c) {
    cr::Camera out;
    out.position = v3(c.position); out.forward = v3(c.forward);
    out.right = v3(c.right); out.up = v3(c.up);
    out.yfov = c.yfov; out.aspect = c.aspect; out.nearClip = c.near_clip; out.farClip = c.far_clip;
    return out;
}

cr::RenderOptions options(const cr_render_options& o) {
    cr::RenderOptions out;
    out.width = o.width; out.height = o.height; out.samples = o.samples;
    out.bounces = o.bounces; out.threads = o.threads; out.seed = o.seed;
    out.nextEventEstimation = o.next_event_estimation != 0;
    out.russianRoulette = o.russian_roulette != 0;
    return out;
}
}  // namespace

extern "C" {

size_t ref_last_error(char* buf, size_t n) {
    if (buf && n) {
        const size_t k = std::min(n - 1, lastError.size());
        std::memcpy(buf, lastError.data(), k);
        buf[k] = 0;
    }
    return lastError.size();
}

// ---- scene ------------------------------------------------------------------------------
void* ref_scene_new(const cr_scene_desc* d) {
    try {
        auto s = std::make_unique<cr::Scene>();
        s->triangles.resize(d->triangle_count);
        if (d->triangle_count) std::memcpy(s->triangles.data(), d->triangles, d->triangle_count * sizeof(cr_triangle));
        for (uint32_t i = 0; i < d->material_count; ++i) s->materials.push_back(material(d->materials[i]));
        for (uint32_t i = 0; i < d->light_count; ++i) {
            const cr_punctual_light& l = d->lights[i];
            cr::PunctualLight p;
            p.type = l.type == CR_LIGHT_DIRECTIONAL ? cr::LightType::Directional
                   : l.type == CR_LIGHT_SPOT ? cr::LightType::Spot : cr::LightType::Point;
            p.position = v3(l.position); p.direction = v3(l.direction); p.color = v3(l.color);
            p.intensity = l.intensity; p.range = l.range; p.innerCone = l.inner_cone; p.outerCone = l.outer_cone;
            s->lights.push_back(p);
        }
        for (uint32_t i = 0; i < d->image_count; ++i) {
            cr::Image im;
            im.width = d->images[i].width; im.height = d->images[i].height;
            const size_t n = static_cast<size_t>(im.width) * static_cast<size_t>(im.height);
            im.pixels.resize(n);
            if (n) std::memcpy(im.pixels.data(), d->images[i].pixels, n * sizeof(cr::Vec4));
            s->images.push_back(std::move(im));
        }
        for (uint32_t i = 0; i < d->texture_count; ++i) {
            const cr_texture& t = d->textures[i];
            auto wrap = [](int32_t w) { return w == CR_WRAP_CLAMP ? cr::Wrap::Clamp : w == CR_WRAP_MIRROR ? cr::Wrap::Mirror : cr::Wrap::Repeat; };
            s->textures.push_back({t.image, wrap(t.wrap_s), wrap(t.wrap_t), t.linear != 0});
        }
        return s.release();
    } catch (const std::exception& e) { fail(e); return nullptr; }
}
void ref_scene_free(void* s) { delete static_cast<cr::Scene*>(s); }

int ref_scene_finalize(void* s, char* warnings, size_t n) {
    try {
        auto* scene = static_cast<cr::Scene*>(s);
        scene->warnings.clear();
        scene->finalize();
        std::string joined;
        for (const auto& w : scene->warnings) { if (!joined.empty()) joined += '\n'; joined += w; }
        if (warnings && n) {
            const size_t k = std::min(n - 1, joined.size());
            std::memcpy(warnings, joined.data(), k);
            warnings[k] = 0;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
uint64_t ref_scene_triangle_count(const void* s) { return static_cast<const cr::Scene*>(s)->triangles.size(); }
void ref_scene_get_triangles(const void* s, cr_triangle* out) {
    const auto* scene = static_cast<const cr::Scene*>(s);
    if (!scene->triangles.empty()) std::memcpy(out, scene->triangles.data(), scene->triangles.size() * sizeof(cr_triangle));
}

// ---- BVH --------------------------------------------------------------------------------
void* ref_bvh_new(const void* s) {
    try {
        auto b = std::make_unique<cr::Bvh>();
        b->build(*static_cast<const cr::Scene*>(s));
        return b.release();
    } catch (const std::exception& e) { fail(e); return nullptr; }
}
void ref_bvh_free(void* b) { delete static_cast<cr::Bvh*>(b); }
uint64_t ref_bvh_node_count(const void* b) { return static_cast<const cr::Bvh*>(b)->nodeCount(); }
void ref_bvh_export(const void* b, cr_bvh_node* nodes, uint32_t* indices) {
    const auto* bvh = static_cast<const cr::Bvh*>(b);
    const auto& ns = bvh->*get(BvhNodesTag{});
    const auto& is = bvh->*get(BvhIndicesTag{});
    for (size_t i = 0; i < ns.size(); ++i) {
        put3(nodes[i].lo, ns[i].box.lo); put3(nodes[i].hi, ns[i].box.hi);
        nodes[i].first = ns[i].first; nodes[i].count = ns[i].count;
    }
    if (!is.empty()) std::memcpy(indices, is.data(), is.size() * sizeof(uint32_t));
}

// Bvh::intersect per ray; hits are read as the incoming Hit and written back as the
// reference leaves them (untouched on a miss).
int ref_intersect(const void* s, const void* b, const cr_ray* rays, uint64_t n, int any,
                  uint32_t ignore, cr_hit* hits, uint8_t* found) {
    try {
        const auto& scene = *static_cast<const cr::Scene*>(s);
        const auto& bvh = *static_cast<const cr::Bvh*>(b);
        for (uint64_t i = 0; i < n; ++i) {
            cr::Hit h;
            std::memcpy(&h, &hits[i], sizeof(h));
            found[i] = bvh.intersect(scene, ray(rays[i]), h, any != 0, ignore) ? 1 : 0;
            std::memcpy(&hits[i], &h, sizeof(h));
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
// Bvh::intersect over rays that each carry their own ignoreTriangle (the rays a render
// traced), split across `threads` host threads.
int ref_intersect_rays(const void* s, const void* b, const cr_ray* rays, const uint32_t* ignores, uint64_t n,
                       int any, cr_hit* hits, uint8_t* found, int threads) {
    try {
        const auto& scene = *static_cast<const cr::Scene*>(s);
        const auto& bvh = *static_cast<const cr::Bvh*>(b);
        const uint64_t workers = std::max<uint64_t>(1, std::min<uint64_t>(threads > 0 ? threads : 1, n));
        std::vector<std::thread> pool;
        std::vector<std::string> errors(workers);
        for (uint64_t w = 0; w < workers; ++w) {
            pool.emplace_back([&, w] {
                try {
                    for (uint64_t i = w; i < n; i += workers) {
                        cr::Hit h;
                        std::memcpy(&h, &hits[i], sizeof(h));
                        found[i] = bvh.intersect(scene, ray(rays[i]), h, any != 0, ignores[i]) ? 1 : 0;
                        std::memcpy(&hits[i], &h, sizeof(h));
                    }
                } catch (const std::exception& e) { errors[w] = e.what(); }
            });
        }
        for (auto& t : pool) t.join();
        for (auto& e : errors)
            if (!e.empty()) throw std::runtime_error(e);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
// intersectTriangle and Bounds::intersect (geometry.cpp:120-182), one call each.
int ref_intersect_triangle(const cr_triangle* t, const cr_ray* r, cr_hit* hit) {
    cr::Triangle tri; std::memcpy(&tri, t, sizeof(tri));
    cr::Hit h; std::memcpy(&h, hit, sizeof(h));
    const bool ok = cr::intersectTriangle(tri, ray(*r), h);
    std::memcpy(hit, &h, sizeof(h));
    return ok ? 1 : 0;
}
int ref_bounds_intersect(const float* lo, const float* hi, const cr_ray* r, float* nearDistance) {
    cr::Bounds b; b.lo = v3(lo); b.hi = v3(hi);
    return b.intersect(ray(*r), *nearDistance) ? 1 : 0;
}

// ---- camera, offsets --------------------------------------------------------------------
int ref_camera_generate(const cr_camera* c, const float* px, const float* py, uint64_t n,
                        int width, int height, cr_ray* out) {
    try {
        const cr::Camera cam = camera(*c);
        for (uint64_t i = 0; i < n; ++i) {
            const cr::Ray r = cam.generate(px[i], py[i], width, height);
            std::memcpy(&out[i], &r, sizeof(r));
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
int ref_offset_ray(const float* position, const float* normal, const float* direction, float maxDistance, cr_ray* out) {
    try {
        const cr::Ray r = cr::offsetRay(v3(position), v3(normal), v3(direction), maxDistance);
        std::memcpy(out, &r, sizeof(r));
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
uint64_t ref_sample_seed(uint64_t seed, uint64_t pixel, uint64_t sample) { return cr::sampleSeed(seed, pixel, sample); }

// ---- environment ------------------------------------------------------------------------
void* ref_env_new(const cr_environment_desc* e, float rotationDegrees) {
    try {
        if (!e->pixels) return new cr::Environment(v3(e->constant));
        cr::Image im;
        im.width = e->width; im.height = e->height;
        im.pixels.resize(static_cast<size_t>(e->width) * static_cast<size_t>(e->height));
        std::memcpy(im.pixels.data(), e->pixels, im.pixels.size() * sizeof(cr::Vec4));
        return new cr::Environment(std::move(im), rotationDegrees, e->intensity);
    } catch (const std::exception& ex) { fail(ex); return nullptr; }
}
void ref_env_free(void* e) { delete static_cast<cr::Environment*>(e); }
// CDF, weight sum, integral and stored rotation/intensity, as the reference holds them.
uint64_t ref_env_export(const void* e, double* cdf, double* weightSumIntegral, float* rotationIntensity) {
    const auto* env = static_cast<const cr::Environment*>(e);
    const auto& c = env->*get(EnvCdfTag{});
    if (cdf && !c.empty()) std::memcpy(cdf, c.data(), c.size() * sizeof(double));
    if (weightSumIntegral) { weightSumIntegral[0] = env->*get(EnvWeightSumTag{}); weightSumIntegral[1] = env->integral(); }
    if (rotationIntensity) { rotationIntensity[0] = env->*get(EnvRotationTag{}); rotationIntensity[1] = env->*get(EnvIntensityTag{}); }
    return c.size();
}
// Draw n environment samples from one stream (Environment::sample, render.cpp:67-84).
void ref_env_sample(const void* e, uint64_t* rngState, uint64_t n, float* dirs, float* pdfs) {
    const auto* env = static_cast<const cr::Environment*>(e);
    cr::Rng rng(*rngState);
    for (uint64_t i = 0; i < n; ++i) { const cr::Vec3 d = env->sample(rng, pdfs[i]); put3(dirs + 3 * i, d); }
    *rngState = rng.state;
}
void ref_env_eval(const void* e, const float* dirs, uint64_t n, float* radiance, float* pdfs) {
    const auto* env = static_cast<const cr::Environment*>(e);
    for (uint64_t i = 0; i < n; ++i) {
        const cr::Vec3 d = v3(dirs + 3 * i);
        put3(radiance + 3 * i, env->radiance(d));
        pdfs[i] = env->pdf(d);
    }
}

// ---- BSDF -------------------------------------------------------------------------------
// Surface given as 24 floats: normal, geometricNormal, tangent, bitangent (3 each), baseColor
// (3), metallic, roughness, transmission, ior, thickness, frontFace, doubleSided.
static cr::Surface surface(const float* f) {
    cr::Surface s;
    s.normal = v3(f); s.geometricNormal = v3(f + 3); s.tangent = v3(f + 6); s.bitangent = v3(f + 9);
    s.baseColor = v3(f + 12);
    s.metallic = f[15]; s.roughness = f[16]; s.transmission = f[17]; s.ior = f[18]; s.thickness = f[19];
    s.frontFace = f[20] != 0; s.doubleSided = f[21] != 0;
    return s;
}
// n samples of sampleBsdf from one stream; out per sample: dir(3) weight(3) pdf eta delta transmitted ok
void ref_sample_bsdf(const float* surf, const float* wo, uint64_t* rngState, uint64_t n, float* out) {
    const cr::Surface s = surface(surf);
    cr::Rng rng(*rngState);
    for (uint64_t i = 0; i < n; ++i) {
        const cr::BsdfSample b = cr::sampleBsdf(s, v3(wo), rng);
        float* o = out + 11 * i;
        put3(o, b.direction); put3(o + 3, b.weight);
        o[6] = b.pdf; o[7] = b.eta; o[8] = b.delta; o[9] = b.transmitted; o[10] = static_cast<bool>(b) ? 1.f : 0.f;
    }
    *rngState = rng.state;
}
void ref_evaluate_bsdf(const float* surf, const float* wo, const float* wi, uint64_t n, float* out) {
    const cr::Surface s = surface(surf);
    for (uint64_t i = 0; i < n; ++i) {
        const cr::BsdfEval e = cr::evaluateBsdf(s, v3(wo), v3(wi + 3 * i));
        put3(out + 4 * i, e.value); out[4 * i + 3] = e.pdf;
    }
}

// ---- render -----------------------------------------------------------------------------
int ref_options_validate(const cr_render_options* o) {
    try { options(*o).validate(); return 0; } catch (const std::exception& e) { return fail(e); }
}
int ref_render(const void* s, const void* b, const cr_camera* c, const void* e, const cr_render_options* o,
               float* film, cr_render_stats* stats) {
    try {
        const cr::RenderResult r = cr::render(*static_cast<const cr::Scene*>(s), *static_cast<const cr::Bvh*>(b),
                                              camera(*c), *static_cast<const cr::Environment*>(e), options(*o));
        if (film && !r.pixels.empty()) std::memcpy(film, r.pixels.data(), r.pixels.size() * sizeof(cr::Vec3));
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->seconds = r.seconds; stats->workers = r.workers;
            stats->camera_samples = r.cameraSamples; stats->boundary_retries = r.boundaryRetries;
        }
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// ---- io::writePng / io::writeHdr (image.cpp:193-230), to files -----------------------------------
int ref_write_png(const char* path, int width, int height, const float* rgb, float exposure) {
    try {
        std::vector<cr::Vec3> px(static_cast<size_t>(width > 0 && height > 0 ? width : 0) * static_cast<size_t>(height > 0 ? height : 0));
        for (size_t i = 0; i < px.size(); ++i) px[i] = v3(rgb + 3 * i);
        cr::io::writePng(path, width, height, px, exposure);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
int ref_write_hdr(const char* path, int width, int height, const float* rgb) {
    try {
        std::vector<cr::Vec3> px(static_cast<size_t>(width > 0 && height > 0 ? width : 0) * static_cast<size_t>(height > 0 ? height : 0));
        for (size_t i = 0; i < px.size(); ++i) px[i] = v3(rgb + 3 * i);
        cr::io::writeHdr(path, width, height, px);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"
