// Host-side restatements of CPU-Renderer's preparation steps and the C ABI entry points
// that need no GPU: option validation (render.cpp:97-104), Scene::finalize
// (geometry.cpp:296-397), Bvh::build (geometry.cpp:463-550), the environment CDF
// (render.cpp:12-42) and the light-selection table (render.cpp:131-160).
//
// This file is compiled by the host compiler with the reference's floating-point rules (no
// FMA, IEEE float/double, glibc libm), so the arrays it produces are bit-identical to the
// reference's. The tests compare node arrays, CDFs and finalized triangles against the
// reference built from its own sources.
#include "cr_host.h"

#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <sstream>
#include <thread>

namespace crh {
namespace {

constexpr float pi = 3.14159265358979323846f;
constexpr float infinity = std::numeric_limits<float>::infinity();

// ---- value types mirroring math.h ------------------------------------------------------
struct Vec3 {
    float x = 0, y = 0, z = 0;
    Vec3() = default;
    explicit Vec3(float s) : x(s), y(s), z(s) {}
    Vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
Vec3 operator*(Vec3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
Vec3 operator/(Vec3 a, float b) { return a * (1.0f / b); }
float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
Vec3 cross(Vec3 a, Vec3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float lengthSquared(Vec3 a) { return dot(a, a); }
float length(Vec3 a) { return std::sqrt(lengthSquared(a)); }
Vec3 normalize(Vec3 a) { const float l = length(a); return l > 0 ? a / l : Vec3{}; }
bool finite(Vec3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
Vec3 vmin(Vec3 a, Vec3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
Vec3 vmax(Vec3 a, Vec3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
float luminance(Vec3 a) { return dot(a, {0.2126f, 0.7152f, 0.0722f}); }
Vec3 v3(const float* p) { return {p[0], p[1], p[2]}; }
void put(float* o, Vec3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

struct Frame {
    Vec3 x, y, z;
    explicit Frame(Vec3 normal) : z(normal) {
        x = normalize(cross(std::abs(z.z) < 0.999f ? Vec3{0, 0, 1} : Vec3{0, 1, 0}, z));
        y = cross(z, x);
    }
};

struct DVec3 {
    double x, y, z;
    explicit DVec3(Vec3 v) : x(v.x), y(v.y), z(v.z) {}
    DVec3(double a, double b, double c) : x(a), y(b), z(c) {}
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
DVec3 operator+(DVec3 a, DVec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
DVec3 operator-(DVec3 a, DVec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
DVec3 operator*(DVec3 a, double b) { return {a.x * b, a.y * b, a.z * b}; }
double preciseDot(DVec3 a, DVec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DVec3 preciseCross(DVec3 a, DVec3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
Vec3 unit(DVec3 v, Vec3 fallback = {}) {
    const double squared = preciseDot(v, v);
    if (!(squared > 0) || !std::isfinite(squared)) return fallback;
    const double inverse = 1 / std::sqrt(squared);
    return {static_cast<float>(v.x * inverse), static_cast<float>(v.y * inverse), static_cast<float>(v.z * inverse)};
}
Vec3 unit(Vec3 v, Vec3 fallback = {}) { return unit(DVec3(v), fallback); }
Vec3 orthogonalized(DVec3 v, Vec3 n, Vec3 fallback = {}) {
    const double normalSquared = preciseDot(DVec3(n), DVec3(n));
    if (!(normalSquared > 0)) return fallback;
    const DVec3 projected = v - DVec3(n) * (preciseDot(v, DVec3(n)) / normalSquared);
    constexpr double tolerance = 4 * std::numeric_limits<float>::epsilon();
    if (preciseDot(projected, projected) <= preciseDot(v, v) * tolerance * tolerance) return fallback;
    return unit(projected, fallback);
}
bool nonzero(Vec3 v) { return v.x != 0 || v.y != 0 || v.z != 0; }

struct Bounds {
    Vec3 lo{infinity}, hi{-infinity};
    void expand(Vec3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void expand(const Bounds& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
};
Bounds triangleBounds(const cr_triangle& t) {
    Bounds b;
    for (const auto& v : t.v) b.expand(v3(v.position));
    return b;
}
Vec3 centroid(const cr_triangle& t) {  // geometry.cpp:57-60
    const DVec3 c = (DVec3(v3(t.v[0].position)) + DVec3(v3(t.v[1].position)) + DVec3(v3(t.v[2].position))) * (1.0 / 3.0);
    return {static_cast<float>(c.x), static_cast<float>(c.y), static_cast<float>(c.z)};
}
double boundsArea(const Bounds& b) {  // geometry.cpp:61-65
    if (b.lo.x > b.hi.x || b.lo.y > b.hi.y || b.lo.z > b.hi.z) return 0;
    const DVec3 d = DVec3(b.hi) - DVec3(b.lo);
    return 2 * (d.x * d.y + d.y * d.z + d.z * d.x);
}

// ---- BVH build ----------------------------------------------------------------------------
constexpr int binCount = 16;      // geometry.cpp:12-14
constexpr int maxBvhDepth = 48;
constexpr uint32_t leafSize = 4;

// Two-pointer partition in the order libstdc++'s std::partition uses for bidirectional
// iterators (advance from the front while the predicate holds, retreat from the back while it
// does not, swap, repeat). The reference partitions with std::partition
// (geometry.cpp:539-541); following the same swap order gives the same leaf contents.
template <class It, class Pred>
It partitionTwoPointer(It first, It last, Pred pred) {
    for (;;) {
        for (;;) {
            if (first == last) return first;
            if (pred(*first)) ++first; else break;
        }
        --last;
        for (;;) {
            if (first == last) return first;
            if (!pred(*last)) --last; else break;
        }
        std::iter_swap(first, last);
        ++first;
    }
}

struct Builder {
    const cr_triangle* tris;
    std::vector<cr_bvh_node>& nodes;
    std::vector<uint32_t>& indices;
    std::vector<Vec3> centroids;
    std::vector<Bounds> boxes;

    void setNode(uint32_t n, const Bounds& b, uint32_t first, uint32_t count) {
        put(nodes[n].lo, b.lo); put(nodes[n].hi, b.hi);
        nodes[n].first = first; nodes[n].count = count;
    }
    void subdivide(uint32_t nodeIndex, uint32_t begin, uint32_t end, int depth) {
        Bounds bounds, centers;
        for (uint32_t i = begin; i < end; ++i) {
            bounds.expand(boxes[indices[i]]);
            centers.expand(centroids[indices[i]]);
        }
        setNode(nodeIndex, bounds, begin, end - begin);
        if (end - begin <= leafSize || depth >= maxBvhDepth) return;
        const double parentArea = boundsArea(bounds);
        if (!(parentArea > 0)) return;
        struct Bin { Bounds bounds; uint32_t count = 0; };
        std::array<std::array<Bin, binCount>, 3> bins{};
        const auto binAt = [&](float center, int axis) {
            const double extent = static_cast<double>(centers.hi[axis]) - centers.lo[axis];
            if (!(extent > 0)) return 0;
            return std::clamp(static_cast<int>((static_cast<double>(center) - centers.lo[axis]) / extent * binCount), 0, binCount - 1);
        };
        for (uint32_t i = begin; i < end; ++i) {
            const Bounds& box = boxes[indices[i]];
            const Vec3 center = centroids[indices[i]];
            for (int axis = 0; axis < 3; ++axis) {
                Bin& bin = bins[axis][binAt(center[axis], axis)];
                bin.bounds.expand(box);
                ++bin.count;
            }
        }
        int bestAxis = -1, bestSplit = -1;
        double bestCost = static_cast<double>(end - begin) * parentArea;
        for (int axis = 0; axis < 3; ++axis) {
            if (centers.lo[axis] == centers.hi[axis]) continue;
            std::array<Bounds, binCount> rightBounds{};
            std::array<uint32_t, binCount> rightCount{};
            Bounds right;
            uint32_t count = 0;
            for (int b = binCount - 1; b >= 0; --b) {
                if (bins[axis][b].count) right.expand(bins[axis][b].bounds);
                count += bins[axis][b].count;
                rightBounds[b] = right;
                rightCount[b] = count;
            }
            Bounds left;
            count = 0;
            for (int b = 0; b < binCount - 1; ++b) {
                if (bins[axis][b].count) left.expand(bins[axis][b].bounds);
                count += bins[axis][b].count;
                if (!count || !rightCount[b + 1]) continue;
                const double cost = parentArea + count * boundsArea(left) + rightCount[b + 1] * boundsArea(rightBounds[b + 1]);
                if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestSplit = b; }
            }
        }
        if (bestAxis < 0) return;
        const auto middle = partitionTwoPointer(indices.begin() + begin, indices.begin() + end, [&](uint32_t index) {
            return binAt(centroids[index][bestAxis], bestAxis) <= bestSplit;
        });
        const uint32_t mid = static_cast<uint32_t>(middle - indices.begin());
        if (mid == begin || mid == end) return;
        const uint32_t firstChild = static_cast<uint32_t>(nodes.size());
        nodes.resize(nodes.size() + 2);
        nodes[nodeIndex].first = firstChild;
        nodes[nodeIndex].count = 0;
        subdivide(firstChild, begin, mid, depth + 1);
        subdivide(firstChild + 1, mid, end, depth + 1);
    }
};

// ---- finalize helpers (geometry.cpp:48-116) ----------------------------------------------
bool finite4(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]) && std::isfinite(v[3]); }
bool finite2(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]); }
bool uvDirections(const cr_triangle& t, int set, DVec3& tangent, DVec3& bitangent) {
    const double du1 = static_cast<double>(t.v[1].uv[set][0]) - t.v[0].uv[set][0];
    const double dv1 = static_cast<double>(t.v[1].uv[set][1]) - t.v[0].uv[set][1];
    const double du2 = static_cast<double>(t.v[2].uv[set][0]) - t.v[0].uv[set][0];
    const double dv2 = static_cast<double>(t.v[2].uv[set][1]) - t.v[0].uv[set][1];
    const double determinant = du1 * dv2 - dv1 * du2;
    if (determinant == 0) return false;
    const DVec3 e1 = DVec3(v3(t.v[1].position)) - DVec3(v3(t.v[0].position));
    const DVec3 e2 = DVec3(v3(t.v[2].position)) - DVec3(v3(t.v[0].position));
    const double sign = determinant < 0 ? -1 : 1;
    tangent = (e1 * dv2 - e2 * dv1) * sign;
    bitangent = (e2 * du1 - e1 * du2) * sign;
    return nonzero(unit(tangent)) && nonzero(unit(bitangent));
}
const cr_texture_slot* slots(const cr_material& m, int k) {
    const cr_texture_slot* s[5] = {&m.base_color_texture, &m.metallic_roughness_texture, &m.normal_texture,
                                   &m.emissive_texture, &m.transmission_texture};
    return s[k];
}

}  // namespace

thread_local std::string g_lastError;

cr_status set_last_error(cr_status status, const std::string& message) {
    g_lastError = message;
    return status;
}
const std::string& last_error_text() { return g_lastError; }

namespace {
std::atomic<uint64_t> g_allocations{0};
std::atomic<int64_t> g_failCountdown{-1};  // allocations left before the injected failure; -1: none
}
void count_allocation() { g_allocations.fetch_add(1, std::memory_order_relaxed); }
uint64_t allocation_count() { return g_allocations.load(std::memory_order_relaxed); }
void inject_allocation_failure(int64_t nth) { g_failCountdown.store(nth < 0 ? -1 : nth, std::memory_order_relaxed); }
bool injected_allocation_failure() {
    int64_t v = g_failCountdown.load(std::memory_order_relaxed);
    while (v >= 0 && !g_failCountdown.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) {
    }
    return v == 0;
}

void validate_options(const cr_render_options& o) {
    if (o.width < 1 || o.height < 1 || o.width > 16384 || o.height > 16384)
        throw Error(CR_ERR_INVALID_ARGUMENT, "Width and height must be in [1, 16384]");
    const uint64_t pixels = static_cast<uint64_t>(o.width) * static_cast<uint64_t>(o.height);
    if (pixels > 67108864 || pixels > std::numeric_limits<std::size_t>::max() / (3 * sizeof(float)))
        throw Error(CR_ERR_INVALID_ARGUMENT, "Image exceeds the 64-megapixel allocation limit");
    if (o.samples < 1 || o.samples > 1048576) throw Error(CR_ERR_INVALID_ARGUMENT, "Samples must be in [1, 1048576]");
    if (o.bounces < 1 || o.bounces > 64) throw Error(CR_ERR_INVALID_ARGUMENT, "Bounces must be in [1, 64]");
    if (o.threads < 0 || o.threads > 256) throw Error(CR_ERR_INVALID_ARGUMENT, "Threads must be 0 (automatic) or in [1, 256]");
}

void finalize(std::vector<cr_triangle>& triangles, const cr_material* materials, uint32_t materialCount,
              const cr_image* images, uint32_t imageCount, const cr_texture* textures, uint32_t textureCount,
              std::vector<std::string>& warnings) {
    for (uint32_t i = 0; i < imageCount; ++i) {
        const cr_image& image = images[i];
        if (image.width <= 0 || image.height <= 0 || !image.pixels)
            throw Error(CR_ERR_INVALID_ARGUMENT, "Image " + std::to_string(i) + " has invalid dimensions or pixel count");
        const size_t n = static_cast<size_t>(image.width) * static_cast<size_t>(image.height);
        for (size_t p = 0; p < n; ++p)
            if (!finite4(image.pixels + 4 * p)) throw Error(CR_ERR_INVALID_ARGUMENT, "Image " + std::to_string(i) + " contains non-finite pixels");
    }
    for (uint32_t i = 0; i < textureCount; ++i) {
        const cr_texture& texture = textures[i];
        if (texture.image < 0 || static_cast<uint32_t>(texture.image) >= imageCount)
            throw Error(CR_ERR_INVALID_ARGUMENT, "Texture " + std::to_string(i) + " has an invalid image index");
        const auto validWrap = [](int32_t w) { return w == CR_WRAP_REPEAT || w == CR_WRAP_CLAMP || w == CR_WRAP_MIRROR; };
        if (!validWrap(texture.wrap_s) || !validWrap(texture.wrap_t))
            throw Error(CR_ERR_INVALID_ARGUMENT, "Texture " + std::to_string(i) + " has an invalid wrap mode");
    }
    for (uint32_t i = 0; i < materialCount; ++i) {
        const cr_material& m = materials[i];
        const std::string label = "Material " + std::to_string(i);
        const auto inUnit = [](float v) { return std::isfinite(v) && v >= 0 && v <= 1; };
        if (!finite4(m.base_color) || !inUnit(m.base_color[0]) || !inUnit(m.base_color[1]) || !inUnit(m.base_color[2]) ||
            !inUnit(m.base_color[3]) || !inUnit(m.metallic) || !inUnit(m.roughness) || !inUnit(m.transmission) ||
            !inUnit(m.alpha_cutoff) || !finite(v3(m.emission)) || m.emission[0] < 0 || m.emission[1] < 0 || m.emission[2] < 0 ||
            !std::isfinite(m.ior) || m.ior <= 0 || !std::isfinite(m.thickness) || m.thickness < 0 ||
            std::isnan(m.attenuation_distance) || m.attenuation_distance <= 0 ||
            !inUnit(m.attenuation_color[0]) || !inUnit(m.attenuation_color[1]) || !inUnit(m.attenuation_color[2]) ||
            !std::isfinite(m.normal_scale))
            throw Error(CR_ERR_INVALID_ARGUMENT, label + " has non-finite or out-of-range parameters");
        for (int k = 0; k < 5; ++k) {
            const cr_texture_slot* slot = slots(m, k);
            if (slot->texture < -1 || (slot->texture >= 0 && static_cast<uint32_t>(slot->texture) >= textureCount))
                throw Error(CR_ERR_INVALID_ARGUMENT, label + " has an invalid texture index");
            if (slot->texture >= 0 && (slot->texcoord < 0 || slot->texcoord > 1 || !finite2(slot->offset) ||
                                       !finite2(slot->scale) || !std::isfinite(slot->rotation)))
                throw Error(CR_ERR_INVALID_ARGUMENT, label + " has invalid texture coordinates or transform");
        }
        if (m.normal_texture.texture >= 0 && (m.normal_texture.scale[0] == 0 || m.normal_texture.scale[1] == 0))
            warnings.push_back(label + " has a singular normal-map UV transform; using the untransformed tangent frame");
    }
    for (size_t i = 0; i < triangles.size(); ++i) {
        const cr_triangle& t = triangles[i];
        if (t.material >= materialCount)
            throw Error(CR_ERR_INVALID_ARGUMENT, "Triangle " + std::to_string(i) + " has an invalid material index");
        for (const cr_vertex& v : t.v)
            if (!finite(v3(v.position)) || !finite(v3(v.normal)) || !finite4(v.tangent) || !finite2(v.uv[0]) || !finite2(v.uv[1]))
                throw Error(CR_ERR_INVALID_ARGUMENT, "Triangle " + std::to_string(i) + " contains non-finite vertex data");
    }
    size_t kept = 0, degenerate = 0, firstDegenerate = 0, generatedNormals = 0, fallbackTangents = 0;
    for (size_t i = 0; i < triangles.size(); ++i) {
        cr_triangle t = triangles[i];
        const DVec3 normal = preciseCross(DVec3(v3(t.v[1].position)) - DVec3(v3(t.v[0].position)),
                                          DVec3(v3(t.v[2].position)) - DVec3(v3(t.v[0].position)));
        const double twiceArea = std::sqrt(preciseDot(normal, normal));
        if (twiceArea * 0.5 > std::numeric_limits<float>::max())
            throw Error(CR_ERR_INVALID_ARGUMENT, "Triangle " + std::to_string(i) + " area exceeds the supported finite range");
        t.area = static_cast<float>(twiceArea * 0.5);
        if (!(t.area > 0)) {
            if (degenerate == 0) firstDegenerate = i;
            ++degenerate;
            continue;
        }
        const Vec3 gn = unit(normal);
        put(t.geometric_normal, gn);
        const cr_material& material = materials[t.material];
        const int uvSet = material.normal_texture.texture >= 0 ? material.normal_texture.texcoord : 0;
        DVec3 uvTangent{0, 0, 0}, uvBitangent{0, 0, 0};
        const bool usableUvs = uvDirections(t, uvSet, uvTangent, uvBitangent);
        for (cr_vertex& vertex : t.v) {
            Vec3 n = unit(v3(vertex.normal));
            float handedness = vertex.tangent[3] < 0 ? -1.0f : 1.0f;
            if (!nonzero(n) || dot(n, gn) == 0) {
                n = gn;
                ++generatedNormals;
            } else if (dot(n, gn) < 0) {
                n = -n;
                handedness = -handedness;
            }
            Vec3 tangent = orthogonalized(DVec3(Vec3{vertex.tangent[0], vertex.tangent[1], vertex.tangent[2]}), n);
            if (!nonzero(tangent)) {
                if (usableUvs) tangent = orthogonalized(uvTangent, n);
                if (nonzero(tangent)) {
                    handedness = preciseDot(DVec3(cross(n, tangent)), uvBitangent) < 0 ? -1.0f : 1.0f;
                } else {
                    tangent = Frame(n).x;
                    handedness = 1;
                    if (material.normal_texture.texture >= 0) ++fallbackTangents;
                }
            }
            put(vertex.normal, n);
            vertex.tangent[0] = tangent.x; vertex.tangent[1] = tangent.y; vertex.tangent[2] = tangent.z;
            vertex.tangent[3] = handedness;
        }
        triangles[kept] = t;
        ++kept;
    }
    triangles.resize(kept);
    if (degenerate) warnings.push_back("Skipped " + std::to_string(degenerate) + " degenerate triangles (first input triangle " + std::to_string(firstDegenerate) + ")");
    if (generatedNormals) warnings.push_back("Generated flat normals for " + std::to_string(generatedNormals) + " missing or tangential vertex normals");
    if (fallbackTangents) warnings.push_back("Used orthogonal fallback tangents for " + std::to_string(fallbackTangents) + " normal-mapped vertices with degenerate UVs");
}

void build_bvh(const cr_triangle* triangles, uint64_t count, std::vector<cr_bvh_node>& nodes, std::vector<uint32_t>& indices) {
    nodes.clear();
    indices.clear();
    if (count == 0) return;
    if (count > std::numeric_limits<uint32_t>::max() / 2)
        throw Error(CR_ERR_LENGTH, "Too many triangles for 32-bit BVH node indices");
    for (uint64_t i = 0; i < count; ++i)
        for (const cr_vertex& v : triangles[i].v)
            if (!finite(v3(v.position))) throw Error(CR_ERR_INVALID_ARGUMENT, "Cannot build BVH from non-finite geometry");
    indices.resize(count);
    std::iota(indices.begin(), indices.end(), uint32_t{0});
    nodes.reserve(2 * count);
    nodes.emplace_back();
    Builder b{triangles, nodes, indices, {}, {}};
    b.centroids.resize(count);
    b.boxes.resize(count);
    for (uint64_t i = 0; i < count; ++i) { b.centroids[i] = centroid(triangles[i]); b.boxes[i] = triangleBounds(triangles[i]); }
    b.subdivide(0, 0, static_cast<uint32_t>(count), 0);
}

void parallel_for(uint64_t n, const std::function<void(uint64_t, uint64_t)>& fn, uint64_t grain) {
    const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t parts = std::min<uint64_t>(hw, (n + grain - 1) / std::max<uint64_t>(1, grain));
    if (parts <= 1) { if (n) fn(0, n); return; }
    std::vector<std::thread> pool;
    pool.reserve(parts);
    for (uint64_t k = 0; k < parts; ++k) {
        const uint64_t b = n * k / parts, e = n * (k + 1) / parts;
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto& t : pool) t.join();
}

void build_environment(const cr_environment_desc& e, EnvTables& out, bool alias) {
    out = EnvTables{};
    if (!e.pixels) {  // Environment(Vec3) (render.cpp:12-14)
        const Vec3 c = v3(e.constant);
        if (!finite(c) || std::min({c.x, c.y, c.z}) < 0) throw Error(CR_ERR_INVALID_ARGUMENT, "Invalid environment radiance");
        put(out.constant, c);
        out.integral = 4 * pi * luminance(c);
        return;
    }
    if (e.width <= 0 || e.height <= 0) throw Error(CR_ERR_INVALID_ARGUMENT, "Invalid environment image dimensions");
    if (!std::isfinite(e.rotation_radians) || !std::isfinite(e.intensity) || e.intensity < 0)
        throw Error(CR_ERR_INVALID_ARGUMENT, "Invalid environment rotation/intensity");
    out.hasImage = true;
    out.width = e.width; out.height = e.height;
    out.rotation = e.rotation_radians; out.intensity = e.intensity;
    const int W = e.width, H = e.height;
    const size_t n = static_cast<size_t>(W) * static_cast<size_t>(H);
    auto solidAngle = [&](int row) {  // render.cpp:17-20
        const double a = static_cast<double>(pi) * row / H, b = static_cast<double>(pi) * (row + 1) / H;
        return (2 * static_cast<double>(pi) / W) * (std::cos(a) - std::cos(b));
    };
    std::vector<double> omegas(H);
    for (int y = 0; y < H; ++y) omegas[y] = solidAngle(y);
    // Texel weights in parallel; the running sums below stay sequential, in the reference's
    // order, so the CDF is bit-identical (render.cpp:29-41).
    std::unique_ptr<double[]> light(new double[n]);  // every entry is written below
    std::atomic<bool> bad{false};
    parallel_for(n, [&](uint64_t b, uint64_t en) {
        for (uint64_t i = b; i < en; ++i) {
            const float* p = e.pixels + 4 * i;
            const Vec3 color{p[0], p[1], p[2]};
            if (!finite(color) || std::min({p[0], p[1], p[2]}) < 0) bad = true;
            light[i] = luminance(color) * out.intensity;
        }
    });
    if (bad) throw Error(CR_ERR_INVALID_ARGUMENT, "Non-finite or negative HDR environment pixel");
    out.cdf.reserve(n);  // appended in order, without a zero fill first
    for (int y = 0; y < H; ++y) {
        const double omega = omegas[y];
        const size_t row = static_cast<size_t>(y) * W;
        for (int x = 0; x < W; ++x) {
            const double l = light[row + x];
            out.integral += l * omega;
            out.weightSum += (l + 1e-9) * omega;
            out.cdf.push_back(out.weightSum);
        }
    }
    if (e.cdf) {  // the caller's own copy of the same table
        for (size_t i = 0; i < n; ++i)
            if (e.cdf[i] != out.cdf[i]) throw Error(CR_ERR_INVALID_ARGUMENT, "Environment CDF does not match its image");
    }
    // Per-texel density as Environment::pdf/sample evaluate it (render.cpp:82, 93).
    out.pdf.resize(n);
    parallel_for(n, [&](uint64_t b, uint64_t en) {
        for (uint64_t i = b; i < en; ++i) {
            const int y = static_cast<int>(i / W);
            out.pdf[i] = static_cast<float>((out.cdf[i] - (i ? out.cdf[i - 1] : 0)) / (out.weightSum * omegas[y]));
        }
    });
    out.rowCos.resize(H + 1);
    for (int y = 0; y <= H; ++y) out.rowCos[y] = std::cos(pi * static_cast<float>(y) / static_cast<float>(H));
    // Bracket table: upper_bound of j*weightSum/K.
    uint32_t K = 1;
    while (K < n / 32 && K < (1u << 16)) K <<= 1;
    out.coarse.resize(K);
    parallel_for(K, [&](uint64_t b, uint64_t en) {
        for (uint64_t j = b; j < en; ++j) {
            const double pick = out.weightSum * (static_cast<double>(j) / K);
            out.coarse[j] = static_cast<uint32_t>(std::upper_bound(out.cdf.begin(), out.cdf.end(), pick) - out.cdf.begin());
        }
    }, 4096);
    if (alias) build_alias(out);
}

// Walker's alias method (Walker 1977) with Vose's construction (Vose 1991) over the texel
// probabilities of the CDF. The device draws a 48-bit uniform x (two 24-bit draws) and forms
// x*n = col*2^48 + r: col is the column, r the residual. The x of column c are the integers
// x0_c, x0_c+1, ... (count_c of them, x0_c = ceil(c*2^48/n)) and their residuals rise in steps
// of n from r0_c = x0_c*n - c*2^48, so "the first K_c of them take texel c, the rest its alias"
// is the test r < K_c*n + r0_c. With K_c = round(threshold_c * count_c) every texel's
// probability under the sampler is an exact integer count over 2^48; the density the sampler
// reports, for light samples and for the MIS weight of BSDF-sampled directions alike, is that
// probability over the texel's solid angle, so the estimator is unbiased however the
// thresholds rounded.
namespace {
constexpr int kAliasBits = 48;
struct AliasColumn {
    uint64_t count, r0;
};
AliasColumn alias_column(uint64_t c, uint64_t n) {
    using u128 = unsigned __int128;
    auto ceilDiv = [&](u128 a) { return static_cast<uint64_t>((a + n - 1) / n); };
    const u128 lo = static_cast<u128>(c) << kAliasBits, hi = static_cast<u128>(c + 1) << kAliasBits;
    const uint64_t x0 = ceilDiv(lo), x1 = ceilDiv(hi);
    return {x1 - x0, static_cast<uint64_t>(static_cast<u128>(x0) * n - lo)};
}
}  // namespace

std::vector<uint64_t> alias_masses(const EnvTables& t) {
    const uint64_t n = t.aliasThreshold.size();
    std::vector<uint64_t> mass(n, 0);
    for (uint64_t c = 0; c < n; ++c) {
        const AliasColumn col = alias_column(c, n);
        // K_c: how many of the column's x fall below its threshold
        const uint64_t T = t.aliasThreshold[c];
        const uint64_t own = T <= col.r0 ? 0 : std::min<uint64_t>(col.count, (T - col.r0 + n - 1) / n);
        mass[c] += own;
        mass[t.aliasIndex[c]] += col.count - own;
    }
    return mass;
}

void build_alias(EnvTables& out) {
    if (!out.hasImage || !out.aliasThreshold.empty()) return;
    const uint64_t n = out.cdf.size();
    std::vector<double> threshold(n, 1.0), scaled(n);
    out.aliasIndex.resize(n);
    std::vector<uint32_t> small, large;
    for (uint64_t i = 0; i < n; ++i) {
        scaled[i] = (out.cdf[i] - (i ? out.cdf[i - 1] : 0)) / out.weightSum * static_cast<double>(n);
        out.aliasIndex[i] = static_cast<uint32_t>(i);
        (scaled[i] < 1.0 ? small : large).push_back(static_cast<uint32_t>(i));
    }
    while (!small.empty() && !large.empty()) {
        const uint32_t sm = small.back(); small.pop_back();
        const uint32_t l = large.back();
        threshold[sm] = scaled[sm];
        out.aliasIndex[sm] = l;
        scaled[l] = (scaled[l] + scaled[sm]) - 1.0;
        if (scaled[l] < 1.0) { large.pop_back(); small.push_back(l); }
    }
    // columns left on either list keep threshold 1 (rounding leftovers: their own texel)
    out.aliasThreshold.resize(n);
    for (uint64_t c = 0; c < n; ++c) {
        const AliasColumn col = alias_column(c, n);
        const double k = std::nearbyint(std::min(1.0, std::max(0.0, threshold[c])) * static_cast<double>(col.count));
        const uint64_t K = std::min<uint64_t>(col.count, static_cast<uint64_t>(k));
        out.aliasThreshold[c] = K * n + col.r0;
    }
    const std::vector<uint64_t> mass = alias_masses(out);
    out.aliasPdf.resize(n);
    const int W = out.width, H = out.height;
    for (uint64_t i = 0; i < n; ++i) {
        const int y = static_cast<int>(i / static_cast<uint64_t>(W));
        const double a = static_cast<double>(pi) * y / H, b = static_cast<double>(pi) * (y + 1) / H;
        const double omega = (2 * static_cast<double>(pi) / W) * (std::cos(a) - std::cos(b));
        out.aliasPdf[i] = static_cast<float>(std::ldexp(static_cast<double>(mass[i]), -kAliasBits) / omega);
    }
}

LightScan scan_lights(const cr_triangle* triangles, uint64_t count, const cr_material* materials) {
    // The scene box and the emitters' weights in parallel: positions are finite after
    // finalize, so min/max in any order give the same box; the weights go into per-part lists
    // that build_lights reads in triangle order, so its running total is summed in the
    // reference's order.
    constexpr uint64_t kParts = 64;
    LightScan scan;
    scan.count = count;
    std::vector<Bounds> partBox(kParts);
    scan.emitters.resize(kParts);
    parallel_for(kParts, [&](uint64_t pb, uint64_t pe) {
        for (uint64_t part = pb; part < pe; ++part) {
            const uint64_t b = count * part / kParts, e = count * (part + 1) / kParts;
            Bounds local;
            for (uint64_t i = b; i < e; ++i) {
                const cr_triangle& t = triangles[i];
                local.expand(triangleBounds(t));
                const cr_material& m = materials[t.material];
                const double w = static_cast<double>(t.area) * pi * luminance(v3(m.emission)) * (m.double_sided ? 2 : 1);
                if (w > 0) scan.emitters[part].push_back({static_cast<uint32_t>(i), w});
            }
            partBox[part] = local;
        }
    }, 1);
    Bounds box;
    for (const Bounds& b : partBox) box.expand(b);
    scan.radius2 = count == 0 ? 1 : std::max(1.0, static_cast<double>(lengthSquared(box.hi - box.lo)) * 0.25);
    return scan;
}

void build_lights(const cr_triangle* triangles, uint64_t count, const cr_material* materials,
                  const cr_punctual_light* lights, uint32_t lightCount, double envIntegral, LightTables& out) {
    build_lights(scan_lights(triangles, count, materials), lights, lightCount, envIntegral, out);
}

void build_lights(const LightScan& scan, const cr_punctual_light* lights, uint32_t lightCount, double envIntegral,
                  LightTables& out) {
    out = LightTables{};
    out.triangleProbability.assign(scan.count, 0.0f);
    const double radius2 = scan.radius2;
    double total = 0;
    auto add = [&](uint32_t type, uint32_t index, double weight) {
        if (weight > 0) { total += weight; out.entries.push_back({total, type, index, 0.0f, 0u}); }
    };
    for (uint32_t i = 0; i < lightCount; ++i) {
        const cr_punctual_light& l = lights[i];
        add(crg::kLightPunctual, i, static_cast<double>(luminance(v3(l.color))) * l.intensity *
                                        (l.type == CR_LIGHT_DIRECTIONAL ? pi * radius2 : 4 * pi));
    }
    for (const auto& part : scan.emitters)
        for (const auto& [index, weight] : part) add(crg::kLightTriangle, index, weight);
    add(crg::kLightEnvironment, 0, envIntegral * pi * radius2);
    double last = 0, cumulative = 0;
    for (auto& e : out.entries) {
        const double probability = 0.95 * (e.cdf - last) / total + 0.05 / static_cast<double>(out.entries.size());
        last = e.cdf;
        cumulative += probability;
        e.probability = static_cast<float>(probability);
        e.cdf = cumulative;
        if (e.type == crg::kLightTriangle) out.triangleProbability[e.index] = e.probability;
        if (e.type == crg::kLightEnvironment) out.environmentProbability = e.probability;
    }
    if (!out.entries.empty()) out.entries.back().cdf = 1;
}

void camera_setup(const cr_camera& c, int width, int height, crg::DevCamera& out) {
    const Vec3 position = v3(c.position), forward = v3(c.forward), right = v3(c.right), up = v3(c.up);
    if (width <= 0 || height <= 0 || !finite(position) || !finite(forward) || !finite(right) || !finite(up) ||
        !std::isfinite(c.yfov) || c.yfov <= 0 || c.yfov >= pi || !std::isfinite(c.aspect) || c.aspect < 0 ||
        !std::isfinite(c.near_clip) || c.near_clip < 0 || std::isnan(c.far_clip) || c.far_clip <= c.near_clip)
        throw Error(CR_ERR_INVALID_ARGUMENT, "Invalid perspective camera or image dimensions");
    const Vec3 f = unit(forward);
    const Vec3 r = orthogonalized(DVec3(right), f);
    const Vec3 u = orthogonalized(DVec3(orthogonalized(DVec3(up), f)), r);
    if (!nonzero(f) || !nonzero(r) || !nonzero(u)) throw Error(CR_ERR_INVALID_ARGUMENT, "Degenerate camera basis");
    put(out.position, position);
    put(out.f, f); put(out.r, r); put(out.u, u);
    out.ratio = c.aspect > 0 ? c.aspect : static_cast<double>(width) / height;
    out.halfHeight = std::tan(static_cast<double>(c.yfov) * 0.5);
    out.nearClip = c.near_clip;
    out.farClip = c.far_clip;
}

std::string sample_error_message(const crg::DevError& e) {
    std::string cause;
    switch (e.code) {
        case crg::kErrNonFiniteThroughput: cause = "Non-finite path throughput"; break;
        case crg::kErrNonFiniteRadiance: cause = "Non-finite or negative path radiance"; break;
        case crg::kErrNestedVolume: cause = "Nested/intersecting refractive volumes are unsupported; separate the closed meshes"; break;
        case crg::kErrExitWithoutEntry: {
            std::ostringstream detail;
            detail.precision(9);
            detail << "Refractive exit without entry; check outward normals and keep the camera outside closed volumes"
                   << "; bounce " << e.depth << ", triangle " << e.triangle << ", material " << e.material
                   << ", t " << e.t << ", point (" << e.point[0] << ',' << e.point[1] << ',' << e.point[2]
                   << "), origin (" << e.origin[0] << ',' << e.origin[1] << ',' << e.origin[2]
                   << "), direction (" << e.direction[0] << ',' << e.direction[1] << ',' << e.direction[2] << ')';
            cause = detail.str();
            break;
        }
        case crg::kErrInvalidSecondaryRay: cause = "Invalid secondary ray"; break;
        case crg::kErrOffsetOverflow: cause = "Secondary ray offset exceeds finite coordinates"; break;
        case crg::kErrUnrepresentableCameraRay: cause = "Unrepresentable perspective ray"; break;
        case crg::kErrStackOverflow: cause = "BVH traversal exceeded its bounded stack"; break;
        case crg::kErrInvalidSurfaceHit: cause = "Invalid surface hit"; break;
        case crg::kErrTextureCoordinates: cause = "Non-finite texture coordinates or transform"; break;
        default: cause = "Unknown device failure " + std::to_string(e.code); break;
    }
    return "Pixel (" + std::to_string(e.x) + "," + std::to_string(e.y) + "), sample " + std::to_string(e.sample) + ": " + cause;
}

// ---- output encoding --------------------------------------------------------------------------

void check_image_dims(int width, int height, const std::string& label) {
    constexpr int maxDimension = 16384;
    constexpr uint64_t maxPixels = 16777216;
    if (width <= 0 || height <= 0 || width > maxDimension || height > maxDimension ||
        static_cast<uint64_t>(width) > maxPixels / static_cast<uint64_t>(height))
        throw Error(CR_ERR_INVALID_ARGUMENT,
                    label + ": image dimensions must be positive, at most 16384 per axis and 16777216 pixels");
}

namespace {
float linear_to_srgb(float v) {  // math.h:62
    return v <= 0.0031308f ? 12.92f * v : 1.055f * std::pow(v, 1 / 2.4f) - 0.055f;
}
}  // namespace

unsigned char display_channel(float value, double exposureScale) {  // image.cpp:119-124
    const double x = static_cast<double>(value) * exposureScale;
    const double filmic = std::clamp((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0);
    const float srgb = linear_to_srgb(static_cast<float>(filmic));
    return static_cast<unsigned char>(std::lround(std::clamp(srgb, 0.0f, 1.0f) * 255.0f));
}

void display_thresholds(float exposure, float out[256]) {
    if (!std::isfinite(exposure) || exposure < -100 || exposure > 100)  // image.cpp:196-197
        throw Error(CR_ERR_INVALID_ARGUMENT, "PNG exposure must be finite and between -100 and 100 stops");
    const double scale = std::exp2(static_cast<double>(exposure));
    constexpr uint32_t finiteEnd = 0x7f800000u;  // bit pattern of +inf; non-negative floats sort by bits
    auto at = [&](uint32_t bits) { float f; std::memcpy(&f, &bits, 4); return display_channel(f, scale); };
    const unsigned char top = at(finiteEnd - 1);
    out[0] = 0.0f;
    for (int k = 1; k < 256; ++k) {
        if (top < k) { out[k] = std::numeric_limits<float>::infinity(); continue; }
        uint32_t lo = 0, hi = finiteEnd - 1;  // invariant: at(hi) >= k
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (at(mid) >= k) hi = mid; else lo = mid + 1;
        }
        std::memcpy(&out[k], &hi, 4);
    }
}

std::string hdr_header(int width, int height) {  // stb_image_write.h 1.16, stbi_write_hdr_core
    return "#?RADIANCE\n# Written by stb_image_write.h\nFORMAT=32-bit_rle_rgbe\n"
           "EXPOSURE=          1.0000000000000\n\n-Y " + std::to_string(height) + " +X " + std::to_string(width) + "\n";
}

}  // namespace crh

// ---- C ABI entry points that need no GPU -------------------------------------------------------
extern "C" {

int cr_gpu_abi_version(void) { return CR_GPU_ABI_VERSION; }

size_t cr_gpu_last_error(char* buf, size_t n) {
    const std::string& s = crh::g_lastError;
    if (buf && n) {
        const size_t k = std::min(n - 1, s.size());
        std::memcpy(buf, s.data(), k);
        buf[k] = 0;
    }
    return s.size();
}

cr_status cr_options_validate(const cr_render_options* options) {
    try {
        if (!options) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "options is NULL");
        crh::validate_options(*options);
        return CR_OK;
    } catch (const crh::Error& e) { return crh::set_last_error(e.status, e.what()); }
}

cr_status cr_scene_finalize(cr_triangle* triangles, uint64_t* triangle_count, const cr_material* materials,
                            uint32_t material_count, const cr_image* images, uint32_t image_count,
                            const cr_texture* textures, uint32_t texture_count, char* warnings, size_t warnings_size) {
    try {
        if (!triangle_count || (*triangle_count && !triangles)) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "triangles is NULL");
        std::vector<cr_triangle> tris(triangles, triangles + *triangle_count);
        std::vector<std::string> w;
        crh::finalize(tris, materials, material_count, images, image_count, textures, texture_count, w);
        if (!tris.empty()) std::memcpy(triangles, tris.data(), tris.size() * sizeof(cr_triangle));
        *triangle_count = tris.size();
        if (warnings && warnings_size) {
            std::string joined;
            for (const auto& s : w) { if (!joined.empty()) joined += '\n'; joined += s; }
            const size_t k = std::min(warnings_size - 1, joined.size());
            std::memcpy(warnings, joined.data(), k);
            warnings[k] = 0;
        }
        return CR_OK;
    } catch (const crh::Error& e) { return crh::set_last_error(e.status, e.what()); }
    catch (const std::bad_alloc&) { return crh::set_last_error(CR_ERR_OUT_OF_MEMORY, "host allocation failed"); }
}

cr_status cr_bvh_build(const cr_triangle* triangles, uint64_t triangle_count, cr_bvh_node* nodes,
                       uint64_t* node_count, uint32_t* indices) {
    try {
        std::vector<cr_bvh_node> n;
        std::vector<uint32_t> idx;
        crh::build_bvh(triangles, triangle_count, n, idx);
        if (!n.empty()) std::memcpy(nodes, n.data(), n.size() * sizeof(cr_bvh_node));
        if (!idx.empty()) std::memcpy(indices, idx.data(), idx.size() * sizeof(uint32_t));
        if (node_count) *node_count = n.size();
        return CR_OK;
    } catch (const crh::Error& e) { return crh::set_last_error(e.status, e.what()); }
    catch (const std::bad_alloc&) { return crh::set_last_error(CR_ERR_OUT_OF_MEMORY, "host allocation failed"); }
}

float cr_environment_rotation(float degrees) {  // render.cpp:24
    constexpr float pi = 3.14159265358979323846f;
    return std::fmod(degrees, 360.0f) * pi / 180;
}

cr_status cr_environment_tables(const cr_environment_desc* environment, double* cdf, double* weight_sum_integral) {
    try {
        if (!environment) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "environment is NULL");
        crh::EnvTables t;
        crh::build_environment(*environment, t);
        if (cdf && !t.cdf.empty()) std::memcpy(cdf, t.cdf.data(), t.cdf.size() * sizeof(double));
        if (weight_sum_integral) { weight_sum_integral[0] = t.weightSum; weight_sum_integral[1] = t.integral; }
        return CR_OK;
    } catch (const crh::Error& e) { return crh::set_last_error(e.status, e.what()); }
    catch (const std::bad_alloc&) { return crh::set_last_error(CR_ERR_OUT_OF_MEMORY, "host allocation failed"); }
}

cr_status cr_display_thresholds(float exposure, float* out256) {
    try {
        if (!out256) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        crh::display_thresholds(exposure, out256);
        return CR_OK;
    } catch (const crh::Error& e) {
        return crh::set_last_error(e.status, e.what());
    }
}

}  // extern "C"
