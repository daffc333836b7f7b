// CPU restatement of CPU-Renderer's per-path radiance loop — TEST INFRASTRUCTURE ONLY.
//
// This is the oracle: a scalar C++ restatement of the reference's algorithm, written for
// this repository and pinned against the reference compiled from its own sources
// (oracle/_ref, tests/test_oracle.py) and against the committed golden fixtures. Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product
// (libcr_b200.so) never links or calls it.
//
// Each function cites the reference lines it restates. Arithmetic follows the reference's
// expressions and association order; built with the reference's Release flags it rounds
// identically (so renders are bit-identical to the reference's, which the tests check).
// The BVH is taken from the caller (the node and index arrays of Bvh::build); closest hits
// can also be computed by brute force over all triangles (test_geometry.cpp:396-407).
#include "cr_gpu.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace oracle {
namespace {

constexpr float pi = 3.14159265358979323846f;          // math.h:13
constexpr float inf = std::numeric_limits<float>::infinity();
constexpr uint32_t noTriangle = std::numeric_limits<uint32_t>::max();

// ---- math.h ---------------------------------------------------------------------------------
struct V3 {
    float x = 0, y = 0, z = 0;
    V3() = default;
    explicit V3(float s) : x(s), y(s), z(s) {}
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
V3 operator*(V3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
V3 operator*(float a, V3 b) { return b * a; }
V3 operator/(V3 a, float b) { return a * (1.0f / b); }
V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
V3& operator*=(V3& a, V3 b) { a = a * b; return a; }
V3& operator*=(V3& a, float b) { a = a * b; return a; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float lengthSquared(V3 a) { return dot(a, a); }
float length(V3 a) { return std::sqrt(lengthSquared(a)); }
V3 normalize(V3 a) { const float l = length(a); return l > 0 ? a / l : V3{}; }
bool finite(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
V3 clamp(V3 a, float lo, float hi) { return {std::clamp(a.x, lo, hi), std::clamp(a.y, lo, hi), std::clamp(a.z, lo, hi)}; }
float maxComponent(V3 a) { return std::max({a.x, a.y, a.z}); }
float luminance(V3 a) { return dot(a, {0.2126f, 0.7152f, 0.0722f}); }
V3 mix(V3 a, V3 b, float t) { return a * (1 - t) + b * t; }
V3 vexp(V3 a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
V3 reflect(V3 i, V3 n) { return i - 2 * dot(i, n) * n; }
float srgbToLinear(float v) { return v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f); }
V3 v3(const float* p) { return {p[0], p[1], p[2]}; }
bool nonzero(V3 v) { return v.x != 0 || v.y != 0 || v.z != 0; }

struct Frame {  // math.h:95-103
    V3 x, y, z;
    explicit Frame(V3 n) : z(n) { x = normalize(cross(std::abs(z.z) < 0.999f ? V3{0, 0, 1} : V3{0, 1, 0}, z)); y = cross(z, x); }
    V3 local(V3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    V3 world(V3 v) const { return x * v.x + y * v.y + z * v.z; }
};
struct Rng {  // math.h:106-116
    uint64_t state;
    explicit Rng(uint64_t s) : state(s) {}
    uint32_t next() {
        state += 0x9e3779b97f4a7c15ULL;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return static_cast<uint32_t>((z ^ (z >> 31)) >> 32);
    }
    float uniform() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
};
uint64_t sampleSeed(uint64_t seed, uint64_t pixel, uint64_t sample) {  // math.h:118-121
    Rng h(seed ^ (pixel * 0xd2b74407b1ce6e93ULL) ^ (sample * 0xca5a826395121157ULL));
    const uint64_t hi = h.next();
    return (hi << 32) | h.next();
}
float powerHeuristic(float a, float b) {  // math.h:124-128
    if (a <= 0) return 0;
    const double aa = static_cast<double>(a) * a, bb = static_cast<double>(b) * b;
    return static_cast<float>(aa / (aa + bb));
}

// ---- geometry.cpp helpers (17-47) --------------------------------------------------------------
struct D3 {
    double x, y, z;
    explicit D3(V3 v) : x(v.x), y(v.y), z(v.z) {}
    D3(double a, double b, double c) : x(a), y(b), z(c) {}
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 operator*(D3 a, double b) { return {a.x * b, a.y * b, a.z * b}; }
double pdot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
D3 pcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 unit(D3 v, V3 fb = {}) {
    const double sq = pdot(v, v);
    if (!(sq > 0) || !std::isfinite(sq)) return fb;
    const double inv = 1 / std::sqrt(sq);
    return {static_cast<float>(v.x * inv), static_cast<float>(v.y * inv), static_cast<float>(v.z * inv)};
}
V3 unit(V3 v, V3 fb = {}) { return unit(D3(v), fb); }
V3 orthogonalized(D3 v, V3 n, V3 fb = {}) {
    const double ns = pdot(D3(n), D3(n));
    if (!(ns > 0)) return fb;
    const D3 p = v - D3(n) * (pdot(v, D3(n)) / ns);
    constexpr double tol = 4 * std::numeric_limits<float>::epsilon();
    if (pdot(p, p) <= pdot(v, v) * tol * tol) return fb;
    return unit(p, fb);
}

struct Ray { V3 o, d; float tmin = 0, tmax = inf; V3 lo{}; };
struct Hit { double t = inf, u = 0, v = 0; uint32_t tri = 0; };

struct Failure : std::runtime_error {
    bool boundary;
    Failure(const std::string& m, bool b = false) : std::runtime_error(m), boundary(b) {}
};

bool validRay(const Ray& r) {  // geometry.cpp:52-55
    return finite(r.o) && finite(r.lo) && finite(r.d) && nonzero(r.d) && !std::isnan(r.tmin) && !std::isnan(r.tmax) && r.tmin <= r.tmax;
}

// ---- scene ----------------------------------------------------------------------------------------
struct Image { int w = 0, h = 0; std::vector<float> px; };
struct Env {
    bool image = false;
    V3 constant{};
    int w = 0, h = 0;
    std::vector<float> px;
    float rotation = 0, intensity = 1;
    double integral = 0, weightSum = 0;
    std::vector<double> cdf;
};
struct LightEntry { int type; uint32_t index; double cdf; float probability; };
struct Scene {
    std::vector<cr_triangle> tris;
    std::vector<cr_material> mats;
    std::vector<cr_punctual_light> lights;
    std::vector<Image> images;
    std::vector<cr_texture> textures;
    std::vector<cr_bvh_node> nodes;
    std::vector<uint32_t> indices;
    bool brute = false;
    Env env;
    // Lights (render.cpp:120-160)
    std::vector<LightEntry> entries;
    std::vector<float> triProb;
    float envProb = 0;
};

// Environment (render.cpp:12-94)
double solidAngle(const Env& e, int row) {
    const double a = static_cast<double>(pi) * row / e.h, b = static_cast<double>(pi) * (row + 1) / e.h;
    return (2 * static_cast<double>(pi) / e.w) * (std::cos(a) - std::cos(b));
}
void buildEnv(Env& e) {
    if (!e.image) { e.integral = 4 * pi * luminance(e.constant); return; }
    e.cdf.reserve(static_cast<size_t>(e.w) * e.h);
    for (int y = 0; y < e.h; ++y) {
        const double omega = solidAngle(e, y);
        for (int x = 0; x < e.w; ++x) {
            const float* p = &e.px[4 * (static_cast<size_t>(y) * e.w + x)];
            const double light = luminance(V3{p[0], p[1], p[2]}) * e.intensity;
            e.integral += light * omega;
            e.weightSum += (light + 1e-9) * omega;
            e.cdf.push_back(e.weightSum);
        }
    }
}
float envU(const Env& e, V3 d, float& v) {
    float u = (std::atan2(d.z, d.x) - e.rotation) / (2 * pi) + 0.5f;
    u -= std::floor(u);
    v = std::acos(std::clamp(d.y, -1.0f, 1.0f)) / pi;
    return u;
}
V3 envRadiance(const Env& e, V3 d) {
    if (!e.image) return e.constant;
    float cv;
    const float cu = envU(e, d, cv);
    const float px = cu * static_cast<float>(e.w) - 0.5f, py = cv * static_cast<float>(e.h) - 0.5f;
    const int x = static_cast<int>(std::floor(px)), y = static_cast<int>(std::floor(py));
    const float tx = px - static_cast<float>(x), ty = py - static_cast<float>(y);
    auto texel = [&](int ix, int iy) {
        ix = (ix % e.w + e.w) % e.w;
        iy = std::clamp(iy, 0, e.h - 1);
        const float* p = &e.px[4 * (static_cast<size_t>(iy) * e.w + ix)];
        return V3{p[0], p[1], p[2]};
    };
    return mix(mix(texel(x, y), texel(x + 1, y), tx), mix(texel(x, y + 1), texel(x + 1, y + 1), tx), ty) * e.intensity;
}
V3 envSample(const Env& e, Rng& rng, float& density) {
    if (!e.image) {
        const float y = 1 - 2 * rng.uniform(), phi = 2 * pi * rng.uniform(), r = std::sqrt(std::max(0.0f, 1 - y * y));
        density = 1 / (4 * pi);
        return {r * std::cos(phi), y, r * std::sin(phi)};
    }
    const double pick = rng.uniform() * e.weightSum;
    auto it = std::upper_bound(e.cdf.begin(), e.cdf.end(), pick);
    const size_t index = std::min(static_cast<size_t>(it - e.cdf.begin()), e.cdf.size() - 1);
    const int x = static_cast<int>(index % e.w), y = static_cast<int>(index / e.w);
    const float u = (static_cast<float>(x) + rng.uniform()) / static_cast<float>(e.w);
    const float c0 = std::cos(pi * static_cast<float>(y) / static_cast<float>(e.h));
    const float c1 = std::cos(pi * static_cast<float>(y + 1) / static_cast<float>(e.h));
    const float cosT = c0 + (c1 - c0) * rng.uniform(), sinT = std::sqrt(std::max(0.0f, 1 - cosT * cosT));
    const float phi = (u - 0.5f) * 2 * pi + e.rotation;
    density = static_cast<float>((e.cdf[index] - (index ? e.cdf[index - 1] : 0)) / (e.weightSum * solidAngle(e, y)));
    return {sinT * std::cos(phi), cosT, sinT * std::sin(phi)};
}
float envPdf(const Env& e, V3 d) {
    if (!e.image) return 1 / (4 * pi);
    float cv;
    const float cu = envU(e, d, cv);
    const int x = std::min(static_cast<int>(cu * static_cast<float>(e.w)), e.w - 1);
    const int y = std::min(static_cast<int>(cv * static_cast<float>(e.h)), e.h - 1);
    const size_t index = static_cast<size_t>(y) * e.w + x;
    return static_cast<float>((e.cdf[index] - (index ? e.cdf[index - 1] : 0)) / (e.weightSum * solidAngle(e, y)));
}

// Texture sampler (geometry.cpp:68-98, 238-275)
double wrapC(double v, int w) {
    if (w == CR_WRAP_CLAMP) return std::clamp(v, 0.0, 1.0);
    if (w == CR_WRAP_REPEAT) return v - std::floor(v);
    double r = std::fmod(v, 2.0);
    if (r < 0) r += 2;
    return r <= 1 ? r : 2 - r;
}
int wrapI(int64_t i, int size, int w) {
    const int64_t n = size;
    if (w == CR_WRAP_CLAMP) return static_cast<int>(std::clamp(i, int64_t{0}, n - 1));
    const int64_t period = w == CR_WRAP_MIRROR ? 2 * n : n;
    i %= period;
    if (i < 0) i += period;
    if (w == CR_WRAP_MIRROR && i >= n) i = period - 1 - i;
    return static_cast<int>(i);
}
struct F4 { float x = 1, y = 1, z = 1, w = 1; };
F4 interp(F4 a, F4 b, float t) { return {a.x * (1 - t) + b.x * t, a.y * (1 - t) + b.y * t, a.z * (1 - t) + b.z * t, a.w * (1 - t) + b.w * t}; }
F4 sampleTex(const Scene& S, const cr_texture_slot& slot, float u0x, float u0y, float u1x, float u1y, bool srgb) {
    if (slot.texture == -1) return {};
    const cr_texture& tex = S.textures[slot.texture];
    const Image& im = S.images[tex.image];
    const float ux = slot.texcoord == 0 ? u0x : u1x, uy = slot.texcoord == 0 ? u0y : u1y;
    if (!std::isfinite(ux) || !std::isfinite(uy)) throw Failure("Non-finite texture coordinates or transform");
    const double c = std::cos(static_cast<double>(slot.rotation)), s = std::sin(static_cast<double>(slot.rotation));
    const double x = static_cast<double>(ux) * slot.scale[0], y = static_cast<double>(uy) * slot.scale[1];
    const double u = wrapC(c * x - s * y + slot.offset[0], tex.wrap_s);
    const double v = wrapC(s * x + c * y + slot.offset[1], tex.wrap_t);
    auto texel = [&](int64_t ix, int64_t iy) {
        const int tx = wrapI(ix, im.w, tex.wrap_s), ty = wrapI(iy, im.h, tex.wrap_t);
        const float* p = &im.px[4 * (static_cast<size_t>(ty) * im.w + tx)];
        F4 val{p[0], p[1], p[2], p[3]};
        if (srgb) { val.x = srgbToLinear(val.x); val.y = srgbToLinear(val.y); val.z = srgbToLinear(val.z); }
        return val;
    };
    if (!tex.linear) return texel(static_cast<int64_t>(std::floor(u * im.w)), static_cast<int64_t>(std::floor(v * im.h)));
    const double px = u * im.w - 0.5, py = v * im.h - 0.5;
    const int64_t ix = static_cast<int64_t>(std::floor(px)), iy = static_cast<int64_t>(std::floor(py));
    const float fx = static_cast<float>(px - std::floor(px)), fy = static_cast<float>(py - std::floor(py));
    return interp(interp(texel(ix, iy), texel(ix + 1, iy), fx), interp(texel(ix, iy + 1), texel(ix + 1, iy + 1), fx), fy);
}
void interpUv(const cr_triangle& t, double hu, double hv, int set, float& ox, float& oy) {
    const double w = 1.0 - hu - hv;
    ox = static_cast<float>(w * t.v[0].uv[set][0] + hu * t.v[1].uv[set][0] + hv * t.v[2].uv[set][0]);
    oy = static_cast<float>(w * t.v[0].uv[set][1] + hu * t.v[1].uv[set][1] + hv * t.v[2].uv[set][1]);
}

// Scene::accepts (geometry.cpp:279-292)
bool accepts(const Scene& S, const cr_triangle& t, const Ray& r, double hu, double hv) {
    const cr_material& m = S.mats[t.material];
    if (!m.double_sided && m.transmission <= 0) {
        V3 n = v3(t.geometric_normal);
        if (!nonzero(n)) n = unit(pcross(D3(v3(t.v[1].position)) - D3(v3(t.v[0].position)), D3(v3(t.v[2].position)) - D3(v3(t.v[0].position))));
        if (pdot(D3(n), D3(r.d)) >= 0) return false;
    }
    if (m.alpha_mode == CR_ALPHA_MASK) {
        float a, b, c, d;
        interpUv(t, hu, hv, 0, a, b);
        interpUv(t, hu, hv, 1, c, d);
        return m.base_color[3] * sampleTex(S, m.base_color_texture, a, b, c, d, false).w >= m.alpha_cutoff;
    }
    return true;
}

// intersectTriangle (geometry.cpp:147-182)
bool intersectTriangle(const cr_triangle& tri, const Ray& ray, Hit& hit) {
    if (!validRay(ray) || std::isnan(hit.t)) return false;
    const double limit = std::min(static_cast<double>(ray.tmax), hit.t);
    if (limit < ray.tmin) return false;
    int kz = 0;
    if (std::abs(ray.d.y) > std::abs(ray.d[kz])) kz = 1;
    if (std::abs(ray.d.z) > std::abs(ray.d[kz])) kz = 2;
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (ray.d[kz] < 0) std::swap(kx, ky);
    const double sx = static_cast<double>(ray.d[kx]) / ray.d[kz], sy = static_cast<double>(ray.d[ky]) / ray.d[kz], sz = 1.0 / ray.d[kz];
    const D3 o = D3(ray.o) + D3(ray.lo);
    const D3 a = D3(v3(tri.v[0].position)) - o, b = D3(v3(tri.v[1].position)) - o, c = D3(v3(tri.v[2].position)) - o;
    const double ax = a[kx] - sx * a[kz], ay = a[ky] - sy * a[kz];
    const double bx = b[kx] - sx * b[kz], by = b[ky] - sy * b[kz];
    const double cx = c[kx] - sx * c[kz], cy = c[ky] - sy * c[kz];
    const double w0 = cx * by - cy * bx, w1 = ax * cy - ay * cx, w2 = bx * ay - by * ax;
    if ((w0 < 0 || w1 < 0 || w2 < 0) && (w0 > 0 || w1 > 0 || w2 > 0)) return false;
    const double det = w0 + w1 + w2;
    if (det == 0 || !std::isfinite(det)) return false;
    const double t = (w0 * (sz * a[kz]) + w1 * (sz * b[kz]) + w2 * (sz * c[kz])) / det;
    if (!std::isfinite(t) || std::abs(t) > std::numeric_limits<float>::max() || t < ray.tmin || t > limit) return false;
    hit.t = t; hit.u = w1 / det; hit.v = w2 / det;
    return true;
}

// Bvh::intersect (geometry.cpp:554-639) over the caller's node/index arrays, or the brute
// force oracle of test_geometry.cpp:396-407.
bool intersect(const Scene& S, const Ray& ray, Hit& hit, bool any, uint32_t ignore = noTriangle) {
    if (S.brute) {
        if (!validRay(ray) || std::isnan(hit.t)) return false;
        bool found = false;
        const double upper = hit.t;
        for (uint32_t i = 0; i < S.tris.size(); ++i) {
            if (i == ignore) continue;
            Hit c; c.t = upper; c.tri = i;
            if (!intersectTriangle(S.tris[i], ray, c) || !accepts(S, S.tris[i], ray, c.u, c.v)) continue;
            if (any) { hit = c; return true; }
            if (!found || c.t < hit.t || (c.t == hit.t && i < hit.tri)) { found = true; hit = c; }
        }
        return found;
    }
    if (S.nodes.empty() || !validRay(ray) || std::isnan(hit.t)) return false;
    Ray clipped = ray;
    double closest = std::min(static_cast<double>(ray.tmax), hit.t);
    clipped.tmax = std::min(clipped.tmax, std::nextafter(static_cast<float>(closest), inf));
    const float query = clipped.tmax;
    if (query < ray.tmin) return false;
    double inverse[3] = {0, 0, 0};
    const D3 po = D3(ray.o) + D3(ray.lo);
    for (int a = 0; a < 3; ++a) if (ray.d[a] != 0) inverse[a] = 1.0 / ray.d[a];
    auto box = [&](const cr_bvh_node& n, float& nearD) {
        double nearT = clipped.tmin, farT = clipped.tmax;
        for (int a = 0; a < 3; ++a) {
            const double origin = po[a];
            if (ray.d[a] == 0) { if (origin < n.lo[a] || origin > n.hi[a]) return false; continue; }
            double lo = (static_cast<double>(n.lo[a]) - origin) * inverse[a];
            double hi = (static_cast<double>(n.hi[a]) - origin) * inverse[a];
            if (inverse[a] < 0) std::swap(lo, hi);
            constexpr double err = 4 * std::numeric_limits<double>::epsilon();
            lo -= std::abs(lo) * err; hi += std::abs(hi) * err;
            nearT = std::max(nearT, lo); farT = std::min(farT, hi);
            if (nearT > farT) return false;
        }
        nearD = std::max(clipped.tmin, std::nextafter(static_cast<float>(nearT), -inf));
        return true;
    };
    float rootNear = 0;
    if (!box(S.nodes[0], rootNear)) return false;
    struct Entry { uint32_t node; float nearD; };
    Entry stack[50];
    size_t size = 0;
    stack[size++] = {0, rootNear};
    bool found = false;
    while (size) {
        const Entry e = stack[--size];
        if (e.nearD > clipped.tmax) continue;
        const cr_bvh_node& n = S.nodes[e.node];
        if (n.count) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) {
                const uint32_t index = S.indices[i];
                if (index == ignore) continue;
                Hit c; c.t = closest; c.tri = index;
                if (!intersectTriangle(S.tris[index], clipped, c) || !accepts(S, S.tris[index], clipped, c.u, c.v)) continue;
                if (any) { hit = c; return true; }
                if (!found || c.t < hit.t || (c.t == hit.t && index < hit.tri)) {
                    hit = c; closest = c.t;
                    clipped.tmax = std::min(query, std::nextafter(static_cast<float>(c.t), inf));
                    found = true;
                }
            }
        } else {
            float ln = 0, rn = 0;
            const bool l = box(S.nodes[n.first], ln), r = box(S.nodes[n.first + 1], rn);
            if (size + l + r > 50) throw std::logic_error("BVH traversal exceeded its bounded stack");
            if (l && r) {
                if (ln <= rn) { stack[size++] = {n.first + 1, rn}; stack[size++] = {n.first, ln}; }
                else { stack[size++] = {n.first, ln}; stack[size++] = {n.first + 1, rn}; }
            } else if (l) stack[size++] = {n.first, ln};
            else if (r) stack[size++] = {n.first + 1, rn};
        }
    }
    return found;
}

// offsetRay (geometry.cpp:186-209)
Ray offsetRay(V3 p, V3 gn, V3 dir, float maxDistance = inf) {
    if (!finite(p) || !finite(gn) || !finite(dir) || !nonzero(gn) || !nonzero(dir) || std::isnan(maxDistance) || maxDistance < 0)
        throw Failure("Invalid secondary ray");
    dir = unit(dir);
    V3 n = unit(gn);
    if (pdot(D3(n), D3(dir)) < 0) n = -n;
    const double scale = std::max({std::abs(static_cast<double>(p.x)), std::abs(static_cast<double>(p.y)), std::abs(static_cast<double>(p.z))});
    const double dist = 4 * std::numeric_limits<float>::epsilon() * scale;
    V3 o = p;
    for (int a = 0; a < 3; ++a) {
        o[a] = static_cast<float>(static_cast<double>(p[a]) + dist * n[a]);
        if (n[a] != 0) o[a] = std::nextafter(o[a], n[a] > 0 ? inf : -inf);
    }
    if (!finite(o)) throw Failure("Secondary ray offset exceeds finite coordinates");
    float limit = maxDistance;
    if (std::isfinite(limit)) {
        const double adv = pdot(D3(o) - D3(p), D3(dir));
        limit = static_cast<float>(std::max(0.0, static_cast<double>(limit) - adv));
        limit = std::nextafter(limit, 0.0f);
    }
    Ray r; r.o = o; r.d = dir; r.tmin = 0; r.tmax = limit;
    return r;
}

// surfaceAt (geometry.cpp:401-459)
struct Surface {
    V3 position, gn, normal, tangent, bitangent, low, baseColor, emission, attColor;
    float metallic = 0, roughness = 1, transmission = 0, ior = 1.5f, thickness = 0, attDistance = inf;
    uint32_t material = 0;
    bool front = true, doubleSided = false;
};
Surface surfaceAt(const Scene& S, V3 dir, uint32_t index, double hu, double hv) {
    const cr_triangle& t = S.tris[index];
    const cr_material& m = S.mats[t.material];
    const double w = 1.0 - hu - hv;
    const D3 p = D3(v3(t.v[0].position)) * w + D3(v3(t.v[1].position)) * hu + D3(v3(t.v[2].position)) * hv;
    Surface s;
    s.position = {static_cast<float>(p.x), static_cast<float>(p.y), static_cast<float>(p.z)};
    s.low = {static_cast<float>(p.x - s.position.x), static_cast<float>(p.y - s.position.y), static_cast<float>(p.z - s.position.z)};
    s.gn = v3(t.geometric_normal);
    s.front = pdot(D3(dir), D3(s.gn)) < 0;
    s.normal = unit(D3(v3(t.v[0].normal)) * w + D3(v3(t.v[1].normal)) * hu + D3(v3(t.v[2].normal)) * hv, s.gn);
    if (dot(s.normal, s.gn) < 0) s.normal = -s.normal;
    auto tg = [](const cr_vertex& v) { return D3(V3{v.tangent[0], v.tangent[1], v.tangent[2]}); };
    s.tangent = orthogonalized(tg(t.v[0]) * w + tg(t.v[1]) * hu + tg(t.v[2]) * hv, s.normal, Frame(s.normal).x);
    float hand = w * t.v[0].tangent[3] + hu * t.v[1].tangent[3] + hv * t.v[2].tangent[3] < 0 ? -1.0f : 1.0f;
    s.bitangent = cross(s.normal, s.tangent) * hand;
    float a, b, c, d;
    interpUv(t, hu, hv, 0, a, b);
    interpUv(t, hu, hv, 1, c, d);
    const F4 base = sampleTex(S, m.base_color_texture, a, b, c, d, true);
    s.baseColor = V3{m.base_color[0], m.base_color[1], m.base_color[2]} * V3{base.x, base.y, base.z};
    const F4 mr = sampleTex(S, m.metallic_roughness_texture, a, b, c, d, false);
    s.metallic = std::clamp(m.metallic * mr.z, 0.0f, 1.0f);
    s.roughness = std::clamp(m.roughness * mr.y, 0.0f, 1.0f);
    const F4 em = sampleTex(S, m.emissive_texture, a, b, c, d, true);
    s.emission = v3(m.emission) * V3{em.x, em.y, em.z};
    s.transmission = std::clamp(m.transmission * sampleTex(S, m.transmission_texture, a, b, c, d, false).x, 0.0f, 1.0f);
    s.ior = m.ior; s.thickness = m.thickness; s.attDistance = m.attenuation_distance; s.attColor = v3(m.attenuation_color);
    s.material = t.material; s.doubleSided = m.double_sided != 0;
    if (m.normal_texture.texture >= 0) {
        const cr_texture_slot& slot = m.normal_texture;
        if (slot.scale[0] != 0 && slot.scale[1] != 0) {
            const double cr = std::cos(static_cast<double>(slot.rotation)), sr = std::sin(static_cast<double>(slot.rotation));
            const D3 tt = D3(s.tangent) * (cr / slot.scale[0]) - D3(s.bitangent) * (sr / slot.scale[1]);
            s.tangent = orthogonalized(tt, s.normal, s.tangent);
            if ((slot.scale[0] < 0) != (slot.scale[1] < 0)) hand = -hand;
            s.bitangent = cross(s.normal, s.tangent) * hand;
        }
        const F4 tx = sampleTex(S, slot, a, b, c, d, false);
        const D3 mapped = D3(s.tangent) * ((2.0 * tx.x - 1) * m.normal_scale) + D3(s.bitangent) * ((2.0 * tx.y - 1) * m.normal_scale) +
                          D3(s.normal) * (2.0 * tx.z - 1);
        s.normal = unit(mapped, s.normal);
        if (dot(s.normal, s.gn) < 0) s.normal = -s.normal;
        s.tangent = orthogonalized(D3(s.tangent), s.normal, Frame(s.normal).x);
        s.bitangent = cross(s.normal, s.tangent) * hand;
    }
    return s;
}

// BSDF (bsdf.cpp)
float fresnelDielectric(float c, float ei, float et) {
    if (ei == et) return 0;
    c = std::clamp(std::abs(c), 0.0f, 1.0f);
    const float eta = ei / et;
    const float s2 = eta * eta * std::max(0.0f, 1 - c * c);
    if (s2 >= 1) return 1;
    const float ct = std::sqrt(1 - s2);
    const float ds = ei * c + et * ct, dp = et * c + ei * ct;
    if (ds == 0 || dp == 0) return 1;
    const float rs = (ei * c - et * ct) / ds, rp = (et * c - ei * ct) / dp;
    return 0.5f * (rs * rs + rp * rp);
}
bool refractDir(V3 wo, V3 n, float ratio, V3& wi) {
    const float ci = dot(wo, n);
    const float s2 = ratio * ratio * std::max(0.0f, 1 - ci * ci);
    if (s2 >= 1) return false;
    wi = normalize(-wo * ratio + n * (ratio * ci - std::sqrt(1 - s2)));
    return true;
}
V3 absorption(V3 color, float d) {
    if (!std::isfinite(d)) return {};
    if (!(d > 0)) throw Failure("Attenuation distance must be positive");
    color = clamp(color, 1e-8f, 1);
    return {-std::log(color.x) / d, -std::log(color.y) / d, -std::log(color.z) / d};
}
V3 beer(V3 c, float d) {
    if (d == inf) return {c.x > 0 ? 0.0f : 1.0f, c.y > 0 ? 0.0f : 1.0f, c.z > 0 ? 0.0f : 1.0f};
    return vexp(c * (-std::max(0.0f, d)));
}
float distribution(float a, V3 h) {
    if (h.z <= 0) return 0;
    const float a2 = a * a;
    const float d = (h.x * h.x + h.y * h.y) + a2 * h.z * h.z;
    return a2 / (pi * d * d);
}
float smithG1(float a, V3 v) {
    const float c2 = v.z * v.z;
    if (c2 == 0) return 0;
    return 2 / (1 + std::sqrt(1 + a * a * (v.x * v.x + v.y * v.y) / c2));
}
V3 visibleNormal(V3 wo, float a, float u, float v) {
    const V3 vh = normalize({a * wo.x, a * wo.y, wo.z});
    const float l2 = vh.x * vh.x + vh.y * vh.y;
    const V3 t1 = l2 > 0 ? V3{-vh.y, vh.x, 0} / std::sqrt(l2) : V3{1, 0, 0};
    const V3 t2 = cross(vh, t1);
    const float r = std::sqrt(u), phi = 2 * pi * v;
    const float x = r * std::cos(phi);
    float y = r * std::sin(phi);
    const float s = 0.5f * (1 + vh.z);
    y = (1 - s) * std::sqrt(std::max(0.0f, 1 - x * x)) + s * y;
    const V3 nh = t1 * x + t2 * y + vh * std::sqrt(std::max(0.0f, 1 - x * x - y * y));
    return normalize({a * nh.x, a * nh.y, std::max(0.0f, nh.z)});
}
struct Ctx {
    const Surface& s;
    Frame frame;
    V3 wo;
    float etaI, etaT, eta, alpha, dp = 0, dtp = 0;
    bool thin, smooth, matched = false;
    float fresnel(float c) const { const float f = fresnelDielectric(c, etaI, etaT); return thin ? 2 * f / (1 + f) : f; }
    V3 reflection(float f, float c) const {
        const float sch = std::pow(1 - std::clamp(std::abs(c), 0.0f, 1.0f), 5.0f);
        return V3{(1 - s.metallic) * f} + (s.baseColor + (V3{1} - s.baseColor) * sch) * s.metallic;
    }
    V3 transmission(float f) const { return s.baseColor * ((1 - s.metallic) * s.transmission * (1 - f)); }
    float reflProb(float f, float c) const {
        if (matched) return 1;
        const float r = luminance(reflection(f, c)), t = luminance(transmission(f));
        return r + t > 0 ? r / (r + t) : 1;
    }
    float micro() const { return std::max(0.0f, 1 - dp - dtp); }
    Ctx(const Surface& surf, V3 out)
        : s(surf), frame(dot(out, surf.normal) > 0 ? surf.normal : -surf.normal), wo(frame.local(out)),
          etaI(s.thickness > 0 && !s.front ? s.ior : 1), etaT(s.thickness > 0 && !s.front ? 1 : s.ior), eta(etaT / etaI),
          alpha(std::max(0.001f, s.roughness * s.roughness)), thin(s.thickness <= 0 && s.transmission > 0), smooth(s.roughness <= 0.001f) {
        if (thin) { etaI = 1; etaT = s.ior; eta = s.ior; }
        matched = std::abs(etaI - etaT) <= std::sqrt(std::numeric_limits<float>::epsilon()) * std::max(etaI, etaT);
        if (matched) etaI = etaT = eta = 1;
        const float f = fresnel(wo.z);
        const float diffuse = (1 - s.metallic) * (1 - s.transmission) * luminance(s.baseColor) * (1 - f);
        const float transmit = (1 - s.metallic) * s.transmission * (1 - f) * luminance(s.baseColor);
        const float total = diffuse + luminance(reflection(f, wo.z)) + transmit;
        if (total > 0) { dp = diffuse / total; if (matched) dtp = transmit / total; }
    }
};
struct Eval { V3 value{}; float pdf = 0; };
struct Sample {
    V3 dir{}, weight{};
    float pdf = 0, eta = 1;
    bool delta = false, transmitted = false;
    explicit operator bool() const { return maxComponent(weight) > 0 && finite(weight) && finite(dir); }
};
Eval evalLocal(const Ctx& c, V3 wi) {
    Eval r;
    const float no = c.wo.z, ni = std::abs(wi.z);
    if (no <= 1e-7f || ni <= 1e-7f) return r;
    const bool refl = wi.z > 0;
    if (!refl && (c.matched || c.thin)) return r;
    if (refl) {
        const float diffuse = (1 - c.s.metallic) * (1 - c.s.transmission) * (1 - c.fresnel(no)) * (1 - c.fresnel(ni));
        r.value = c.s.baseColor * (diffuse / pi);
        r.pdf = c.dp * ni / pi;
    }
    if (c.smooth) return r;
    V3 h = normalize(refl ? c.wo + wi : c.wo + wi * c.eta);
    if (h.z < 0) h = -h;
    const float oh = dot(c.wo, h), ih = dot(wi, h);
    if (oh <= 0 || (refl ? ih <= 0 : ih >= 0)) return r;
    const float f = c.fresnel(oh), pr = c.reflProb(f, oh);
    const float d = distribution(c.alpha, h), g1 = smithG1(c.alpha, c.wo), g = g1 * smithG1(c.alpha, wi);
    const float pdfH = d * g1 * oh / no;
    if (refl) {
        r.value += c.reflection(f, oh) * (d * g / (4 * no * ni));
        r.pdf += c.micro() * pr * pdfH / (4 * oh);
    } else {
        const float den = oh + c.eta * ih, den2 = den * den;
        if (den2 < 1e-20f) return {};
        r.value = c.transmission(f) * (d * g * std::abs(oh * ih) / (no * ni * den2));
        r.pdf = c.micro() * (1 - pr) * pdfH * c.eta * c.eta * std::abs(ih) / den2;
    }
    return r;
}
bool geoSide(const Surface& s, V3 wo, V3 wi, bool tr) {
    const float d = dot(wo, s.gn) * dot(wi, s.gn);
    return tr ? d < 0 : d > 0;
}
Eval evaluateBsdf(const Surface& s, V3 wo, V3 wi) {
    const Ctx c(s, wo);
    const V3 l = c.frame.local(wi);
    if (!geoSide(s, wo, wi, l.z < 0)) return {};
    return evalLocal(c, l);
}
Sample sampleBsdf(const Surface& s, V3 wo, Rng& rng) {
    const Ctx c(s, wo);
    Sample out;
    if (c.wo.z <= 1e-7f) return out;
    V3 wi;
    const float lobe = rng.uniform();
    if (lobe < c.dp) {
        const float u = rng.uniform(), phi = 2 * pi * rng.uniform();
        wi = {std::sqrt(u) * std::cos(phi), std::sqrt(u) * std::sin(phi), std::sqrt(1 - u)};
    } else if (lobe < c.dp + c.dtp) {
        out.dir = -wo; out.delta = true; out.transmitted = true; out.pdf = c.dtp;
        out.weight = s.baseColor * ((1 - s.metallic) * s.transmission / out.pdf);
        return geoSide(s, wo, out.dir, true) ? out : Sample{};
    } else {
        const float u = rng.uniform(), v = rng.uniform();
        const V3 h = c.smooth ? V3{0, 0, 1} : visibleNormal(c.wo, c.alpha, u, v);
        const float oh = dot(c.wo, h), f = c.fresnel(oh), pr = c.reflProb(f, oh);
        const bool refl = rng.uniform() < pr;
        if (refl) wi = reflect(-c.wo, h);
        else if (c.thin) wi = -c.wo;
        else if (!refractDir(c.wo, h, 1 / c.eta, wi)) return out;
        if ((refl && wi.z <= 0) || (!refl && wi.z >= 0)) return out;
        out.transmitted = !refl;
        out.eta = out.transmitted && !c.thin ? c.eta : 1;
        if (c.smooth || (!refl && c.thin)) {
            out.delta = true;
            out.dir = normalize(c.frame.world(wi));
            if (!geoSide(s, wo, out.dir, out.transmitted)) return {};
            const float prob = c.micro() * (refl ? pr : 1 - pr);
            if (prob <= 0) return {};
            out.pdf = prob;
            out.weight = (refl ? c.reflection(f, oh) : c.transmission(f) / (out.eta * out.eta)) / prob;
            return out;
        }
    }
    out.dir = normalize(c.frame.world(wi));
    wi = c.frame.local(out.dir);
    if ((wi.z < 0) != out.transmitted || !geoSide(s, wo, out.dir, out.transmitted)) return {};
    const Eval e = evalLocal(c, wi);
    if (e.pdf <= 0 || !std::isfinite(e.pdf)) return {};
    out.pdf = e.pdf;
    out.weight = e.value * (std::abs(wi.z) / e.pdf);
    return out;
}

// Lights (render.cpp:120-229)
void buildLights(Scene& S) {
    S.triProb.assign(S.tris.size(), 0.0f);
    V3 lo{inf}, hi{-inf};
    for (const auto& t : S.tris)
        for (const auto& v : t.v)
            for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], v.position[a]); hi[a] = std::max(hi[a], v.position[a]); }
    const double radius2 = S.tris.empty() ? 1 : std::max(1.0, static_cast<double>(lengthSquared(hi - lo)) * 0.25);
    double total = 0;
    auto add = [&](int type, uint32_t i, double w) { if (w > 0) { total += w; S.entries.push_back({type, i, total, 0}); } };
    for (uint32_t i = 0; i < S.lights.size(); ++i) {
        const auto& l = S.lights[i];
        add(0, i, static_cast<double>(luminance(v3(l.color))) * l.intensity * (l.type == CR_LIGHT_DIRECTIONAL ? pi * radius2 : 4 * pi));
    }
    for (uint32_t i = 0; i < S.tris.size(); ++i) {
        const auto& t = S.tris[i];
        const auto& m = S.mats[t.material];
        add(1, i, static_cast<double>(t.area) * pi * luminance(v3(m.emission)) * (m.double_sided ? 2 : 1));
    }
    add(2, 0, S.env.integral * pi * radius2);
    double last = 0, cum = 0;
    for (auto& e : S.entries) {
        const double p = 0.95 * (e.cdf - last) / total + 0.05 / static_cast<double>(S.entries.size());
        last = e.cdf; cum += p;
        e.probability = static_cast<float>(p); e.cdf = cum;
        if (e.type == 1) S.triProb[e.index] = e.probability;
        if (e.type == 2) S.envProb = e.probability;
    }
    if (!S.entries.empty()) S.entries.back().cdf = 1;
}
float trianglePdf(const Scene& S, uint32_t i, V3 from, V3 point) {
    const auto& t = S.tris[i];
    const V3 dir = point - from;
    const float len2 = lengthSquared(dir), cosine = std::abs(dot(v3(t.geometric_normal), normalize(dir)));
    return cosine > 1e-8f ? S.triProb[i] * len2 / (t.area * cosine) : 0;
}
struct LightSample { V3 dir, radiance, target, targetNormal; float distance = inf, pdf = 0; bool delta = false; };
LightSample sampleLight(const Scene& S, V3 from, Rng& rng) {
    LightSample out;
    if (S.entries.empty()) return out;
    const double u = rng.uniform();
    auto it = std::lower_bound(S.entries.begin(), S.entries.end(), u, [](const LightEntry& e, double v) { return e.cdf < v; });
    const auto& e = it == S.entries.end() ? S.entries.back() : *it;
    if (e.type == 2) {
        out.dir = envSample(S.env, rng, out.pdf);
        out.pdf *= e.probability;
        out.radiance = envRadiance(S.env, out.dir);
        return out;
    }
    if (e.type == 0) {
        const auto& l = S.lights[e.index];
        out.delta = true; out.pdf = e.probability;
        float att = 1;
        if (l.type == CR_LIGHT_DIRECTIONAL) out.dir = -v3(l.direction);
        else {
            const V3 delta = v3(l.position) - from;
            const float r2 = lengthSquared(delta);
            if (r2 < 1e-12f) return {};
            out.distance = std::sqrt(r2); out.dir = delta / out.distance; out.target = v3(l.position);
            att = 1 / r2;
            if (std::isfinite(l.range)) { const float q = out.distance / l.range; att *= std::max(0.0f, 1 - q * q * q * q); }
            if (l.type == CR_LIGHT_SPOT) {
                const float ca = dot(v3(l.direction), -out.dir), outer = std::cos(l.outer_cone), inner = std::cos(l.inner_cone);
                const float fo = std::clamp((ca - outer) / std::max(1e-7f, inner - outer), 0.0f, 1.0f);
                att *= fo * fo;
            }
        }
        out.radiance = v3(l.color) * (l.intensity * att);
        return out;
    }
    const auto& t = S.tris[e.index];
    const float r = std::sqrt(rng.uniform()), u1 = 1 - r, u2 = r * rng.uniform(), u0 = 1 - u1 - u2;
    out.target = v3(t.v[0].position) * u0 + v3(t.v[1].position) * u1 + v3(t.v[2].position) * u2;
    out.targetNormal = v3(t.geometric_normal);
    const V3 delta = out.target - from;
    out.distance = length(delta);
    if (out.distance < 1e-7f) return {};
    out.dir = delta / out.distance;
    Ray ray; ray.o = from; ray.d = out.dir;
    if (!accepts(S, t, ray, u1, u2)) return {};
    const Surface s = surfaceAt(S, out.dir, e.index, u1, u2);
    if (!s.front && !s.doubleSided) return {};
    out.radiance = s.emission;
    out.pdf = trianglePdf(S, e.index, from, out.target);
    return out;
}

// trace (render.cpp:233-348)
V3 trace(const Scene& S, Ray ray, const cr_render_options& o, Rng& rng, bool precise) {
    V3 radiance{}, T{1}, lastPos{}, A{};
    float lastPdf = 0, etaScale = 1;
    bool lastDelta = true;
    int medium = -1;
    uint32_t prev = noTriangle;
    for (int depth = 0; depth <= o.bounces; ++depth) {
        Hit hit;
        if (!intersect(S, ray, hit, false, prev)) {
            if (medium >= 0) T *= beer(A, inf);
            const float w = lastDelta || !o.next_event_estimation ? 1 : powerHeuristic(lastPdf, S.envProb * envPdf(S.env, ray.d));
            radiance += T * envRadiance(S.env, ray.d) * w;
            break;
        }
        if (medium >= 0) T *= beer(A, static_cast<float>(hit.t));
        const Surface s = surfaceAt(S, ray.d, hit.tri, hit.u, hit.v);
        if (s.front || s.doubleSided) {
            const float w = lastDelta || !o.next_event_estimation ? 1 : powerHeuristic(lastPdf, trianglePdf(S, hit.tri, lastPos, s.position));
            radiance += T * s.emission * w;
        }
        if (depth == o.bounces) break;
        const V3 wo = -ray.d;
        if (o.next_event_estimation) {
            const LightSample light = sampleLight(S, s.position, rng);
            const bool enclosed = medium >= 0 && s.thickness <= 0 && !std::isfinite(light.distance);
            if (!enclosed && light.pdf > 0 && maxComponent(light.radiance) > 0) {
                const Eval b = evaluateBsdf(s, wo, light.dir);
                if (maxComponent(b.value) > 0) {
                    Ray sh;
                    if (precise) { sh.o = s.position; sh.d = light.dir; sh.lo = s.low; }
                    else sh = offsetRay(s.position, s.gn, light.dir);
                    if (std::isfinite(light.distance)) {
                        V3 end = light.target;
                        if (lengthSquared(light.targetNormal) > 0) end = offsetRay(end, light.targetNormal, -light.dir).o;
                        const V3 delta = end - sh.o;
                        sh.tmax = length(delta) * (1 - 2e-6f); sh.d = normalize(delta);
                    }
                    Hit blocker;
                    if (!intersect(S, sh, blocker, true, precise ? hit.tri : noTriangle)) {
                        const float w = light.delta ? 1 : powerHeuristic(light.pdf, b.pdf);
                        V3 shA = A;
                        bool shIn = medium >= 0;
                        if (s.thickness > 0 && dot(wo, s.gn) * dot(light.dir, s.gn) < 0) {
                            shIn = s.front;
                            shA = s.front ? absorption(s.attColor, s.attDistance) : V3{};
                        }
                        const V3 tr = shIn ? beer(shA, light.distance) : V3{1};
                        radiance += T * b.value * light.radiance * tr * (std::abs(dot(s.normal, light.dir)) * w / light.pdf);
                    }
                }
            }
        }
        const Sample smp = sampleBsdf(s, wo, rng);
        if (!smp) break;
        T *= smp.weight;
        if (!finite(T)) throw Failure("Non-finite path throughput");
        if (smp.transmitted && s.thickness > 0) {
            if (s.front) {
                if (medium >= 0) throw Failure("Nested/intersecting refractive volumes are unsupported; separate the closed meshes", true);
                medium = static_cast<int>(s.material); A = absorption(s.attColor, s.attDistance);
            } else {
                if (medium < 0) {
                    std::ostringstream d;
                    d.precision(9);
                    d << "Refractive exit without entry; check outward normals and keep the camera outside closed volumes"
                      << "; bounce " << depth << ", triangle " << hit.tri << ", material " << s.material << ", t " << hit.t
                      << ", point (" << s.position.x << ',' << s.position.y << ',' << s.position.z << "), origin (" << ray.o.x
                      << ',' << ray.o.y << ',' << ray.o.z << "), direction (" << ray.d.x << ',' << ray.d.y << ',' << ray.d.z << ')';
                    throw Failure(d.str(), true);
                }
                medium = -1; A = {};
            }
            etaScale *= smp.eta * smp.eta;
        }
        lastPdf = smp.pdf; lastDelta = smp.delta; lastPos = s.position;
        if (precise) { ray = Ray{}; ray.o = s.position; ray.d = smp.dir; ray.lo = s.low; }
        else ray = offsetRay(s.position, s.gn, smp.dir);
        prev = precise ? hit.tri : noTriangle;
        if (o.russian_roulette && depth >= 3) {
            const float survive = std::clamp(maxComponent(T) * etaScale, 0.05f, 0.95f);
            if (rng.uniform() >= survive) break;
            T *= 1 / survive;
        }
    }
    if (!finite(radiance) || std::min({radiance.x, radiance.y, radiance.z}) < 0) throw Failure("Non-finite or negative path radiance");
    return radiance;
}

// Camera::generate (geometry.cpp:213-234)
Ray generate(const cr_camera& c, float px, float py, int W, int H) {
    const V3 pos = v3(c.position), fw = v3(c.forward), rt = v3(c.right), up = v3(c.up);
    if (W <= 0 || H <= 0 || !std::isfinite(px) || !std::isfinite(py) || !finite(pos) || !finite(fw) || !finite(rt) || !finite(up) ||
        !std::isfinite(c.yfov) || c.yfov <= 0 || c.yfov >= pi || !std::isfinite(c.aspect) || c.aspect < 0 || !std::isfinite(c.near_clip) ||
        c.near_clip < 0 || std::isnan(c.far_clip) || c.far_clip <= c.near_clip)
        throw Failure("Invalid perspective camera or image dimensions");
    const V3 f = unit(fw);
    const V3 r = orthogonalized(D3(rt), f);
    const V3 u = orthogonalized(D3(orthogonalized(D3(up), f)), r);
    if (!nonzero(f) || !nonzero(r) || !nonzero(u)) throw Failure("Degenerate camera basis");
    const double ratio = c.aspect > 0 ? c.aspect : static_cast<double>(W) / H;
    const double hh = std::tan(static_cast<double>(c.yfov) * 0.5);
    const double x = (2 * static_cast<double>(px) / W - 1) * ratio * hh;
    const double y = (1 - 2 * static_cast<double>(py) / H) * hh;
    const V3 d = unit(D3(f) + D3(r) * x + D3(u) * y);
    const double proj = pdot(D3(d), D3(f));
    const double nearT = c.near_clip / proj;
    if (!(proj > 0) || !std::isfinite(nearT) || nearT > std::numeric_limits<float>::max()) throw Failure("Unrepresentable perspective ray");
    Ray ray; ray.o = pos; ray.d = d; ray.tmin = static_cast<float>(nearT); ray.tmax = static_cast<float>(c.far_clip / proj);
    return ray;
}

thread_local std::string lastError;

Scene makeScene(const cr_scene_desc* d, const cr_environment_desc* e, int brute) {
    Scene S;
    S.tris.assign(d->triangles, d->triangles + d->triangle_count);
    S.mats.assign(d->materials, d->materials + d->material_count);
    if (d->light_count) S.lights.assign(d->lights, d->lights + d->light_count);
    for (uint32_t i = 0; i < d->image_count; ++i) {
        Image im; im.w = d->images[i].width; im.h = d->images[i].height;
        im.px.assign(d->images[i].pixels, d->images[i].pixels + 4 * static_cast<size_t>(im.w) * im.h);
        S.images.push_back(std::move(im));
    }
    if (d->texture_count) S.textures.assign(d->textures, d->textures + d->texture_count);
    if (d->bvh_node_count) {
        S.nodes.assign(d->bvh_nodes, d->bvh_nodes + d->bvh_node_count);
        S.indices.assign(d->bvh_indices, d->bvh_indices + d->bvh_index_count);
    } else if (!brute && d->triangle_count) {
        throw std::invalid_argument("the oracle needs the BVH arrays or brute-force mode");
    }
    S.brute = brute != 0;
    if (e && e->pixels) {
        S.env.image = true; S.env.w = e->width; S.env.h = e->height;
        S.env.px.assign(e->pixels, e->pixels + 4 * static_cast<size_t>(e->width) * e->height);
        S.env.rotation = e->rotation_radians; S.env.intensity = e->intensity;
    } else if (e) {
        S.env.constant = v3(e->constant);
    }
    buildEnv(S.env);
    buildLights(S);
    return S;
}

// ---- output encoding (src/io/image.cpp, src/io/file.h; stb_image_write 1.16) ---------------------
// The checker for the device encoder: per-pixel direct evaluation of the reference's display
// mapping, and the Radiance writer of the codec io::writeHdr calls, restated from its published
// algorithm (third_party/stb_image_write.h: stbiw__linear_to_rgbe, stbiw__write_hdr_scanline,
// stbi_write_hdr_core).

void imagePixels(int width, int height, const std::string& label) {  // file.h:84-89
    if (width <= 0 || height <= 0 || width > 16384 || height > 16384 ||
        static_cast<std::size_t>(width) > 16777216u / static_cast<std::size_t>(height))
        throw std::runtime_error(label + ": image dimensions must be positive, at most 16384 per axis and 16777216 pixels");
}

void validateOutput(int width, int height, const float* rgb, const std::string& label, bool hdr) {  // image.cpp:100-113
    imagePixels(width, height, label);
    const std::size_t n = static_cast<std::size_t>(width) * height;
    for (std::size_t i = 0; i < n; ++i) {
        const float r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        if (!std::isfinite(r) || !std::isfinite(g) || !std::isfinite(b) || r < 0 || g < 0 || b < 0)
            throw std::runtime_error(label + ": pixels must contain finite, nonnegative linear radiance");
        if (hdr && std::max({r, g, b}) >= std::ldexp(1.0f, 127))
            throw std::runtime_error(label + ": radiance exceeds the Radiance RGBE exponent range");
    }
}

float linearToSrgb(float v) { return v <= 0.0031308f ? 12.92f * v : 1.055f * std::pow(v, 1 / 2.4f) - 0.055f; }  // math.h:62

unsigned char displayChannel(float value, double exposureScale) {  // image.cpp:119-124
    const double x = static_cast<double>(value) * exposureScale;
    const double filmic = std::clamp((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0);
    const float srgb = linearToSrgb(static_cast<float>(filmic));
    return static_cast<unsigned char>(std::lround(std::clamp(srgb, 0.0f, 1.0f) * 255.0f));
}

void rgbe(const float* linear, unsigned char* out) {  // stbiw__linear_to_rgbe
    const float m = std::max(linear[0], std::max(linear[1], linear[2]));
    if (m < 1e-32f) { out[0] = out[1] = out[2] = out[3] = 0; return; }
    int e;
    const float normalize = static_cast<float>(std::frexp(m, &e)) * 256.0f / m;
    for (int c = 0; c < 3; ++c) out[c] = static_cast<unsigned char>(static_cast<int>(linear[c] * normalize));
    out[3] = static_cast<unsigned char>(e + 128);
}

// stbiw__write_hdr_scanline: run-length coding of each component of one scanline.
void hdrScanline(const float* row, int width, std::vector<unsigned char>& out) {
    std::vector<unsigned char> q(4 * static_cast<std::size_t>(width));
    for (int x = 0; x < width; ++x) rgbe(row + 3 * x, &q[4 * x]);
    if (width < 8 || width >= 32768) { out.insert(out.end(), q.begin(), q.end()); return; }
    out.push_back(2); out.push_back(2);
    out.push_back(static_cast<unsigned char>((width & 0xff00) >> 8)); out.push_back(static_cast<unsigned char>(width & 0xff));
    for (int c = 0; c < 4; ++c) {
        auto comp = [&](int x) { return q[4 * x + c]; };
        int x = 0;
        while (x < width) {
            int r = x;  // start of the next run of three
            while (r + 2 < width && !(comp(r) == comp(r + 1) && comp(r) == comp(r + 2))) ++r;
            if (r + 2 >= width) r = width;
            for (; x < r;) {  // literal pieces of at most 128
                const int len = std::min(r - x, 128);
                out.push_back(static_cast<unsigned char>(len));
                for (int k = 0; k < len; ++k) out.push_back(comp(x + k));
                x += len;
            }
            if (r + 2 < width) {  // the run, in pieces of at most 127
                while (r < width && comp(r) == comp(x)) ++r;
                for (; x < r;) {
                    const int len = std::min(r - x, 127);
                    out.push_back(static_cast<unsigned char>(len + 128));
                    out.push_back(comp(x));
                    x += len;
                }
            }
        }
    }
}

}  // namespace
}  // namespace oracle

using namespace oracle;

extern "C" {

size_t oracle_last_error(char* buf, size_t n) {
    if (buf && n) {
        const size_t k = std::min(n - 1, lastError.size());
        std::memcpy(buf, lastError.data(), k);
        buf[k] = 0;
    }
    return lastError.size();
}

// Bvh::intersect per ray (brute = 1: scan every triangle).
int oracle_intersect(const cr_scene_desc* d, int brute, const cr_ray* rays, uint64_t n, int any, uint32_t ignore, cr_hit* hits, uint8_t* found) {
    try {
        const Scene S = makeScene(d, nullptr, brute);
        for (uint64_t i = 0; i < n; ++i) {
            Ray r; r.o = v3(rays[i].origin); r.d = v3(rays[i].direction); r.tmin = rays[i].tmin; r.tmax = rays[i].tmax; r.lo = v3(rays[i].origin_low);
            Hit h; h.t = hits[i].t; h.u = hits[i].u; h.v = hits[i].v; h.tri = hits[i].triangle;
            found[i] = intersect(S, r, h, any != 0, ignore) ? 1 : 0;
            if (found[i]) { hits[i].t = h.t; hits[i].u = h.u; hits[i].v = h.v; hits[i].triangle = h.tri; }
        }
        return 0;
    } catch (const std::exception& e) { lastError = e.what(); return 2; }
}

// cr::render (render.cpp:352-456) with `threads` worker threads over pixel rows. The film is
// the FP64 sum of each pixel's samples in index order; per_sample (optional) receives
// samples*W*H*3 floats, sample-major.
int oracle_render(const cr_scene_desc* d, const cr_environment_desc* e, const cr_camera* cam, const cr_render_options* o,
                  int threads, float* film, float* per_sample, uint64_t* retries) {
    try {
        const Scene S = makeScene(d, e, 0);
        const int W = o->width, H = o->height;
        std::atomic<int> nextRow{0};
        std::atomic<uint64_t> retry{0};
        std::string error;
        std::atomic<bool> failed{false};
        std::vector<std::string> errors(H);
        auto worker = [&] {
            for (;;) {
                const int y = nextRow.fetch_add(1);
                if (y >= H || failed.load()) return;
                for (int x = 0; x < W; ++x) {
                    const uint64_t pixel = static_cast<uint64_t>(y) * W + x;
                    double r = 0, g = 0, b = 0;
                    int sample = 0;
                    try {
                        for (sample = 0; sample < o->samples; ++sample) {
                            Rng rng(sampleSeed(o->seed, pixel, static_cast<uint64_t>(sample)));
                            const float dx = rng.uniform(), dy = rng.uniform();
                            const Ray ray = generate(*cam, static_cast<float>(x) + dx, static_cast<float>(y) + dy, W, H);
                            const Rng initial = rng;
                            V3 L;
                            try { L = trace(S, ray, *o, rng, false); }
                            catch (const Failure& f) {
                                if (!f.boundary) throw;
                                retry.fetch_add(1);
                                rng = initial;
                                L = trace(S, ray, *o, rng, true);
                            }
                            if (per_sample) {
                                float* p = per_sample + 3 * (static_cast<uint64_t>(sample) * W * H + pixel);
                                p[0] = L.x; p[1] = L.y; p[2] = L.z;
                            }
                            r += L.x; g += L.y; b += L.z;
                        }
                    } catch (const std::exception& ex) {
                        errors[y] = "Pixel (" + std::to_string(x) + "," + std::to_string(y) + "), sample " + std::to_string(sample) + ": " + ex.what();
                        failed.store(true);
                        return;
                    }
                    film[3 * pixel] = static_cast<float>(r / o->samples);
                    film[3 * pixel + 1] = static_cast<float>(g / o->samples);
                    film[3 * pixel + 2] = static_cast<float>(b / o->samples);
                }
            }
        };
        std::vector<std::thread> pool;
        const int n = std::max(1, threads);
        for (int i = 0; i < n; ++i) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        for (const auto& m : errors) if (!m.empty()) { lastError = m; return 2; }
        if (retries) *retries = retry.load();
        return 0;
    } catch (const std::exception& ex) { lastError = ex.what(); return 2; }
}

// io::writePng's pixels (format 0), RGBE quads (1) or io::writeHdr's whole file (2).
int oracle_encode(const float* rgb, int width, int height, int format, float exposure, unsigned char* out,
                  uint64_t capacity, uint64_t* size) {
    try {
        std::vector<unsigned char> bytes;
        if (format == 0) {
            validateOutput(width, height, rgb, "PNG output", false);
            if (!std::isfinite(exposure) || exposure < -100 || exposure > 100)
                throw std::runtime_error("PNG exposure must be finite and between -100 and 100 stops");
            const double scale = std::exp2(static_cast<double>(exposure));
            const std::size_t n = 3 * static_cast<std::size_t>(width) * height;
            bytes.resize(n);
            for (std::size_t i = 0; i < n; ++i) bytes[i] = displayChannel(rgb[i], scale);
        } else {
            validateOutput(width, height, rgb, "HDR output", true);
            if (format == 1) {
                bytes.resize(4 * static_cast<std::size_t>(width) * height);
                for (std::size_t i = 0; i < static_cast<std::size_t>(width) * height; ++i) rgbe(rgb + 3 * i, &bytes[4 * i]);
            } else {
                const std::string header = "#?RADIANCE\n# Written by stb_image_write.h\nFORMAT=32-bit_rle_rgbe\n"
                                           "EXPOSURE=          1.0000000000000\n\n-Y " + std::to_string(height) +
                                           " +X " + std::to_string(width) + "\n";
                bytes.assign(header.begin(), header.end());
                for (int y = 0; y < height; ++y) hdrScanline(rgb + 3 * static_cast<std::size_t>(y) * width, width, bytes);
            }
        }
        *size = bytes.size();
        if (out && capacity >= bytes.size()) std::memcpy(out, bytes.data(), bytes.size());
        return 0;
    } catch (const std::exception& ex) { lastError = ex.what(); return 1; }
}

}  // extern "C"
