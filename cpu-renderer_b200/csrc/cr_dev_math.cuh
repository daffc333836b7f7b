// Device value types and scalar helpers that reproduce the reference's arithmetic
// (CPU-Renderer src/math.h) operation for operation.
//
// The reference is compiled for x86-64 without FMA, so every float/double + - * / sqrt
// is one IEEE round-to-nearest operation in source order. This translation unit is built
// with --fmad=false (no contraction) and the default IEEE division/sqrt, which makes the
// same expressions round identically here. Expressions below keep the reference's
// association order; std::min/max/clamp keep their NaN behaviour ((b<a)?b:a etc.), which
// differs from fminf/fmaxf.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CR_HD __host__ __device__ __forceinline__
#define CR_D __device__ __forceinline__

namespace crg {

constexpr float kPi = 3.14159265358979323846f;          // math.h:13
constexpr float kInf = __builtin_huge_valf();
constexpr float kFltMax = 3.40282346638528859812e+38f;
constexpr float kFltEps = 1.1920928955078125e-07f;
constexpr double kDblEps = 2.220446049250313080847e-16;
constexpr uint32_t kNoTriangle = 0xffffffffu;

// std::min / std::max / std::clamp semantics (first argument wins ties and NaN compares).
template <class T> CR_HD T smin(T a, T b) { return (b < a) ? b : a; }
template <class T> CR_HD T smax(T a, T b) { return (a < b) ? b : a; }
template <class T> CR_HD T sclamp(T v, T lo, T hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
// std::max({a,b,c}) / std::min({a,b,c}): keep the first extreme element.
template <class T> CR_HD T smax3(T a, T b, T c) { T r = a; if (r < b) r = b; if (r < c) r = c; return r; }
template <class T> CR_HD T smin3(T a, T b, T c) { T r = a; if (b < r) r = b; if (c < r) r = c; return r; }

CR_D bool isfin(float x) { return isfinite(x); }
CR_D bool isfin(double x) { return isfinite(x); }

// std::nextafter(float, direction) for the two directions the reference uses.
CR_D float next_up(float x) {
    if (isnan(x)) return x;
    if (x == kInf) return x;
    if (x == 0.0f) return __int_as_float(1);
    int32_t i = __float_as_int(x);
    return __int_as_float(x > 0.0f ? i + 1 : i - 1);
}
CR_D float next_down(float x) {
    if (isnan(x)) return x;
    if (x == -kInf) return x;
    if (x == 0.0f) return -__int_as_float(1);
    int32_t i = __float_as_int(x);
    return __int_as_float(x > 0.0f ? i - 1 : i + 1);
}
// nextafter(x, 0.0f) for a finite non-negative limit (geometry.cpp:206).
CR_D float next_toward_zero(float x) {
    if (isnan(x) || x == 0.0f) return x;
    int32_t i = __float_as_int(x);
    return __int_as_float(i - 1);  // magnitude shrinks by one ulp for either sign
}

// Transcendentals. glibc's float functions are not correctly rounded, and CUDA's float
// versions err by up to two ulp; evaluating in double and rounding once is correctly
// rounded in all but ~2^-28 of cases, which keeps device paths as close to the host's as
// a portable method allows. CR_FAST_TRANSCENDENTALS switches to the float versions.
// x^5 for the Schlick factor (bsdf.cpp:150, std::pow(x, 5.0f)): x*x is exact in double, two
// more double products leave a relative error below 2^-52, so the float rounding is the
// correctly rounded x^5 except within ~2^-28 of a rounding boundary — the same quality as
// rounding a double pow(), at a fraction of its cost.
CR_D float fpow5(float x) {
    const double d = x, d2 = d * d, d4 = d2 * d2;
    return static_cast<float>(d4 * d);
}
#ifdef CR_FAST_TRANSCENDENTALS
CR_D void fsincos(float x, float& s, float& c) { sincosf(x, &s, &c); }
CR_D float fcos(float x) { return cosf(x); }
CR_D float fsin(float x) { return sinf(x); }
CR_D float fpow(float x, float y) { return powf(x, y); }
CR_D float fexp(float x) { return expf(x); }
CR_D float flog(float x) { return logf(x); }
CR_D float fatan2(float y, float x) { return atan2f(y, x); }
CR_D float facos(float x) { return acosf(x); }
#else
CR_D void fsincos(float x, float& s, float& c) {
    double sd, cd;
    sincos(static_cast<double>(x), &sd, &cd);
    s = static_cast<float>(sd);
    c = static_cast<float>(cd);
}
CR_D float fcos(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
CR_D float fsin(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
CR_D float fpow(float x, float y) { return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y))); }
CR_D float fexp(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
CR_D float flog(float x) { return static_cast<float>(log(static_cast<double>(x))); }
CR_D float fatan2(float y, float x) { return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x))); }
CR_D float facos(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
#endif

// ---- Vec3 (math.h:16-58) ----------------------------------------------------------------
struct V3 {
    float x, y, z;
    CR_HD V3() : x(0), y(0), z(0) {}
    CR_HD explicit V3(float s) : x(s), y(s), z(s) {}
    CR_HD V3(float a, float b, float c) : x(a), y(b), z(c) {}
    CR_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
CR_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
CR_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
CR_HD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
CR_HD V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
CR_HD V3 operator*(V3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
CR_HD V3 operator*(float a, V3 b) { return b * a; }
CR_HD V3 operator/(V3 a, float b) { return a * (1.0f / b); }
CR_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CR_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
CR_HD float lengthSquared(V3 a) { return dot(a, a); }
CR_D float length(V3 a) { return sqrtf(lengthSquared(a)); }
CR_D V3 normalize(V3 a) { const float l = length(a); return l > 0 ? a / l : V3{}; }
CR_D bool finite3(V3 a) { return isfin(a.x) && isfin(a.y) && isfin(a.z); }
CR_HD bool nonzero(V3 v) { return v.x != 0 || v.y != 0 || v.z != 0; }
CR_HD float maxComponent(V3 a) { return smax3(a.x, a.y, a.z); }
CR_HD float luminance(V3 a) { return dot(a, {0.2126f, 0.7152f, 0.0722f}); }
CR_HD V3 mix(V3 a, V3 b, float t) { return a * (1 - t) + b * t; }
CR_D V3 vexp(V3 a) { return {fexp(a.x), fexp(a.y), fexp(a.z)}; }
CR_HD V3 reflect(V3 i, V3 n) { return i - 2 * dot(i, n) * n; }
CR_HD V3 vclamp(V3 a, float lo, float hi) { return {sclamp(a.x, lo, hi), sclamp(a.y, lo, hi), sclamp(a.z, lo, hi)}; }
CR_HD V3 v3(const float* p) { return {p[0], p[1], p[2]}; }
CR_HD V3 v3(float4 p) { return {p.x, p.y, p.z}; }

// Orthonormal shading basis (math.h:95-103).
struct Frame {
    V3 x, y, z;
    CR_D explicit Frame(V3 normal) : z(normal) {
        x = normalize(cross(fabsf(z.z) < 0.999f ? V3{0, 0, 1} : V3{0, 1, 0}, z));
        y = cross(z, x);
    }
    CR_D V3 local(V3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    CR_D V3 world(V3 v) const { return x * v.x + y * v.y + z * v.z; }
};

// ---- DVec3 (geometry.cpp:17-47) ---------------------------------------------------------
struct D3 {
    double x, y, z;
    CR_HD D3() : x(0), y(0), z(0) {}
    CR_HD explicit D3(V3 v) : x(v.x), y(v.y), z(v.z) {}
    CR_HD D3(double a, double b, double c) : x(a), y(b), z(c) {}
    CR_HD double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
CR_HD D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
CR_HD D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
CR_HD D3 operator*(D3 a, double b) { return {a.x * b, a.y * b, a.z * b}; }
CR_HD double pdot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CR_HD D3 pcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
CR_D V3 unit(D3 v, V3 fallback = V3{}) {
    const double squared = pdot(v, v);
    if (!(squared > 0) || !isfin(squared)) return fallback;
    const double inverse = 1 / sqrt(squared);
    return {static_cast<float>(v.x * inverse), static_cast<float>(v.y * inverse), static_cast<float>(v.z * inverse)};
}
CR_D V3 unit(V3 v, V3 fallback = V3{}) { return unit(D3(v), fallback); }
CR_D V3 orthogonalized(D3 v, V3 n, V3 fallback = V3{}) {
    const double normalSquared = pdot(D3(n), D3(n));
    if (!(normalSquared > 0)) return fallback;
    const D3 projected = v - D3(n) * (pdot(v, D3(n)) / normalSquared);
    constexpr double tolerance = 4 * static_cast<double>(kFltEps);
    if (pdot(projected, projected) <= pdot(v, v) * tolerance * tolerance) return fallback;
    return unit(projected, fallback);
}

// ---- RNG (math.h:104-121) ---------------------------------------------------------------
constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ULL;
struct Rng {
    uint64_t state;
    CR_HD explicit Rng(uint64_t seed) : state(seed) {}
    CR_HD uint32_t next() {
        state += kGolden;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return static_cast<uint32_t>((z ^ (z >> 31)) >> 32);
    }
    CR_HD float uniform() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
};
CR_HD uint64_t sampleSeed(uint64_t seed, uint64_t pixel, uint64_t sample) {
    Rng hash(seed ^ (pixel * 0xd2b74407b1ce6e93ULL) ^ (sample * 0xca5a826395121157ULL));
    const uint64_t hi = hash.next();
    return (hi << 32) | hash.next();
}
// MIS power heuristic (math.h:124-128).
CR_D float powerHeuristic(float a, float b) {
    if (a <= 0) return 0;
    const double aa = static_cast<double>(a) * a, bb = static_cast<double>(b) * b;
    return static_cast<float>(aa / (aa + bb));
}

}  // namespace crg
