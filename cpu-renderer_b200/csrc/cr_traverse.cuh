// Closest-hit and any-hit BVH traversal (CPU-Renderer src/geometry.cpp:147-182, 554-639).
//
// Two traversals share one node layout (NodePair) and one triangle decision:
//
//  * intersect_exact  — the reference's Bvh::intersect restated in FP64: the same widened
//    slab test, the same child order and stack discipline, the same leaf loop. Used for
//    precise-replay rays (non-zero originLow), rays with sub-1e-30 direction components,
//    and on request (cr_gpu_tuning::exact_traversal).
//
//  * intersect_fast   — FP32 slab tests made conservative (every box the exact test accepts
//    is accepted, see box_fast), near-first order, and an FP32 watertight edge-function
//    prefilter with a rigorous error bound that only discards triangles the FP64 test
//    would also reject. Every candidate that survives is decided by tri_exact, the
//    reference's FP64 arithmetic. The closest hit is the minimum (t, index) over accepted
//    candidates; visiting a superset of the boxes therefore yields the same triangle, t, u
//    and v as the reference (ties on t go to the lower index, geometry.cpp:609).
#pragma once
#include "cr_dev_math.cuh"
#include "cr_internal.h"

namespace crg {

struct TRay {
    V3 o, d;
    float tmin, tmax;
    V3 olow;
};

struct HitRec {
    double t, u, v;
    uint32_t tri;
    uint32_t flags;  // kTri* flags of the hit triangle
};

// validRay (geometry.cpp:52-55).
CR_D bool validRay(const TRay& r) {
    return finite3(r.o) && finite3(r.olow) && finite3(r.d) && nonzero(r.d) &&
           !isnan(r.tmin) && !isnan(r.tmax) && r.tmin <= r.tmax;
}

// ---- the reference's triangle arithmetic (geometry.cpp:154-181) ---------------------------
struct ExactSetup {
    int kx, ky, kz;
    double sx, sy, sz;
    D3 origin;
};
CR_D ExactSetup exact_setup(const TRay& r) {
    ExactSetup e;
    int kz = 0;
    if (fabsf(r.d.y) > fabsf(r.d[kz])) kz = 1;
    if (fabsf(r.d.z) > fabsf(r.d[kz])) kz = 2;
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (r.d[kz] < 0) { const int t = kx; kx = ky; ky = t; }
    e.kx = kx; e.ky = ky; e.kz = kz;
    e.sx = static_cast<double>(r.d[kx]) / r.d[kz];
    e.sy = static_cast<double>(r.d[ky]) / r.d[kz];
    e.sz = 1.0 / r.d[kz];
    e.origin = D3(r.o) + D3(r.olow);
    return e;
}
// Returns true and t (plus w1, w2, det for u = w1/det, v = w2/det) when the reference's
// intersectTriangle would accept the triangle on [tmin, limit].
CR_D bool tri_exact(const ExactSetup& E, V3 p0, V3 p1, V3 p2, double tmin, double limit,
                    double& t, double& w1o, double& w2o, double& deto) {
    const D3 a = D3(p0) - E.origin, b = D3(p1) - E.origin, c = D3(p2) - E.origin;
    const double akz = a[E.kz], bkz = b[E.kz], ckz = c[E.kz];
    const double ax = a[E.kx] - E.sx * akz, ay = a[E.ky] - E.sy * akz;
    const double bx = b[E.kx] - E.sx * bkz, by = b[E.ky] - E.sy * bkz;
    const double cx = c[E.kx] - E.sx * ckz, cy = c[E.ky] - E.sy * ckz;
    const double w0 = cx * by - cy * bx, w1 = ax * cy - ay * cx, w2 = bx * ay - by * ax;
    if ((w0 < 0 || w1 < 0 || w2 < 0) && (w0 > 0 || w1 > 0 || w2 > 0)) return false;
    const double det = w0 + w1 + w2;
    if (det == 0 || !isfin(det)) return false;
    const double tt = (w0 * (E.sz * akz) + w1 * (E.sz * bkz) + w2 * (E.sz * ckz)) / det;
    if (!isfin(tt) || fabs(tt) > static_cast<double>(kFltMax) || tt < tmin || tt > limit) return false;
    t = tt; w1o = w1; w2o = w2; deto = det;
    return true;
}

// Scene::accepts sidedness rule (geometry.cpp:282-286); alpha masks are handled by the
// caller through accepts_alpha.
CR_D bool accepts_cull(const DevScene& S, uint32_t tri, V3 dir) {
    const float4 n = S.tri_ng[tri];
    return !(pdot(D3(V3{n.x, n.y, n.z}), D3(dir)) >= 0);
}

// Implemented in cr_shade.cuh (needs the texture sampler).
CR_D bool accepts_alpha(const DevScene& S, uint32_t tri, double u, double v);

// NOALPHA: the scene has no alpha-masked triangle (no kTriAlphaMask flag is set), so the
// instantiation leaves the texture lookup of the alpha test out of the traversal.
template <bool NOALPHA = false>
CR_D bool accepts(const DevScene& S, uint32_t tri, uint32_t flags, V3 dir, double w1, double w2, double det) {
    if ((flags & kTriCull) && !accepts_cull(S, tri, dir)) return false;
    if (!NOALPHA && (flags & kTriAlphaMask)) return accepts_alpha(S, tri, w1 / det, w2 / det);
    return true;
}

CR_D void load_pair(const NodePair* pairs, uint32_t p, float4& a, float4& b, float4& c, uint4& d) {
    const float4* q = reinterpret_cast<const float4*>(pairs + p);
    a = __ldg(q); b = __ldg(q + 1); c = __ldg(q + 2);
    d = __ldg(reinterpret_cast<const uint4*>(q + 3));
}

// ---- exact traversal (geometry.cpp:554-639) ------------------------------------------------
// Optional visit counters (node pairs fetched, triangles tested) for the roofline numerator.
struct VisitCount { uint32_t pairs = 0, tris = 0; };

template <bool ANY, bool COUNT = false, bool NOALPHA = false>
__device__ bool intersect_exact(const DevScene& S, const TRay& ray, double hitT, uint32_t ignore,
                                HitRec& hit, int& err, VisitCount* vc = nullptr) {
    double closestLimit = smin(static_cast<double>(ray.tmax), hitT);
    float ctmax = smin(ray.tmax, next_up(static_cast<float>(closestLimit)));
    const float queryLimit = ctmax;
    if (queryLimit < ray.tmin) return false;
    const ExactSetup E = exact_setup(ray);
    double inv[3] = {0, 0, 0};
    const D3 po = E.origin;
    for (int ax = 0; ax < 3; ++ax) if (ray.d[ax] != 0) inv[ax] = 1.0 / ray.d[ax];
    const double boxErr = 4 * kDblEps;
    auto box = [&](float lx, float ly, float lz, float hx, float hy, float hz, float& nearD) -> bool {
        double nearT = ray.tmin, farT = ctmax;
        const float lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz};
#pragma unroll
        for (int axis = 0; axis < 3; ++axis) {
            const double origin = po[axis];
            if (ray.d[axis] == 0) {
                if (origin < lo[axis] || origin > hi[axis]) return false;
                continue;
            }
            double a = (static_cast<double>(lo[axis]) - origin) * inv[axis];
            double b = (static_cast<double>(hi[axis]) - origin) * inv[axis];
            if (inv[axis] < 0) { const double t = a; a = b; b = t; }
            a -= fabs(a) * boxErr;
            b += fabs(b) * boxErr;
            nearT = smax(nearT, a);
            farT = smin(farT, b);
            if (nearT > farT) return false;
        }
        nearD = smax(ray.tmin, next_down(static_cast<float>(nearT)));
        return true;
    };
    float rootNear = 0;
    if (!box(S.root_lo[0], S.root_lo[1], S.root_lo[2], S.root_hi[0], S.root_hi[1], S.root_hi[2], rootNear)) return false;
    constexpr int kRefStack = 50;  // maxBvhDepth + 2 entries (geometry.cpp:590)
    uint32_t stRef[kRefStack], stCnt[kRefStack];
    float stNear[kRefStack];
    int size = 0;
    stRef[0] = S.root_ref; stCnt[0] = S.root_count; stNear[0] = rootNear; size = 1;
    bool found = false;
    double bestW1 = 0, bestW2 = 0, bestDet = 1;
    while (size) {
        --size;
        const uint32_t ref = stRef[size], cnt = stCnt[size];
        const float entryNear = stNear[size];
        if (entryNear > ctmax) continue;
        if (cnt) {
            for (uint32_t i = ref; i < ref + cnt; ++i) {
                const float4 q0 = __ldg(S.tri_pos + 3 * static_cast<uint64_t>(i));
                if (COUNT) ++vc->tris;
                const uint32_t index = __float_as_uint(q0.w);
                if (index == ignore) continue;
                const float4 q1 = __ldg(S.tri_pos + 3 * static_cast<uint64_t>(i) + 1);
                const float4 q2 = __ldg(S.tri_pos + 3 * static_cast<uint64_t>(i) + 2);
                const double limit = smin(static_cast<double>(ctmax), closestLimit);
                if (limit < ray.tmin) continue;
                double t, w1, w2, det;
                if (!tri_exact(E, v3(q0), v3(q1), v3(q2), ray.tmin, limit, t, w1, w2, det)) continue;
                if (!accepts<NOALPHA>(S, index, __float_as_uint(q1.w), ray.d, w1, w2, det)) continue;
                if (ANY) { hit.t = t; hit.u = w1 / det; hit.v = w2 / det; hit.tri = index; hit.flags = __float_as_uint(q1.w); return true; }
                if (!found || t < hit.t || (t == hit.t && index < hit.tri)) {
                    hit.t = t; hit.tri = index; hit.flags = __float_as_uint(q1.w); bestW1 = w1; bestW2 = w2; bestDet = det;
                    closestLimit = t;
                    ctmax = smin(queryLimit, next_up(static_cast<float>(t)));
                    found = true;
                }
            }
        } else {
            float4 a, b, c; uint4 d;
            load_pair(S.pairs, ref, a, b, c, d);
            if (COUNT) ++vc->pairs;
            float leftNear = 0, rightNear = 0;
            const bool left = box(a.x, a.y, a.z, a.w, b.x, b.y, leftNear);
            const bool right = box(b.z, b.w, c.x, c.y, c.z, c.w, rightNear);
            if (size + static_cast<int>(left) + static_cast<int>(right) > kRefStack) { err = kErrStackOverflow; return found; }
            if (left && right) {
                if (leftNear <= rightNear) {
                    stRef[size] = d.z; stCnt[size] = d.w; stNear[size] = rightNear; ++size;
                    stRef[size] = d.x; stCnt[size] = d.y; stNear[size] = leftNear; ++size;
                } else {
                    stRef[size] = d.x; stCnt[size] = d.y; stNear[size] = leftNear; ++size;
                    stRef[size] = d.z; stCnt[size] = d.w; stNear[size] = rightNear; ++size;
                }
            } else if (left) { stRef[size] = d.x; stCnt[size] = d.y; stNear[size] = leftNear; ++size; }
            else if (right) { stRef[size] = d.z; stCnt[size] = d.w; stNear[size] = rightNear; ++size; }
        }
    }
    if (found) { hit.u = bestW1 / bestDet; hit.v = bestW2 / bestDet; }
    return found;
}

// ---- fast traversal ----------------------------------------------------------------------
// Relative slack on FP32 slab distances: each t = (plane - origin) * (1/d) carries three
// roundings (|error| <= 3u|t|, u = 2^-24); 2^-20 covers that five times over, plus the FP64
// triangle test's own error, which is ~1e-16 relative. The absolute term covers products
// that underflow. Widening only ever adds boxes.
constexpr float kBoxRel = 9.5367431640625e-07f;  // 2^-20
constexpr float kBoxAbs = 1e-30f;

struct FastSetup {
    V3 o, inv;
    int kx, ky, kz;
    float Sx, Sy;
    uint32_t zeroAxes;  // bit a set when direction component a is exactly zero
};

// Rays whose FP32 setup is well conditioned: no precise origin, and no direction component
// that is non-zero but below 1e-30 (its FP32 reciprocal could overflow to infinity).
CR_D bool fast_eligible(const TRay& r) {
    if (nonzero(r.olow)) return false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float d = fabsf(r.d[a]);
        if (d != 0.0f && d < 1e-30f) return false;
    }
    return true;
}

CR_D FastSetup fast_setup(const TRay& r) {
    FastSetup f;
    f.o = r.o;
    f.inv = V3{r.d.x != 0 ? 1.0f / r.d.x : 0.0f, r.d.y != 0 ? 1.0f / r.d.y : 0.0f, r.d.z != 0 ? 1.0f / r.d.z : 0.0f};
    f.zeroAxes = (r.d.x == 0 ? 1u : 0u) | (r.d.y == 0 ? 2u : 0u) | (r.d.z == 0 ? 4u : 0u);
    int kz = 0;
    if (fabsf(r.d.y) > fabsf(r.d[kz])) kz = 1;
    if (fabsf(r.d.z) > fabsf(r.d[kz])) kz = 2;
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (r.d[kz] < 0) { const int t = kx; kx = ky; ky = t; }
    f.kx = kx; f.ky = ky; f.kz = kz;
    f.Sx = r.d[kx] / r.d[kz];
    f.Sy = r.d[ky] / r.d[kz];
    return f;
}

// Conservative FP32 slab test. Returns the (lowered) entry distance in tnear. An axis with a
// zero direction component constrains nothing in t; it only requires the origin to lie in
// the slab, compared exactly as the reference does (geometry.cpp:569-571).
CR_D bool box_fast(const FastSetup& F, float lx, float ly, float lz, float hx, float hy, float hz,
                   float tmin, float tmax, float& tnear) {
    const float t0x = (lx - F.o.x) * F.inv.x, t1x = (hx - F.o.x) * F.inv.x;
    const float t0y = (ly - F.o.y) * F.inv.y, t1y = (hy - F.o.y) * F.inv.y;
    const float t0z = (lz - F.o.z) * F.inv.z, t1z = (hz - F.o.z) * F.inv.z;
    float nx = fminf(t0x, t1x), fx = fmaxf(t0x, t1x);
    float ny = fminf(t0y, t1y), fy = fmaxf(t0y, t1y);
    float nz = fminf(t0z, t1z), fz = fmaxf(t0z, t1z);
    if (F.zeroAxes) {
        if (F.zeroAxes & 1u) { if (F.o.x < lx || F.o.x > hx) return false; nx = -kInf; fx = kInf; }
        if (F.zeroAxes & 2u) { if (F.o.y < ly || F.o.y > hy) return false; ny = -kInf; fy = kInf; }
        if (F.zeroAxes & 4u) { if (F.o.z < lz || F.o.z > hz) return false; nz = -kInf; fz = kInf; }
    }
    float tn = fmaxf(fmaxf(nx, ny), nz);
    float tf = fminf(fminf(fx, fy), fz);
    // one rounding fewer than tn - |tn| kBoxRel: the widening needs ~0.2 of its 2^-20, so how
    // its own product rounds does not matter
    tn = __fmaf_rn(-fabsf(tn), kBoxRel, tn) - kBoxAbs;
    tf = __fmaf_rn(fabsf(tf), kBoxRel, tf) + kBoxAbs;
    tn = fmaxf(tn, tmin);
    tf = fminf(tf, tmax);
    tnear = tn;
    return tn <= tf;
}

CR_D float pick(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// FP32 watertight edge functions with a forward error bound (after Woop, Benthin and Wald,
// "Watertight Ray/Triangle Intersection", JCGT 2013, and the bound of Pharr, Jakob and
// Humphreys, PBRT 3rd ed. section 3.9.6). Returns true only when the three edge functions
// have mixed signs by more than their error, i.e. when the FP64 test must reject too.
CR_D bool tri_reject_fast(const FastSetup& F, float4 p0, float4 p1, float4 p2) {
    const float ox = F.o[F.kx], oy = F.o[F.ky], oz = F.o[F.kz];
    const float axk = pick(p0, F.kx) - ox, ayk = pick(p0, F.ky) - oy, azk = pick(p0, F.kz) - oz;
    const float bxk = pick(p1, F.kx) - ox, byk = pick(p1, F.ky) - oy, bzk = pick(p1, F.kz) - oz;
    const float cxk = pick(p2, F.kx) - ox, cyk = pick(p2, F.ky) - oy, czk = pick(p2, F.kz) - oz;
    const float ax = __fmaf_rn(-F.Sx, azk, axk), ay = __fmaf_rn(-F.Sy, azk, ayk);
    const float bx = __fmaf_rn(-F.Sx, bzk, bxk), by = __fmaf_rn(-F.Sy, bzk, byk);
    const float cx = __fmaf_rn(-F.Sx, czk, cxk), cy = __fmaf_rn(-F.Sy, czk, cyk);
    const float w0 = __fmaf_rn(cx, by, -(cy * bx));
    const float w1 = __fmaf_rn(ax, cy, -(ay * cx));
    const float w2 = __fmaf_rn(bx, ay, -(by * ax));
    const float mz = fmaxf(fmaxf(fabsf(azk), fabsf(bzk)), fabsf(czk));
    const float mxk = fmaxf(fmaxf(fabsf(axk), fabsf(bxk)), fabsf(cxk));
    const float myk = fmaxf(fmaxf(fabsf(ayk), fabsf(byk)), fabsf(cyk));
    const float mx = fmaxf(fmaxf(fabsf(ax), fabsf(bx)), fabsf(cx));
    const float my = fmaxf(fmaxf(fabsf(ay), fabsf(by)), fabsf(cy));
    constexpr float g = 6e-7f;  // twice gamma(5) for u = 2^-24
    const float dx = g * (mxk + mz), dy = g * (myk + mz);
    const float dw = 4.0f * ((mx + dx) * dy + (my + dy) * dx + g * (mx + dx) * (my + dy)) + 1e-30f;
    return (w0 < -dw || w1 < -dw || w2 < -dw) && (w0 > dw || w1 > dw || w2 > dw);
}

// The fast traversal in the "while-while" form of Aila and Laine ("Understanding the
// Efficiency of Ray Traversal on GPUs", HPG 2009): an inner loop walks interior nodes and
// postpones the first leaf it reaches, continuing speculatively until every lane of the warp
// holds a leaf; then all lanes test their leaf's triangles together. Lanes therefore run the
// node code and the triangle code in separate loops instead of alternating per iteration.
template <bool ANY, bool COUNT = false, bool NOALPHA = false>
__device__ bool intersect_fast(const DevScene& S, const TRay& ray, double hitT, uint32_t ignore,
                               HitRec& hit, int& err, VisitCount* vc = nullptr) {
    double closestLimit = smin(static_cast<double>(ray.tmax), hitT);
    float ctmax = smin(ray.tmax, next_up(static_cast<float>(closestLimit)));
    const float queryLimit = ctmax;
    if (queryLimit < ray.tmin) return false;
    const FastSetup F = fast_setup(ray);
    const ExactSetup E = exact_setup(ray);
    float rootNear;
    if (!box_fast(F, S.root_lo[0], S.root_lo[1], S.root_lo[2], S.root_hi[0], S.root_hi[1], S.root_hi[2],
                  ray.tmin, ctmax, rootNear)) return false;
    uint32_t stRef[kStackSize], stCnt[kStackSize];
    float stNear[kStackSize];
    int size = 0;
    uint32_t ref = S.root_ref, cnt = S.root_count;   // current node (interior: cnt == 0)
    bool haveNode = true;
    uint32_t leafRef = 0, leafCnt = 0;               // postponed leaf
    bool found = false;
    double bestW1 = 0, bestW2 = 0, bestDet = 1;
    // next stack entry whose entry distance is still inside the current interval
    auto pop = [&]() -> bool {
        while (size > 0) {
            --size;
            if (stNear[size] <= ctmax) { ref = stRef[size]; cnt = stCnt[size]; return true; }
        }
        return false;
    };
    for (;;) {
        if (haveNode && cnt && !leafCnt) { leafRef = ref; leafCnt = cnt; haveNode = pop(); }
        while (haveNode && cnt == 0) {
            float4 a, b, c; uint4 d;
            load_pair(S.pairs, ref, a, b, c, d);
            if (COUNT) ++vc->pairs;
            float n0, n1;
            const bool h0 = box_fast(F, a.x, a.y, a.z, a.w, b.x, b.y, ray.tmin, ctmax, n0);
            const bool h1 = box_fast(F, b.z, b.w, c.x, c.y, c.z, c.w, ray.tmin, ctmax, n1);
            if (h0 && h1) {
                if (size >= kStackSize) { err = kErrStackOverflow; return found; }
                const bool firstNear = n0 <= n1;
                stRef[size] = firstNear ? d.z : d.x; stCnt[size] = firstNear ? d.w : d.y;
                stNear[size] = firstNear ? n1 : n0; ++size;
                ref = firstNear ? d.x : d.z; cnt = firstNear ? d.y : d.w;
            } else if (h0) { ref = d.x; cnt = d.y; }
            else if (h1) { ref = d.z; cnt = d.w; }
            else haveNode = pop();
            if (haveNode && cnt && !leafCnt) { leafRef = ref; leafCnt = cnt; haveNode = pop(); }
            if (__all_sync(__activemask(), leafCnt != 0)) break;
        }
        for (; leafCnt; ++leafRef, --leafCnt) {
            const float4* q = S.tri_pos + 3 * static_cast<uint64_t>(leafRef);
            const float4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
            if (COUNT) ++vc->tris;
            const uint32_t index = __float_as_uint(q0.w);
            if (index == ignore) continue;
            if (tri_reject_fast(F, q0, q1, q2)) continue;
            const double limit = smin(static_cast<double>(ctmax), closestLimit);
            if (limit < ray.tmin) continue;
            double t, w1, w2, det;
            if (!tri_exact(E, v3(q0), v3(q1), v3(q2), ray.tmin, limit, t, w1, w2, det)) continue;
            if (!accepts<NOALPHA>(S, index, __float_as_uint(q1.w), ray.d, w1, w2, det)) continue;
            if (ANY) { hit.t = t; hit.u = w1 / det; hit.v = w2 / det; hit.tri = index; hit.flags = __float_as_uint(q1.w); return true; }
            if (!found || t < hit.t || (t == hit.t && index < hit.tri)) {
                hit.t = t; hit.tri = index; hit.flags = __float_as_uint(q1.w); bestW1 = w1; bestW2 = w2; bestDet = det;
                closestLimit = t;
                ctmax = smin(queryLimit, next_up(static_cast<float>(t)));
                found = true;
            }
        }
        if (!haveNode) break;
    }
    if (found) { hit.u = bestW1 / bestDet; hit.v = bestW2 / bestDet; }
    return found;
}

// Bvh::intersect entry: the reference's preconditions (geometry.cpp:555), then the traversal
// that fits the ray.
template <bool ANY, bool COUNT = false, bool NOALPHA = false>
__device__ bool intersect(const DevScene& S, const TRay& ray, double hitT, uint32_t ignore, bool forceExact,
                          HitRec& hit, int& err, VisitCount* vc = nullptr) {
    if (!S.has_root || !validRay(ray) || isnan(hitT)) return false;
    if (forceExact || !fast_eligible(ray)) return intersect_exact<ANY, COUNT, NOALPHA>(S, ray, hitT, ignore, hit, err, vc);
    return intersect_fast<ANY, COUNT, NOALPHA>(S, ray, hitT, ignore, hit, err, vc);
}

}  // namespace crg
