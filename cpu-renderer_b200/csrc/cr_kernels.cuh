// Device code of the path tracer: per-path functions (camera sample, closest/any hit, one
// bounce of trace()) and the kernels that run them over the path pool. Included by the
// single-render driver (cr_render.cu) and the multi-job engine (cr_engine.cu); kernels that
// both use are templates or static, so each translation unit holds its own instantiation.
#pragma once
#include "cr_shade.cuh"
#include "cr_guide.cuh"

// Minimum resident blocks per SM requested from the register allocator (128-thread blocks).
// k_trace at 12 (40 registers, some spills to L1) measured ~2 % faster than at 8 or 10 on
// the 1M-triangle workload; k_shade above 4 loses more to spills than it gains (also per
// class: the miss kernel at 8 measured slower; the NEE-null kernel, at 110 registers since it
// samples only the BSDF's delta branches, measured the same at 5 and 6 as at 4).
#ifndef CR_TRACE_MIN_BLOCKS
#define CR_TRACE_MIN_BLOCKS 12
#endif
#ifndef CR_SHADE_MIN_BLOCKS
#define CR_SHADE_MIN_BLOCKS 4
#endif

namespace crg {

// A chunk of consecutive sample ids [c0, c1) (id = sample * pixels + pixel); out[] holds the
// radiance of id at j = id - c0, its position in the chunk. Where the chunk is whole samples
// per pixel (spp > 0: samples [s0, s0 + spp) of every pixel) its ids are issued pixel-major:
// position j starts sample s0 + j % spp of pixel j / spp, so the consecutive path slots that
// form a warp start samples of one pixel and trace nearly the same rays for longer (a smooth
// dielectric or a mirror sends them the same way). Either order, each pixel's samples are
// summed in sample order, so the film does not depend on it. A pixel-major chunk may also
// cover a block of pixels only, [p0, p0 + (c1 - c0) / spp): then it holds every sample of them.
struct Chunk {
    uint64_t c0, c1, pixels;
    uint32_t spp = 0, s0 = 0;  // spp 0: sample-major positions
    uint32_t p0 = 0;           // pixel-major: the first pixel
};

// Where a path's sample radiance goes: out[base + sample * sampleStride + pixel * pixelStride].
struct OutRef {
    uint64_t base, sampleStride, pixelStride;
};
CR_D OutRef outOf(const Chunk& C) {
    if (C.spp) return OutRef{0ull - C.s0 - static_cast<uint64_t>(C.p0) * C.spp, 1, C.spp};
    return OutRef{0ull - C.c0, C.pixels, 1};
}
// out[] index of a pixel's sample
CR_D uint64_t outIndex(const OutRef& O, uint32_t pixel, uint32_t sample) {
    return O.base + static_cast<uint64_t>(sample) * O.sampleStride + static_cast<uint64_t>(pixel) * O.pixelStride;
}

// The pixel and sample that position j of the chunk starts.
CR_D void chunkSample(const Chunk& C, uint64_t j, uint32_t& pixel, uint32_t& sample) {
    if (C.spp) {
        pixel = C.p0 + static_cast<uint32_t>(j / C.spp);
        sample = C.s0 + static_cast<uint32_t>(j % C.spp);
    } else {
        const uint64_t id = C.c0 + j;
        pixel = static_cast<uint32_t>(id % C.pixels);
        sample = static_cast<uint32_t>(id / C.pixels);
    }
}

// ---- multi-job pool ----------------------------------------------------------------------------
// In the multi-job engine the paths of many renders (jobs: scene, camera, options) share one
// pool. The host appends sample ranges of its jobs to an issue list; free slots take the next
// positions of the list. Each path remembers its range, which names its job's scene and
// parameters, where its radiance goes, and the counter of finished samples the host polls.
struct IssueRange {
    uint64_t start;    // position of the range's first sample in the issue list
    uint64_t c0, c1;   // the job's sample ids [c0, c1), numbered as in a single render
    uint64_t outBase;  // out[] index of the range's first position
    uint64_t pixels;   // the job's width * height
    uint32_t job;      // job slot
    uint32_t spp;      // > 0: samples [s0, s0 + spp) of every pixel from p0 on, issued pixel-major (see Chunk)
    uint32_t s0;
    uint32_t p0;
};
// The range as a chunk (its positions map to pixels and samples the same way).
CR_HD Chunk rangeChunk(const IssueRange& R) {
    Chunk C{R.c0, R.c1, R.pixels};
    C.spp = R.spp;
    C.s0 = R.s0;
    C.p0 = R.p0;
    return C;
}
struct JobTable {
    const DevScene* scenes;          // [job slot]
    const RenderParams* params;      // [job slot]
    const IssueRange* ranges;        // the issue list
    const unsigned long long* ctl;   // [0] issue end: positions below it may start; [1] range count
    unsigned long long* issued;      // [2] next issue position, ping-pong by iteration parity
    unsigned long long* done;        // [range] finished samples
    unsigned long long* errKeys;     // [job slot] smallest error key
    unsigned long long* retries;     // [job slot] precision replays
    uint2* slot;                     // [path slot] the path's range (x) and job slot (y), one
                                     // load ahead of its scene's fields
    uint32_t refillMin;              // refill only when at least this many slots are free
    // The pool's free slots, a ring over `ring` (capacity `poolSize`): k_regen claims from the
    // head (ping-pong by iteration parity, so every block of a launch reads the same head),
    // k_trace and k_shade append the slots their paths free at the tail. k_regen never appends,
    // so the tail it reads is the same for all its blocks.
    uint32_t* ring;
    unsigned long long* head;        // [2]
    unsigned long long* tail;
    uint64_t poolSize;
};
// All 32 lanes call this together: lanes with pred append slot to the pool's free ring.
CR_D void ringPush(const JobTable& J, bool pred, uint32_t slot) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(J.tail, static_cast<unsigned long long>(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) J.ring[(base + __popc(mask & ((1u << lane) - 1u))) % J.poolSize] = slot;
}

// kStatIterations: pool iterations started (k_regen counts them; read by the ray dump).
enum { kStatRetries = 0, kStatExtendRays = 1, kStatShadowRays = 2, kStatErrorKey = 3, kStatPairs = 4, kStatTris = 5,
       kStatIssued = 6, kStatShadowPairs = 7, kStatShadowTris = 8, kStatIterations = 9, kStatWords = 12 };

CR_D uint64_t errorKey(const RenderParams& P, uint32_t pixel, uint32_t sample) {
    const uint32_t x = pixel % static_cast<uint32_t>(P.width), y = pixel / static_cast<uint32_t>(P.width);
    const uint64_t tilesX = (static_cast<uint64_t>(P.width) + 15) / 16;
    const uint64_t rank = ((y / 16) * tilesX + x / 16) * 256 + (y % 16) * 16 + (x % 16);
    return (rank << 21) | sample;
}

// Error sink: the smallest key is kept for the report; when detail is set (single-sample
// re-run), the full record is written there.
struct ErrSink {
    unsigned long long* minKey;
    DevError* detail;
};
CR_D void raise(const ErrSink& E, const RenderParams& P, uint32_t pixel, uint32_t sample, int code) {
    atomicMin(E.minKey, static_cast<unsigned long long>(errorKey(P, pixel, sample)));
    if (E.detail) {
        E.detail->code = code;
        E.detail->x = static_cast<int32_t>(pixel % static_cast<uint32_t>(P.width));
        E.detail->y = static_cast<int32_t>(pixel / static_cast<uint32_t>(P.width));
        E.detail->sample = static_cast<int32_t>(sample);
        E.detail->key = errorKey(P, pixel, sample);
    }
}

// All 32 lanes call this together; lanes with pred append value to the queue.
CR_D void warpPush(uint32_t* queue, uint32_t* counter, bool pred, uint32_t value) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) queue[base + __popc(mask & ((1u << lane) - 1u))] = value;
}

CR_D float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// Work distribution of the queue-driven kernels: each warp takes the next 32 queue entries from
// a counter as it becomes free, so warps whose rays finish early take more and a launch ends
// when its work does, not when the warp with the longest fixed share does. Returns the first
// entry of the warp's batch (all lanes get the same value).
CR_D uint32_t warpTake(uint32_t* counter) {
    uint32_t base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(counter, 32u);
    return __shfl_sync(0xffffffffu, base, 0);
}

// render.cpp:396-401 plus trace()'s initial state (render.cpp:235-239).
CR_D bool initPath(const DevScene& S, const RenderParams& P, const PathSoA& st, uint32_t slot, uint32_t pixel,
                   uint32_t sample, bool precise, const ErrSink& E) {
    Rng rng(sampleSeed(P.seed, pixel, sample));
    const uint32_t x = pixel % static_cast<uint32_t>(P.width), y = pixel / static_cast<uint32_t>(P.width);
    const float dx = rng.uniform(), dy = rng.uniform();
    TRay ray;
    if (!cameraRay(P.camera, P.width, P.height, static_cast<float>(x) + dx, static_cast<float>(y) + dy, ray)) {
        raise(E, P, pixel, sample, kErrUnrepresentableCameraRay);
        return false;
    }
    st.ray_o[slot] = f4(ray.o, ray.tmin);
    st.ray_d[slot] = f4(ray.d, ray.tmax);
    if (precise) st.ray_lo[slot] = make_float4(0, 0, 0, 0);  // read only for precise rays
    st.thr[slot] = make_float4(1, 1, 1, 1);          // throughput 1, etaScale 1
    st.rad[slot] = make_float4(0, 0, 0, 0);          // radiance 0, lastPdf 0
    // last_pos needs no value yet: it is read only after a non-delta bounce, which writes it
    st.absorb[slot] = make_float4(0, 0, 0, __int_as_float(-1));  // medium -1
    st.flags[slot] = kPathLastDelta | (precise ? kPathPrecise : 0u);
    st.rng[slot] = rng.state;
    st.prev_tri[slot] = kNoTriangle;
    st.pixel[slot] = pixel;
    st.sample[slot] = sample;
    st.depth[slot] = 0;
    if (st.guide.count) st.guide.count[slot] = 0;
    return true;
}

CR_D TRay loadRay(const PathSoA& st, uint32_t path, uint32_t flags) {
    const float4 o = st.ray_o[path], d = st.ray_d[path];
    TRay r;
    r.o = v3(o); r.tmin = o.w; r.d = v3(d); r.tmax = d.w;
    r.olow = (flags & kPathPrecise) ? v3(st.ray_lo[path]) : V3{};
    return r;
}

// Ends a path: the reference's final radiance check (render.cpp:346), then the sample output.
CR_D void finishPath(const RenderParams& P, const OutRef& O, const PathSoA& st, uint32_t path, V3 R, const ErrSink& E) {
    const uint32_t pixel = st.pixel[path], sample = st.sample[path];
    if (!finite3(R) || smin3(R.x, R.y, R.z) < 0) {
        raise(E, P, pixel, sample, kErrNonFiniteRadiance);
        R = V3{};
    }
    st.out[outIndex(O, pixel, sample)] = f4(R, 0);
    if (st.guide.count) guideFinish(st.guide, path, R);
}

// One iteration of trace()'s bounce loop (render.cpp:240-344) for one path, after its
// closest hit is known. cont: the path continues; shadow: a shadow ray was queued (a path
// that ends with a queued shadow ray is finished by k_trace next iteration); freed: the path
// ended and its slot can take a new sample. CLASS specialises the code: kShadeMiss holds only
// environment misses, kShadeNeeNull only hits on kTriNeeNull surfaces (the BSDF's delta
// branches alone), kShadeConductor only hits on kTriConductor surfaces (the BSDF without its
// zero lobes), kShadeGeneric anything.
template <int CLASS, bool GUIDED = false, bool LEAN = false>
CR_D void shadeOne(const DevScene& S, const RenderParams& P, const OutRef& O, const PathSoA& st, uint32_t path,
                   const ErrSink& E, unsigned long long* retries, bool& cont, bool& shadow, bool& freed) {
    cont = false; shadow = false; freed = false;
    uint32_t flags = st.flags[path];
    const bool precise = flags & kPathPrecise;
    const TRay ray = loadRay(st, path, flags);
    const float4 th = st.thr[path], ra = st.rad[path], ab = st.absorb[path];
    V3 T = v3(th), R = v3(ra), A = v3(ab);
    float etaScale = th.w, lastPdf = ra.w;
    int medium = __float_as_int(ab.w);
    bool lastDelta = flags & kPathLastDelta;
    const V3 lastPosition = v3(st.last_pos[path]);
    const uint32_t depth = st.depth[path];
    const uint32_t pixel = st.pixel[path], sample = st.sample[path];
    Rng rng(st.rng[path]);
    const uint32_t tri = st.hit_tri[path];
    int err = 0;
    auto finish = [&](V3 radiance) { finishPath(P, O, st, path, radiance, E); freed = true; };

    if (CLASS == kShadeMiss || (CLASS == kShadeGeneric && tri == kNoTriangle)) {  // render.cpp:242-248
        if (medium >= 0) T = T * beerLambert(A, kInf);
        const float weight = lastDelta || !P.nee ? 1 : powerHeuristic(lastPdf, environmentPdf(S, ray.d));
        R = R + T * envRadiance(S, ray.d) * weight;
        finish(R);
        return;
    }
    // The traversal reported the triangle; t, u and v come from the same FP64 arithmetic.
    const cr_triangle& tr = S.tris[tri];
    const ExactSetup X = exact_setup(ray);
    double t = 0, w1 = 0, w2 = 0, det = 1;
    tri_exact(X, v3(tr.v[0].position), v3(tr.v[1].position), v3(tr.v[2].position), -static_cast<double>(kInf),
              static_cast<double>(kInf), t, w1, w2, det);
    const double hu = w1 / det, hv = w2 / det;
    if (medium >= 0) T = T * beerLambert(A, static_cast<float>(t));
    const Surface s = surfaceAt<LEAN>(S, ray.d, tri, hu, hv, err);
    if (s.frontFace || s.doubleSided) {
        const float weight = lastDelta || !P.nee ? 1 : powerHeuristic(lastPdf, trianglePdf(S, tri, lastPosition, s.position));
        R = R + T * s.emission * weight;
    }
    if (static_cast<int>(depth) == P.bounces) {
        if (err) { raise(E, P, pixel, sample, err); }
        finish(R);
        return;
    }
    const V3 wo = -ray.d;
    bool pending = false;
    TRay sh;
    V3 contrib;
    // Guided renders: at a rough, opaque surface (no delta or transmission lobe) the direction
    // is drawn from the network's mixture with probability a and from the BSDF otherwise
    // (one-sample MIS); both MIS weights of trace() then use the combined density.
    Mixture mix;
    bool guided = false;
    float a = 0;
    if constexpr (GUIDED) {
        guided = s.transmission <= 0 && s.roughness > 1e-3f;
        if (guided) {
            guideDecode(st.guide.mixture + static_cast<uint64_t>(path) * kGuideOut, mix);
            a = st.guide.guideProbability;
        }
    }
    if (CLASS == kShadeNeeNull && P.nee) {
        skipLight(S, rng, P.env_alias != 0);  // zero BSDF: the sample cannot contribute
    } else if (P.nee) {  // render.cpp:262-299
        const LightSample light = sampleLight<LEAN>(S, s.position, rng, P.env_alias, err);
        const bool enclosedInfinite = medium >= 0 && s.thickness <= 0 && !isfin(light.distance);
        if (!enclosedInfinite && light.pdf > 0 && maxComponent(light.radiance) > 0) {
            const BsdfEval bsdf = CLASS == kShadeConductor ? evaluateConductor(s, wo, light.direction)
                                                           : evaluateBsdf(s, wo, light.direction);
            if (maxComponent(bsdf.value) > 0) {
                bool ok = true;
                if (precise) { sh.o = s.position; sh.d = light.direction; sh.tmin = 0; sh.tmax = kInf; sh.olow = s.positionLow; }
                else ok = offsetRay(s.position, s.geometricNormal, light.direction, kInf, sh, err);
                if (ok && isfin(light.distance)) {
                    V3 end = light.target;
                    if (lengthSquared(light.targetNormal) > 0) {
                        TRay moved;
                        ok = offsetRay(end, light.targetNormal, -light.direction, kInf, moved, err);
                        end = moved.o;
                    }
                    const V3 delta = end - sh.o;
                    sh.tmax = length(delta) * (1 - 2e-6f);
                    sh.d = normalize(delta);
                }
                if (ok) {
                    float dirPdf = bsdf.pdf;
                    if constexpr (GUIDED) {
                        if (guided) dirPdf = a * mixturePdf(mix, light.direction) + (1 - a) * bsdf.pdf;
                    }
                    const float weight = light.delta ? 1 : powerHeuristic(light.pdf, dirPdf);
                    V3 shadowAbsorption = A;
                    bool shadowInMedium = medium >= 0;
                    if (s.thickness > 0 && dot(wo, s.geometricNormal) * dot(light.direction, s.geometricNormal) < 0) {
                        shadowInMedium = s.frontFace;
                        shadowAbsorption = s.frontFace ? absorptionCoefficient(s.attenuationColor, s.attenuationDistance) : V3{};
                    }
                    const V3 transmittance = shadowInMedium ? beerLambert(shadowAbsorption, light.distance) : V3{1};
                    contrib = T * bsdf.value * light.radiance * transmittance *
                              (fabsf(dot(s.normal, light.direction)) * weight / light.pdf);
                    pending = true;
                }
            }
        }
    }
    if (err) {  // an exception inside trace(): the sample fails
        raise(E, P, pixel, sample, err);
        finish(V3{});
        return;
    }
    const uint32_t ignore = precise ? tri : kNoTriangle;
    auto queueShadow = [&](bool dead) {
        st.sh_o[path] = f4(sh.o, sh.tmin);
        st.sh_d[path] = f4(sh.d, sh.tmax);
        st.sh_lo[path] = f4(sh.olow, __uint_as_float(ignore));
        st.sh_c[path] = f4(contrib, 0);
        shadow = true;
        if (dead) {
            st.rad[path] = f4(R, lastPdf);
            st.flags[path] = flags | kPathDead | kPathShadow;
        }
    };
    BsdfSample smp;
    if constexpr (GUIDED) {
        if (guided) {
            smp = emptySample();
            V3 fcos{};
            float bsdfPdf = 0;
            if (rng.uniform() < a) {
                const V3 w = sampleMixture(mix, rng);
                const BsdfEval e = evaluateBsdf(s, wo, w);
                if (e.pdf > 0 && maxComponent(e.value) > 0) {
                    smp.direction = w;
                    fcos = e.value * fabsf(dot(s.normal, w));
                    bsdfPdf = e.pdf;
                }
            } else {
                const BsdfSample b = sampleBsdf(s, wo, rng);
                if (b.ok() && !b.delta) {
                    smp.direction = b.direction;
                    fcos = b.weight * b.pdf;
                    bsdfPdf = b.pdf;
                }
            }
            if (bsdfPdf > 0) {
                const float pdf = a * mixturePdf(mix, smp.direction) + (1 - a) * bsdfPdf;
                smp.pdf = pdf;
                smp.weight = fcos * (1 / pdf);
            }
        } else {
            smp = sampleBsdf(s, wo, rng);
        }
    } else if constexpr (CLASS == kShadeConductor) {
        smp = sampleConductor(s, wo, rng);  // render.cpp:302-303
    } else if constexpr (CLASS == kShadeNeeNull) {
        smp = sampleSmooth(s, wo, rng);  // render.cpp:302-303 (the BSDF's delta branches)
    } else {
        smp = sampleBsdf(s, wo, rng);  // render.cpp:302-303
    }
    if (!smp.ok()) {
        if (pending) queueShadow(true); else finish(R);
        return;
    }
    T = T * smp.weight;
    if (!finite3(T)) {
        raise(E, P, pixel, sample, kErrNonFiniteThroughput);
        finish(V3{});
        return;
    }
    int boundary = 0;
    if (smp.transmitted && s.thickness > 0) {  // render.cpp:306-329
        if (s.frontFace) {
            if (medium >= 0) boundary = kErrNestedVolume;
            else { medium = static_cast<int>(s.material); A = absorptionCoefficient(s.attenuationColor, s.attenuationDistance); }
        } else {
            if (medium < 0) boundary = kErrExitWithoutEntry;
            else { medium = -1; A = V3{}; }
        }
        if (!boundary) etaScale *= smp.eta * smp.eta;
    }
    if (boundary) {
        if (!precise) {  // render.cpp:404-411: replay the same sample from split origins
            atomicAdd(retries, 1ull);
            initPath(S, P, st, path, pixel, sample, true, E);
            cont = true;
            return;
        }
        raise(E, P, pixel, sample, boundary);
        if (E.detail && boundary == kErrExitWithoutEntry) {
            E.detail->depth = static_cast<int32_t>(depth);
            E.detail->triangle = tri;
            E.detail->material = s.material;
            E.detail->t = t;
            E.detail->point[0] = s.position.x; E.detail->point[1] = s.position.y; E.detail->point[2] = s.position.z;
            E.detail->origin[0] = ray.o.x; E.detail->origin[1] = ray.o.y; E.detail->origin[2] = ray.o.z;
            E.detail->direction[0] = ray.d.x; E.detail->direction[1] = ray.d.y; E.detail->direction[2] = ray.d.z;
        }
        finish(V3{});
        return;
    }
    lastPdf = smp.pdf;
    lastDelta = smp.delta;
    TRay next;
    if (precise) { next.o = s.position; next.d = smp.direction; next.tmin = 0; next.tmax = kInf; next.olow = s.positionLow; }
    else if (!offsetRay(s.position, s.geometricNormal, smp.direction, kInf, next, err)) {
        raise(E, P, pixel, sample, err);
        finish(V3{});
        return;
    }
    if (P.rr && depth >= 3) {  // render.cpp:337-343
        const float survive = sclamp(maxComponent(T) * etaScale, 0.05f, 0.95f);
        if (rng.uniform() >= survive) {
            if (pending) queueShadow(true); else finish(R);
            return;
        }
        T = T * (1 / survive);
    }
    // continue
    st.ray_o[path] = f4(next.o, next.tmin);
    st.ray_d[path] = f4(next.d, next.tmax);
    if (precise) st.ray_lo[path] = f4(next.olow, 0);
    st.thr[path] = f4(T, etaScale);
    st.rad[path] = f4(R, lastPdf);
    st.last_pos[path] = f4(s.position, 0);
    st.absorb[path] = f4(A, __int_as_float(medium));
    flags = (flags & kPathPrecise) | (lastDelta ? kPathLastDelta : 0u);
    st.flags[path] = flags;
    st.rng[path] = rng.state;
    st.prev_tri[path] = ignore;
    st.depth[path] = depth + 1;
    if (pending) queueShadow(false);
    if constexpr (GUIDED) {  // remember the vertex: its incident light becomes a training sample
        if (guided && st.guide.record) {
            const uint32_t n = st.guide.count[path];
            if (n < kGuideRecords) {
                GuideRecord& r = guideRecords(st.guide, path)[n];
                const float4 ng = S.tri_ng[tri];
                r.feat[0] = (s.position.x - st.guide.lo[0]) * st.guide.inv[0];
                r.feat[1] = (s.position.y - st.guide.lo[1]) * st.guide.inv[1];
                r.feat[2] = (s.position.z - st.guide.lo[2]) * st.guide.inv[2];
                r.feat[3] = wo.x; r.feat[4] = wo.y; r.feat[5] = wo.z;
                r.feat[6] = ng.x; r.feat[7] = ng.y; r.feat[8] = ng.z;
                r.dir[0] = smp.direction.x; r.dir[1] = smp.direction.y; r.dir[2] = smp.direction.z;
                r.pdf = smp.pdf;
                r.base[0] = R.x; r.base[1] = R.y; r.base[2] = R.z;
                r.thr[0] = T.x; r.thr[1] = T.y; r.thr[2] = T.z;
                r.neeOpen = pending ? 1u : 0u;
                st.guide.count[path] = n + 1;
            }
        }
    }
    cont = true;
}

// What follows a shadow ray's any-hit query: an unoccluded contribution c is added to the
// path's radiance (render.cpp:283-296). Returns true when the path had ended and its slot is
// now free.
CR_D bool shadowFinish(const RenderParams& P, const OutRef& O, const PathSoA& st, uint32_t path, const ErrSink& E,
                       bool blocked, int err, float4 c) {
    if (err) raise(E, P, st.pixel[path], st.sample[path], err);
    const float4 ra = st.rad[path];
    V3 R = v3(ra);
    if (!blocked) R = R + v3(c);
    if (st.guide.count) guideNeeResolved(st.guide, path, blocked ? V3{} : v3(c));
    const uint32_t flags = st.flags[path];
    if (flags & kPathDead) { finishPath(P, O, st, path, R, E); return true; }
    st.rad[path] = f4(R, ra.w);
    return false;
}

// What follows a path's closest-hit query: the hit is recorded and its shading class returned.
CR_D int closestFinish(const DevScene& S, const RenderParams& P, const PathSoA& st, uint32_t path, const ErrSink& E,
                       bool found, const HitRec& h, int err) {
    st.hit_tri[path] = found ? h.tri : kNoTriangle;
    if (st.guide.hitT) st.guide.hitT[path] = found ? static_cast<float>(h.t) : 0.0f;
    if (err) raise(E, P, st.pixel[path], st.sample[path], err);
    if (!found) return kShadeMiss;
    if (S.nee_skip && (h.flags & kTriNeeNull)) return kShadeNeeNull;
    return (S.conductor_class && (h.flags & kTriConductor)) ? kShadeConductor : kShadeGeneric;
}

// Records one traced ray and the traversal's answer (cr_gpu_render_trace_dump).
CR_D void dumpRay(const TraceDump& D, const TRay& r, uint32_t ignore, uint32_t kind, uint32_t depth, bool found,
                  const HitRec& h, uint32_t launch) {
    const unsigned long long i = atomicAdd(D.count, 1ull);
    if (i >= D.capacity) return;
    cr_traced_ray& o = D.rays[i];
    o.ray.origin[0] = r.o.x; o.ray.origin[1] = r.o.y; o.ray.origin[2] = r.o.z;
    o.ray.direction[0] = r.d.x; o.ray.direction[1] = r.d.y; o.ray.direction[2] = r.d.z;
    o.ray.tmin = r.tmin; o.ray.tmax = r.tmax;
    o.ray.origin_low[0] = r.olow.x; o.ray.origin_low[1] = r.olow.y; o.ray.origin_low[2] = r.olow.z;
    o.ignore = ignore; o.kind = kind; o.depth = depth; o.found = found ? 1u : 0u; o.launch = launch;
    o.hit.t = found ? h.t : static_cast<double>(kInf);
    o.hit.u = found ? h.u : 0.0;
    o.hit.v = found ? h.v : 0.0;
    o.hit.triangle = found ? h.tri : kNoTriangle;
    o.hit.reserved_ = 0;
}

// Any hit for one queued shadow ray; an unoccluded contribution is added (render.cpp:283-296).
// Returns true when the path had ended and its slot is now free.
template <bool COUNT = false, bool NOALPHA = false>
CR_D bool shadowOne(const DevScene& S, const RenderParams& P, const OutRef& O, const PathSoA& st, uint32_t path,
                    const ErrSink& E, unsigned long long* stats = nullptr) {
    const float4 o = st.sh_o[path], d = st.sh_d[path], lo = st.sh_lo[path], c = st.sh_c[path];
    TRay r;
    r.o = v3(o); r.tmin = o.w; r.d = v3(d); r.tmax = d.w; r.olow = v3(lo);
    HitRec h;
    h.t = kInf; h.u = 0; h.v = 0; h.tri = 0;
    int err = 0;
    VisitCount vc;
    const bool blocked = intersect<true, COUNT, NOALPHA>(S, r, static_cast<double>(kInf), __float_as_uint(lo.w), P.exact_traversal != 0,
                                                h, err, &vc);
    if (COUNT) {
        atomicAdd(&stats[kStatShadowPairs], static_cast<unsigned long long>(vc.pairs));
        atomicAdd(&stats[kStatShadowTris], static_cast<unsigned long long>(vc.tris));
        if (st.dump.rays) dumpRay(st.dump, r, __float_as_uint(lo.w), 1, st.depth[path], blocked, h,
                                  static_cast<uint32_t>(stats[kStatIterations]) - 1);
    }
    return shadowFinish(P, O, st, path, E, blocked, err, c);
}

template <bool COUNT, bool NOALPHA = false>
CR_D int closestOne(const DevScene& S, const RenderParams& P, const PathSoA& st, uint32_t path, const ErrSink& E,
                    unsigned long long* stats) {
    const uint32_t flags = st.flags[path];
    const TRay r = loadRay(st, path, flags);
    HitRec h;
    h.t = kInf; h.u = 0; h.v = 0; h.tri = 0;
    int err = 0;
    VisitCount vc;
    const bool found = intersect<false, COUNT, NOALPHA>(S, r, static_cast<double>(kInf), st.prev_tri[path],
                                               P.exact_traversal != 0, h, err, &vc);
    if (COUNT) {
        atomicAdd(&stats[kStatPairs], static_cast<unsigned long long>(vc.pairs));
        atomicAdd(&stats[kStatTris], static_cast<unsigned long long>(vc.tris));
        if (st.dump.rays) dumpRay(st.dump, r, st.prev_tri[path], 0, st.depth[path], found, h,
                                  static_cast<uint32_t>(stats[kStatIterations]) - 1);
    }
    return closestFinish(S, P, st, path, E, found, h, err);
}

// The job of a path in the multi-job pool.
struct PathJob {
    const DevScene* S;
    const RenderParams* P;
    OutRef O;
    ErrSink E;
    unsigned long long* retries;
    uint32_t r;
};
CR_D PathJob pathJob(const JobTable& J, uint2 sj) {
    const uint32_t r = sj.x, job = sj.y;
    const IssueRange& R = J.ranges[r];
    PathJob pj;
    pj.S = J.scenes + job;
    pj.P = J.params + job;
    pj.O = R.spp ? OutRef{R.outBase - R.s0 - static_cast<uint64_t>(R.p0) * R.spp, 1, R.spp}
                 : OutRef{R.outBase - R.c0, R.pixels, 1};
    pj.E = ErrSink{J.errKeys + job, nullptr};
    pj.retries = J.retries + job;
    pj.r = r;
    return pj;
}
CR_D PathJob pathJob(const JobTable& J, uint32_t path) { return pathJob(J, J.slot[path]); }
// The range holding issue position pos (the last range starting at or before it).
CR_D uint32_t findRange(const JobTable& J, uint32_t count, uint64_t pos) {
    uint32_t lo = 0, hi = count;  // ranges[lo].start <= pos < ranges[hi].start
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (J.ranges[mid].start <= pos) lo = mid; else hi = mid;
    }
    return lo;
}
// All 32 lanes call this together: lanes whose sample finished count it in its range, one
// atomic per distinct range among them.
CR_D void countDone(const JobTable& J, bool finished, uint32_t r) {
    const unsigned active = __ballot_sync(0xffffffffu, finished);
    if (!finished) return;
    const unsigned peers = __match_any_sync(active, r);
    if (static_cast<int>(threadIdx.x & 31) == __ffs(peers) - 1)
        atomicAdd(&J.done[r], static_cast<unsigned long long>(__popc(peers)));
}

// ---- kernels -----------------------------------------------------------------------------------
// Every pool slot starts free (in free[1], which the first k_regen reads).
static __global__ void k_pool_init(Queues q, uint32_t pool) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pool; i += gridDim.x * blockDim.x) q.free[1][i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) q.counts[kCountFree1] = pool;
}

// Free slots take the next sample ids of the chunk, in order (single render), or the next
// positions of the issue list (MULTI: only when `refill`, and only up to the host's issue end;
// slots left without work stay in the free ring, untouched).
template <bool MULTI>
__global__ void __launch_bounds__(128) k_regen(DevScene S, RenderParams P, PathSoA st, Queues q, int cur, Chunk C, ErrSink E,
                                               unsigned long long* stats, JobTable J, int refill) {
    const uint32_t n = MULTI ? 0u : q.counts[kCountFree0 + (cur ^ 1)];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // nothing appends to free[cur] in this launch (the single render's k_regen never
        // appends, the pool's free slots are in the ring)
        if (!MULTI) q.counts[kCountFree0 + cur] = 0;
        for (int c = 0; c < kShadeClasses; ++c) q.counts[kCountShade0 + c] = 0;
        if (stats) stats[kStatIterations] += 1;
    }
    const uint32_t* freeQ = q.free[cur ^ 1];
    if constexpr (!MULTI) {
        for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
            const uint32_t idx = base + threadIdx.x;
            const bool have = idx < n;
            const uint32_t slot = have ? freeQ[idx] : 0;
            const unsigned mask = __ballot_sync(0xffffffffu, have);
            const int lane = threadIdx.x & 31;
            unsigned long long first = 0;
            if (mask) {
                const int leader = __ffs(mask) - 1;
                if (lane == leader) first = atomicAdd(&stats[kStatIssued], static_cast<unsigned long long>(__popc(mask)));
                first = __shfl_sync(0xffffffffu, first, leader);
            }
            const uint64_t id = first + __popc(mask & ((1u << lane) - 1u));
            bool live = false;
            if (have && id < C.c1) {
                uint32_t pixel, sample;
                chunkSample(C, id - C.c0, pixel, sample);
                live = initPath(S, P, st, slot, pixel, sample, false, E);
                if (!live) st.out[id - C.c0] = make_float4(0, 0, 0, 0);
            }
            warpPush(q.extend[cur], &q.counts[kCountExtend0 + cur], live, slot);
        }
    } else {
        const unsigned long long first = J.issued[cur ^ 1];
        const unsigned long long end = J.ctl[0];
        const uint32_t rangeCount = static_cast<uint32_t>(J.ctl[1]);
        const uint64_t avail = end > first ? end - first : 0;
        const unsigned long long head = J.head[cur ^ 1];
        const uint64_t nFree = *J.tail - head;
        const uint32_t claimed = refill && nFree >= J.refillMin ? static_cast<uint32_t>(avail < nFree ? avail : nFree) : 0u;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            J.issued[cur] = first + claimed;
            J.head[cur] = head + claimed;
        }
        for (uint32_t base = blockIdx.x * blockDim.x; base < claimed; base += gridDim.x * blockDim.x) {
            const uint32_t idx = base + threadIdx.x;
            const bool have = idx < claimed;
            const uint32_t slot = have ? J.ring[(head + idx) % J.poolSize] : 0;
            bool live = false, failed = false;
            uint32_t r = 0;
            if (have) {
                const uint64_t pos = first + idx;
                r = findRange(J, rangeCount, pos);
                const IssueRange& R = J.ranges[r];
                const uint64_t j = pos - R.start;
                uint32_t pixel, sample;
                chunkSample(rangeChunk(R), j, pixel, sample);
                J.slot[slot] = make_uint2(r, R.job);
                const ErrSink Ej{J.errKeys + R.job, nullptr};
                live = initPath(J.scenes[R.job], J.params[R.job], st, slot, pixel, sample, false, Ej);
                if (!live) {  // the sample is done (radiance 0); k_trace returns the slot to the ring
                    st.out[R.outBase + j] = make_float4(0, 0, 0, 0);
                    st.flags[slot] = kPathNull;
                    failed = true;
                }
            }
            warpPush(q.extend[cur], &q.counts[kCountExtend0 + cur], have, slot);
            countDone(J, failed, r);
        }
    }
}

// Closest hit for the live queue and any hit for last iteration's shadow rays, one launch.
// NOALPHA: no scene whose paths the launch traces has alpha-masked triangles, see accepts<NOALPHA>.
// BLOCK: threads per block (the multi-job engine tunes it; the register budget per SM, set by the
// minimum resident blocks, stays that of 128-thread blocks).
template <bool COUNT, bool MULTI = false, bool NOALPHA = false, int BLOCK = 128>
__global__ void __launch_bounds__(BLOCK, CR_TRACE_MIN_BLOCKS * 128 / BLOCK) k_trace(DevScene S, RenderParams P, PathSoA st, Queues q, int cur, Chunk C, ErrSink E,
                                               unsigned long long* stats, JobTable J) {
    const uint32_t nE = q.counts[kCountExtend0 + cur];
    const uint32_t nS = q.counts[kCountShadow0 + (cur ^ 1)];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        q.counts[kCountExtend0 + (cur ^ 1)] = 0;
        q.counts[kCountShadow0 + cur] = 0;
        // the next iteration's counters (this iteration's shading launches follow this one)
        q.counts[kCountTraceWork0 + (cur ^ 1)] = 0;
        for (int c = 0; c < kShadeClasses; ++c) q.counts[kCountShadeWork0 + c] = 0;
        stats[kStatExtendRays] += nE;
        stats[kStatShadowRays] += nS;
    }
    const uint32_t total = nE + nS;
    for (uint32_t base = warpTake(&q.counts[kCountTraceWork0 + cur]); base < total;
         base = warpTake(&q.counts[kCountTraceWork0 + cur])) {
        const uint32_t idx = base + (threadIdx.x & 31);
        bool freed = false;
        int cls = -1;
        uint32_t path = 0, r = 0;
        if (idx < nE) {
            path = q.extend[cur][idx];
            if constexpr (MULTI) {
                const uint2 sj = J.slot[path];  // loaded beside the flags, not after them
                if (st.flags[path] == kPathNull) {
                    freed = true;  // a sample whose camera ray failed: only its slot comes back
                } else {
                    const PathJob pj = pathJob(J, sj);
                    cls = closestOne<COUNT, NOALPHA>(*pj.S, *pj.P, st, path, pj.E, stats);
                }
            } else {
                cls = closestOne<COUNT, NOALPHA>(S, P, st, path, E, stats);
            }
        } else if (idx < total) {
            path = q.shadow[cur ^ 1][idx - nE];
            if constexpr (MULTI) {
                const PathJob pj = pathJob(J, path);
                freed = shadowOne<COUNT, NOALPHA>(*pj.S, *pj.P, pj.O, st, path, pj.E, stats);
                r = pj.r;
            } else {
                freed = shadowOne<COUNT, NOALPHA>(S, P, outOf(C), st, path, E, stats);
            }
        }
        if constexpr (MULTI) {
            ringPush(J, freed, path);
            countDone(J, freed && idx >= nE, r);  // a null path's sample was counted by k_regen
        } else {
            warpPush(q.free[cur], &q.counts[kCountFree0 + cur], freed, path);
        }
#pragma unroll
        for (int c = 0; c < kShadeClasses; ++c) warpPush(q.shade[c], &q.counts[kCountShade0 + c], cls == c, path);
    }
}

// LEAN (every scene whose paths the launch shades has no textures, punctual lights or alpha
// masks): the shading code without those features, a smaller kernel with the same arithmetic.
template <int CLASS, bool MULTI = false, bool GUIDED = false, bool LEAN = false, int BLOCK = 128>
__global__ void __launch_bounds__(BLOCK, CR_SHADE_MIN_BLOCKS * 128 / BLOCK) k_shade(DevScene S, RenderParams P, PathSoA st, Queues q, int cur, Chunk C, ErrSink E,
                                               unsigned long long* stats, JobTable J) {
    const uint32_t n = q.counts[kCountShade0 + CLASS];
    const uint32_t* in = q.shade[CLASS];
    for (uint32_t base = warpTake(&q.counts[kCountShadeWork0 + CLASS]); base < n;
         base = warpTake(&q.counts[kCountShadeWork0 + CLASS])) {
        const uint32_t idx = base + (threadIdx.x & 31);
        bool cont = false, shadow = false, freed = false;
        uint32_t path = 0, r = 0;
        if (idx < n) {
            path = in[idx];
            if constexpr (MULTI) {
                const PathJob pj = pathJob(J, path);
                shadeOne<CLASS, false, LEAN>(*pj.S, *pj.P, pj.O, st, path, pj.E, pj.retries, cont, shadow, freed);
                r = pj.r;
            } else {
                shadeOne<CLASS, GUIDED, LEAN>(S, P, outOf(C), st, path, E, &stats[kStatRetries], cont, shadow, freed);
            }
        }
        warpPush(q.extend[cur ^ 1], &q.counts[kCountExtend0 + (cur ^ 1)], cont, path);
        warpPush(q.shadow[cur], &q.counts[kCountShadow0 + cur], shadow, path);
        if constexpr (MULTI) {
            ringPush(J, freed, path);
            countDone(J, freed, r);
        } else {
            warpPush(q.free[cur], &q.counts[kCountFree0 + cur], freed, path);
        }
    }
}

// render.cpp:390-413: each pixel adds the chunk's samples in index order.
static __global__ void k_accumulate(const float4* out, Chunk C, double* acc) {
    if (C.spp) {  // pixel-major chunk: a pixel's samples are consecutive
        const uint64_t count = (C.c1 - C.c0) / C.spp;  // pixels from p0 on
        for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < count;
             p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
            double* a = acc + 3 * (C.p0 + p);
            double r = a[0], g = a[1], b = a[2];
            const float4* o = out + p * C.spp;
            for (uint32_t k = 0; k < C.spp; ++k) {
                const float4 v = o[k];
                r += v.x; g += v.y; b += v.z;
            }
            a[0] = r; a[1] = g; a[2] = b;
        }
        return;
    }
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < C.pixels;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t sBegin = C.c0 > p ? (C.c0 - p + C.pixels - 1) / C.pixels : 0;
        const uint64_t sEnd = C.c1 > p ? (C.c1 - p + C.pixels - 1) / C.pixels : 0;
        double r = acc[3 * p], g = acc[3 * p + 1], b = acc[3 * p + 2];
        for (uint64_t s = sBegin; s < sEnd; ++s) {
            const float4 o = out[s * C.pixels + p - C.c0];
            r += o.x; g += o.y; b += o.z;
        }
        acc[3 * p] = r; acc[3 * p + 1] = g; acc[3 * p + 2] = b;
    }
}
// Copies the chunk's radiance as packed RGB (sample-major) for stream-level comparisons.
static __global__ void k_pack_samples(const float4* out, Chunk C, float* dst) {
    const uint64_t n = C.c1 - C.c0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float4 o = out[i];
        const uint64_t d = C.spp ? (i % C.spp) * C.pixels + i / C.spp : i;
        dst[3 * d] = o.x; dst[3 * d + 1] = o.y; dst[3 * d + 2] = o.z;
    }
}
// render.cpp:415
static __global__ void k_film(const double* acc, float* film, uint64_t pixels, int samples) {
    for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * pixels; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        film[i] = static_cast<float>(acc[i] / samples);
}

// Re-runs one failing sample on one thread with full error capture (same device functions).
static __global__ void k_trace_one(DevScene S, RenderParams P, PathSoA st, uint32_t pixel, uint32_t sample, DevError* detail,
                            unsigned long long* scratchKey, unsigned long long* scratchRetries) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const ErrSink E{scratchKey, detail};
    const uint32_t path = 0;
    const uint64_t pixels = static_cast<uint64_t>(P.width) * P.height;
    const uint64_t id = static_cast<uint64_t>(sample) * pixels + pixel;
    const OutRef O = outOf(Chunk{id, id + 1, pixels});
    if (!initPath(S, P, st, path, pixel, sample, false, E)) return;
    for (int iter = 0; iter < 4 * (P.bounces + 2); ++iter) {
        const uint32_t flags = st.flags[path];
        const TRay r = loadRay(st, path, flags);
        HitRec h;
        h.t = kInf; h.u = 0; h.v = 0; h.tri = 0;
        int err = 0;
        const bool found = intersect<false>(S, r, static_cast<double>(kInf), st.prev_tri[path], P.exact_traversal != 0, h, err);
        if (err) { raise(E, P, pixel, sample, err); return; }
        st.hit_tri[path] = found ? h.tri : kNoTriangle;
        bool cont = false, shadow = false, freed = false;
        shadeOne<kShadeGeneric>(S, P, O, st, path, E, scratchRetries, cont, shadow, freed);
        if (detail->code) return;
        if (shadow) shadowOne(S, P, O, st, path, E);
        if (detail->code || !cont) return;
    }
}

static __global__ void k_intersect_batch(DevScene S, const cr_ray* rays, cr_hit* hits, uint8_t* found, uint64_t n, int any,
                                  uint32_t ignore, int exact, unsigned long long* errIndex) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const cr_ray cr = rays[i];
        TRay r;
        r.o = v3(cr.origin); r.d = v3(cr.direction); r.tmin = cr.tmin; r.tmax = cr.tmax; r.olow = v3(cr.origin_low);
        const cr_hit in = hits[i];
        HitRec h{in.t, in.u, in.v, in.triangle};
        int err = 0;
        const bool f = any ? intersect<true>(S, r, in.t, ignore, exact != 0, h, err)
                           : intersect<false>(S, r, in.t, ignore, exact != 0, h, err);
        if (f) { cr_hit out = in; out.t = h.t; out.u = h.u; out.v = h.v; out.triangle = h.tri; hits[i] = out; }
        found[i] = f ? 1 : 0;
        if (err) atomicMin(errIndex, static_cast<unsigned long long>(i));
    }
}

// Environment samples for checks of the sampler: texel and density of sample i of the stream
// Rng(sampleSeed(seed, i, 0)). S.env_pdf holds the densities of the sampler in use.
static __global__ void k_env_samples(DevScene S, int alias, uint64_t seed, uint64_t first, uint64_t count,
                                     uint32_t* texels, float* densities) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        Rng rng(sampleSeed(seed, first + i, 0));
        const uint64_t index = envPickTexel(S, rng, alias != 0);
        texels[i] = static_cast<uint32_t>(index);
        densities[i] = __ldg(S.env_pdf + index);
    }
}

static __global__ void k_camera_rays(RenderParams P, uint32_t sample, cr_ray* out, unsigned long long* errKey) {
    const uint64_t pixels = static_cast<uint64_t>(P.width) * P.height;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < pixels; p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        Rng rng(sampleSeed(P.seed, p, sample));
        const uint32_t x = static_cast<uint32_t>(p % P.width), y = static_cast<uint32_t>(p / P.width);
        const float dx = rng.uniform(), dy = rng.uniform();
        TRay r;
        cr_ray o;
        if (!cameraRay(P.camera, P.width, P.height, static_cast<float>(x) + dx, static_cast<float>(y) + dy, r)) {
            atomicMin(errKey, static_cast<unsigned long long>(errorKey(P, static_cast<uint32_t>(p), sample)));
            memset(&o, 0, sizeof(o));
        } else {
            o.origin[0] = r.o.x; o.origin[1] = r.o.y; o.origin[2] = r.o.z;
            o.direction[0] = r.d.x; o.direction[1] = r.d.y; o.direction[2] = r.d.z;
            o.tmin = r.tmin; o.tmax = r.tmax;
            o.origin_low[0] = o.origin_low[1] = o.origin_low[2] = 0;
        }
        out[p] = o;
    }
}

}  // namespace crg
