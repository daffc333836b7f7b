// The reference's phase benchmark (tests/benchmark.cpp:18-62) on the device: the same seven
// phases, each one kernel over all its calls, timed with CUDA events on the scene's stream.
//
//   camera          Camera::generate at raster positions drawn from Rng(seed): ray i takes
//                   draws 2i and 2i+1. The reference writes generate(rng.uniform()*W,
//                   rng.uniform()*H, W, H); its build compiler (g++) evaluates the arguments
//                   right to left, so y takes draw 2i and x draw 2i+1 — the same rays.
//   closest hit     Bvh::intersect per ray; the checksum adds t of every hit
//   occlusion       Bvh::intersect(any) per ray; the checksum adds 1 per blocked ray
//   surface         surfaceAt for every hit
//   BSDF sampling   sampleBsdf(surface, -direction) per hit; the checksum adds the pdf
//   BSDF evaluation evaluateBsdf(surface, -direction, surface.normal); the checksum adds the pdf
//   environment     Environment::sample + radiance + pdf; the checksum adds luminance + pdf
//
// The reference draws the BSDF and environment phases from the same sequential generator,
// whose position after each sampleBsdf depends on the lobe it took; here call i of those two
// phases takes its own stream Rng(sampleSeed(seed, i, phase)) instead. Every phase is run
// once untimed, then timed.
#include "cr_kernels.cuh"
#include "cr_driver.h"

#include <cstring>
#include <string>

using namespace crg;
using namespace crd;

namespace {

enum { kPhCamera, kPhClosest, kPhOcclusion, kPhSurface, kPhBsdfSample, kPhBsdfEval, kPhEnv, kPhases };

struct PhaseBuffers {
    float4* rayO;        // origin, tmin
    float4* rayD;        // direction, tmax
    HitRec* hits;
    uint8_t* found;
    Surface* surfaces;
    double* sums;        // [kPhases]
    unsigned long long* counts;  // [0] hits
};

__device__ __forceinline__ uint64_t gridIndex() { return blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ uint64_t gridStride() { return static_cast<uint64_t>(gridDim.x) * blockDim.x; }

__global__ void k_ph_camera(RenderParams P, uint64_t n, uint64_t seed, PhaseBuffers B) {
    for (uint64_t i = gridIndex(); i < n; i += gridStride()) {
        Rng rng(seed + 2 * i * kGolden);  // the generator after 2i draws
        const float y = rng.uniform() * static_cast<float>(P.height);
        const float x = rng.uniform() * static_cast<float>(P.width);
        TRay r;
        if (!cameraRay(P.camera, P.width, P.height, x, y, r)) { r.o = V3{}; r.d = V3{}; r.tmin = 1; r.tmax = 0; }
        B.rayO[i] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
        B.rayD[i] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
    }
}

__device__ __forceinline__ TRay rayAt(const PhaseBuffers& B, uint64_t i) {
    const float4 o = B.rayO[i], d = B.rayD[i];
    TRay r;
    r.o = V3{o.x, o.y, o.z}; r.tmin = o.w;
    r.d = V3{d.x, d.y, d.z}; r.tmax = d.w;
    r.olow = V3{};
    return r;
}

template <bool ANY>
__global__ void k_ph_trace(DevScene S, uint64_t n, PhaseBuffers B) {
    double sum = 0;
    unsigned long long hits = 0;
    for (uint64_t i = gridIndex(); i < n; i += gridStride()) {
        HitRec h;
        h.t = kInf; h.u = 0; h.v = 0; h.tri = 0; h.flags = 0;
        int err = 0;
        const bool f = intersect<ANY>(S, rayAt(B, i), static_cast<double>(kInf), kNoTriangle, false, h, err);
        if (ANY) {
            sum += f ? 1.0 : 0.0;
        } else {
            B.found[i] = f ? 1 : 0;
            B.hits[i] = h;
            if (f) { sum += h.t; ++hits; }
        }
    }
    atomicAdd(&B.sums[ANY ? kPhOcclusion : kPhClosest], sum);
    if (!ANY) atomicAdd(&B.counts[0], hits);
}

__global__ void k_ph_surface(DevScene S, uint64_t n, PhaseBuffers B) {
    for (uint64_t i = gridIndex(); i < n; i += gridStride()) {
        if (!B.found[i]) continue;
        const HitRec h = B.hits[i];
        int err = 0;
        B.surfaces[i] = surfaceAt(S, rayAt(B, i).d, h.tri, h.u, h.v, err);
    }
}

__global__ void k_ph_bsdf(uint64_t n, uint64_t seed, int evaluate, PhaseBuffers B) {
    double sum = 0;
    for (uint64_t i = gridIndex(); i < n; i += gridStride()) {
        if (!B.found[i]) continue;
        const Surface s = B.surfaces[i];
        const V3 wo = -rayAt(B, i).d;
        if (evaluate) {
            sum += evaluateBsdf(s, wo, s.normal).pdf;
        } else {
            Rng rng(sampleSeed(seed, i, kPhBsdfSample));
            sum += sampleBsdf(s, wo, rng).pdf;
        }
    }
    atomicAdd(&B.sums[evaluate ? kPhBsdfEval : kPhBsdfSample], sum);
}

__global__ void k_ph_env(DevScene S, uint64_t n, uint64_t seed, PhaseBuffers B) {
    double sum = 0;
    for (uint64_t i = gridIndex(); i < n; i += gridStride()) {
        Rng rng(sampleSeed(seed, i, kPhEnv));
        float density = 0;
        const V3 d = envSample(S, rng, density, false);
        sum += static_cast<double>(luminance(envRadiance(S, d)) + envPdf(S, d));
    }
    atomicAdd(&B.sums[kPhEnv], sum);
}

}  // namespace

extern "C" cr_status cr_gpu_phase_benchmark(cr_gpu_scene* g, const cr_camera* camera, int32_t width, int32_t height,
                                            uint32_t count, uint64_t seed, cr_phase_timing* out) {
    try {
        if (!g || !camera || !out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        if (count == 0) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "count must be positive");
        std::lock_guard<std::mutex> lock(g->mutex);
        CR_CUDA(cudaSetDevice(g->device));
        cr_render_options o{width, height, 1, 1, 0, seed, 1, 1};
        crh::validate_options(o);
        const RenderParams P = makeParams(*camera, o, cr_gpu_tuning{});
        const uint64_t n = count;
        DevAlloc mem;
        PhaseBuffers B{};
        B.rayO = mem.alloc<float4>(n);
        B.rayD = mem.alloc<float4>(n);
        B.hits = mem.alloc<HitRec>(n);
        B.found = mem.alloc<uint8_t>(n);
        B.surfaces = mem.alloc<Surface>(n);
        B.sums = mem.alloc<double>(kPhases);
        B.counts = mem.alloc<unsigned long long>(1);
        cudaStream_t s = g->stream;
        cudaEvent_t ev[2];
        CR_CUDA(cudaEventCreate(&ev[0]));
        CR_CUDA(cudaEventCreate(&ev[1]));
        const int grid = occupancyGrid(reinterpret_cast<const void*>(k_ph_trace<false>), 128, g->device);
        double seconds[kPhases] = {};
        auto phase = [&](int k, auto&& launch) {
            launch();  // untimed pass
            CR_CUDA(cudaMemsetAsync(B.sums + k, 0, sizeof(double), s));
            if (k == kPhClosest) CR_CUDA(cudaMemsetAsync(B.counts, 0, sizeof(unsigned long long), s));
            CR_CUDA(cudaEventRecord(ev[0], s));
            launch();
            CR_CUDA(cudaEventRecord(ev[1], s));
            CR_CUDA(cudaEventSynchronize(ev[1]));
            CR_CUDA(cudaGetLastError());
            float ms = 0;
            CR_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            seconds[k] = ms / 1e3;
        };
        phase(kPhCamera, [&] { k_ph_camera<<<grid, 128, 0, s>>>(P, n, seed, B); });
        phase(kPhClosest, [&] { k_ph_trace<false><<<grid, 128, 0, s>>>(g->dev, n, B); });
        phase(kPhOcclusion, [&] { k_ph_trace<true><<<grid, 128, 0, s>>>(g->dev, n, B); });
        phase(kPhSurface, [&] { k_ph_surface<<<grid, 128, 0, s>>>(g->dev, n, B); });
        phase(kPhBsdfSample, [&] { k_ph_bsdf<<<grid, 128, 0, s>>>(n, seed, 0, B); });
        phase(kPhBsdfEval, [&] { k_ph_bsdf<<<grid, 128, 0, s>>>(n, seed, 1, B); });
        phase(kPhEnv, [&] { k_ph_env<<<grid, 128, 0, s>>>(g->dev, n, seed, B); });
        double sums[kPhases];
        unsigned long long hits = 0;
        CR_CUDA(cudaMemcpyAsync(sums, B.sums, sizeof(sums), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(&hits, B.counts, sizeof(hits), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        mem.release();
        const uint64_t calls[kPhases] = {n, n, n, hits, hits, hits, n};
        for (int k = 0; k < kPhases; ++k) {
            out[k].seconds = seconds[k];
            out[k].calls = calls[k];
            out[k].checksum = k == kPhCamera || k == kPhSurface ? 0.0 : sums[k];
        }
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}
