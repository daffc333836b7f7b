// Learned path guiding: the proposal network's layout, its input encoding and the mixture of
// von Mises-Fisher lobes it outputs (device side, shared by inference, training and shading).
//
// Network: 4 dense layers, 64 wide: x (64 encoded inputs) -> relu(W1 x + b1) -> relu(W2 . + b2)
// -> relu(W3 . + b3) -> W4 . + b4 (40 outputs = 8 lobes x [logit, log kappa, mean xyz]).
// Weights are kept as FP32 masters (Adam) and an FP16 copy (inference on the tensor cores).
// Every weight matrix is stored [out][in] (in contiguous).
//
// Mixture: q(w) = sum_j pi_j vMF(w | mu_j, kappa_j), pi = softmax(logits), mu_j = normalize(m_j),
// kappa_j = exp(clamp(log kappa, kLogKappaMin, kLogKappaMax)),
// vMF(w | mu, k) = k / (2 pi (1 - exp(-2k))) exp(k (mu . w - 1)).
#pragma once
#include <cuda_fp16.h>

#include "cr_dev_math.cuh"
#include "cr_internal.h"

namespace crg {

constexpr int kGuideIn = 64;       // encoded input width (57 encoded features, zero padded)
constexpr int kGuideWidth = 64;
constexpr int kGuideLobes = 8;
constexpr int kGuideOut = 40;      // 5 per lobe
constexpr int kGuideOutPad = 48;   // output rows padded to the tensor-core tile (n = 8)
constexpr int kGuideFeatures = 9;  // position in [0,1]^3, outgoing direction, normal
// parameter offsets (weights, then biases), in floats / halves
constexpr int kGW1 = 0, kGW2 = kGW1 + kGuideWidth * kGuideIn, kGW3 = kGW2 + kGuideWidth * kGuideWidth,
              kGW4 = kGW3 + kGuideWidth * kGuideWidth, kGWCount = kGW4 + kGuideOutPad * kGuideWidth;
constexpr int kGB1 = kGWCount, kGB2 = kGB1 + kGuideWidth, kGB3 = kGB2 + kGuideWidth, kGB4 = kGB3 + kGuideWidth,
              kGParams = kGB4 + kGuideOutPad;
constexpr float kLogKappaMin = -3.0f, kLogKappaMax = 9.0f;
constexpr int kGuideOctaves = 8;

// Inputs: the 9 features, then sin and cos of 2^k * pi * position for k = 0..kGuideOctaves-1
// (57 of the 64 inputs; 8 octaves resolve 1/256 of the scene's extent).
CR_HD void guideEncode(const float f[kGuideFeatures], float x[kGuideIn]) {
    for (int i = 0; i < kGuideIn; ++i) x[i] = 0.0f;
    for (int i = 0; i < kGuideFeatures; ++i) x[i] = f[i];
    int o = kGuideFeatures;
    for (int k = 0; k < kGuideOctaves; ++k) {
        const float s = static_cast<float>(1 << k) * kPi;
        for (int d = 0; d < 3; ++d) {
            float sn, cs;
#ifdef __CUDA_ARCH__
            sincosf(s * f[d], &sn, &cs);
#else
            sn = std::sin(s * f[d]);
            cs = std::cos(s * f[d]);
#endif
            x[o++] = sn;
            x[o++] = cs;
        }
    }
}

struct Mixture {
    float pi[kGuideLobes];
    V3 mu[kGuideLobes];
    float kappa[kGuideLobes];
};

CR_D void guideDecode(const float* out, Mixture& m) {
    float mx = -1e30f;
    for (int j = 0; j < kGuideLobes; ++j) mx = fmaxf(mx, out[5 * j]);
    float sum = 0;
    for (int j = 0; j < kGuideLobes; ++j) {
        m.pi[j] = expf(out[5 * j] - mx);
        sum += m.pi[j];
        m.kappa[j] = expf(fminf(fmaxf(out[5 * j + 1], kLogKappaMin), kLogKappaMax));
        const V3 raw{out[5 * j + 2], out[5 * j + 3], out[5 * j + 4]};
        const float l = sqrtf(dot(raw, raw));
        m.mu[j] = l > 1e-12f ? raw * (1.0f / l) : V3{0, 0, 1};
    }
    for (int j = 0; j < kGuideLobes; ++j) m.pi[j] /= sum;
}

// log vMF(w | mu, k) = log k - log 2pi - log(1 - e^-2k) + k (mu.w - 1); -expm1(-2k) keeps small
// kappa accurate, and the log form keeps sharp lobes from underflowing.
CR_D float vmfLogPdf(V3 mu, float kappa, V3 w) {
    return logf(kappa) - 1.8378770664093453f - logf(-expm1f(-2 * kappa)) + kappa * (dot(mu, w) - 1);
}

CR_D float mixturePdf(const Mixture& m, V3 w) {
    float lt[kGuideLobes], mx = -1e30f;
    for (int j = 0; j < kGuideLobes; ++j) {
        lt[j] = m.pi[j] > 0 ? logf(m.pi[j]) + vmfLogPdf(m.mu[j], m.kappa[j], w) : -1e30f;
        mx = fmaxf(mx, lt[j]);
    }
    float s = 0;
    for (int j = 0; j < kGuideLobes; ++j) s += expf(lt[j] - mx);
    return expf(mx) * s;
}

// Three draws: the lobe, then the vMF's cosine and azimuth (inverse CDF in the stable form
// w = 1 + log(u + (1 - u) e^-2k) / k).
CR_D V3 sampleMixture(const Mixture& m, Rng& rng) {
    const float pick = rng.uniform();
    int j = 0;
    float acc = m.pi[0];
    while (j + 1 < kGuideLobes && pick >= acc) acc += m.pi[++j];
    const float u = rng.uniform(), phi = 2 * kPi * rng.uniform();
    const float k = m.kappa[j];
    float w = 1 + log1pf(u * expm1f(-2 * k) ) / k;  // log(u e^-2k + 1 - u) = log1p(u (e^-2k - 1))
    w = fminf(1.0f, fmaxf(-1.0f, w));
    const float r = sqrtf(fmaxf(0.0f, 1 - w * w));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const Frame f(m.mu[j]);
    return f.world(V3{r * cp, r * sp, w});
}

// Per-path guiding state of a guided render (structure of arrays over path slots).
constexpr int kGuideRecords = 4;   // guided vertices remembered per path
struct GuideRecord {
    float feat[kGuideFeatures];
    float dir[3];
    float pdf;      // mixture density of dir
    float base[3];  // radiance the path had before light arriving along dir
    float thr[3];   // throughput after the vertex (weight of the light along dir)
    uint32_t neeOpen;  // this vertex's own light sample may still add to the radiance
};
struct GuideSample {  // one training sample
    float feat[kGuideFeatures];
    float dir[3];
    float weight;   // luminance of the incident radiance along dir / its sampling density
};
CR_D GuideRecord* guideRecords(const GuidePathRefs& G, uint32_t path) {
    return static_cast<GuideRecord*>(G.records) + static_cast<uint64_t>(path) * kGuideRecords;
}

// Light arriving at a recorded vertex from its own light sample is not light along the
// recorded direction: it moves the record's base along with the path's radiance.
CR_D void guideNeeResolved(const GuidePathRefs& G, uint32_t path, V3 added) {
    const uint32_t n = G.count[path];
    if (!n) return;
    GuideRecord& r = guideRecords(G, path)[n - 1];
    if (!r.neeOpen) return;
    r.base[0] += added.x; r.base[1] += added.y; r.base[2] += added.z;
    r.neeOpen = 0;
}

// A finished path turns its records into training samples: the light that arrived along each
// recorded direction is (final radiance - base) / throughput after the vertex, and the sample
// weight is its luminance over the direction's sampling density.
CR_D void guideFinish(const GuidePathRefs& G, uint32_t path, V3 R) {
    const uint32_t n = G.count[path];
    const GuideRecord* rec = guideRecords(G, path);
    for (uint32_t i = 0; i < n; ++i) {
        const GuideRecord& r = rec[i];
        const float lx = r.thr[0] > 0 ? (R.x - r.base[0]) / r.thr[0] : 0.0f;
        const float ly = r.thr[1] > 0 ? (R.y - r.base[1]) / r.thr[1] : 0.0f;
        const float lz = r.thr[2] > 0 ? (R.z - r.base[2]) / r.thr[2] : 0.0f;
        const float w = luminance(V3{fmaxf(lx, 0.0f), fmaxf(ly, 0.0f), fmaxf(lz, 0.0f)}) / r.pdf;
        if (!(w > 0) || !isfinite(w)) continue;
        const unsigned long long at = atomicAdd(G.sampleCount, 1ull);
        if (at >= G.sampleCapacity) continue;
        GuideSample& out = static_cast<GuideSample*>(G.samples)[at];
        for (int k = 0; k < kGuideFeatures; ++k) out.feat[k] = r.feat[k];
        out.dir[0] = r.dir[0]; out.dir[1] = r.dir[1]; out.dir[2] = r.dir[2];
        out.weight = w;
    }
    G.count[path] = 0;
}

}  // namespace crg

struct cr_guide;
namespace crg {
// Host side (cr_guide.cu). Inference for the paths of a shading queue (device count), outputs
// at out[path * kGuideOut]; Adam steps over device-resident samples (weightMean <= 0: the
// samples' mean weight, computed on the device). Both run on stream s.
void guideInferPaths(cr_guide* gd, cudaStream_t s, const uint32_t* queue, const uint32_t* queueCount, uint32_t maxRows,
                     const PathSoA& st, const float* hitT, const DevScene& S, V3 lo, V3 inv, float* out);
float guideTrain(cr_guide* gd, cudaStream_t s, const GuideSample* samples, uint64_t n, uint32_t steps, uint32_t batch,
                 float lr, double weightMean);
}  // namespace crg
