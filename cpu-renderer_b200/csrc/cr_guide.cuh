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

namespace crg {

constexpr int kGuideIn = 64;       // encoded input width (33 features, zero padded)
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

// Inputs: the 9 features, then sin and cos of 2^k * pi * position for k = 0..3.
CR_HD void guideEncode(const float f[kGuideFeatures], float x[kGuideIn]) {
    for (int i = 0; i < kGuideIn; ++i) x[i] = 0.0f;
    for (int i = 0; i < kGuideFeatures; ++i) x[i] = f[i];
    int o = kGuideFeatures;
    for (int k = 0; k < 4; ++k) {
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
struct GuidePaths {
    const float* mixture;   // [path][kGuideOut] network outputs of the path's current vertex
    float* hitT;            // [path] closest-hit distance (float)
    GuideRecord* records;   // [path][kGuideRecords]
    uint32_t* count;        // [path] records in use
    GuideSample* samples;   // training samples collected
    unsigned long long* sampleCount;
    uint64_t sampleCapacity;
    V3 boundsLo, boundsInv; // position features = (p - lo) * inv
    float guideProbability; // one-sample MIS: the mixture's share of the directions
    int record;             // collect training samples
};

}  // namespace crg
