// The path-guiding network on the device: inference and training (forward and backward) on the
// tensor cores, Adam, and the cr_guide C ABI.
//
// Inference (k_guide_infer): one warp evaluates 32 rows. Activations live in shared memory as
// FP16 (row stride 72 halves), weights as FP16 [out][in] (same stride); every layer is
// mma.sync.m16n8k16 (FP16 x FP16 -> FP32) over 2 row tiles x (out / 8) column tiles x 4 k steps,
// then bias + ReLU in FP32 and the result rounded back to FP16 for the next layer. The last
// layer's 40 outputs are written as FP32.
//
// Training (k_guide_grad): a block's 128 samples go through the network as GEMMs on the tensor
// cores (TF32 in split precision, FP32 accumulation, with the FP16 weights inference uses); each lane computes the gradient of its sample's weighted negative log-likelihood
// -w log q(dir) with respect to the 40 outputs; deltas and weight gradients are GEMMs again,
// added to the global gradient once per block. k_guide_adam applies Adam (lr, beta1 0.9,
// beta2 0.999, eps 1e-8) to the FP32 masters and refreshes the FP16 copy.
#include "cr_guide.cuh"
#include "cr_driver.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

using namespace crg;
using namespace crd;

namespace crg {

constexpr int kActStride = 72;  // halves per shared-memory row (64 + 8 against bank conflicts)
constexpr int kInferWarps = 4;
constexpr int kWeightRows = 3 * kGuideWidth + kGuideOutPad;  // 240 rows of 64 inputs

struct GuideNetDev {
    const __half* w16;  // [kGParams] FP16 copy (weights then biases)
    const float* w32;   // [kGParams] FP16-rounded values as FP32 (training forward)
};

__device__ __forceinline__ uint32_t pack2(const __half* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One dense layer for the warp's 32 rows: act (32 x 64, FP16) times W^T (W: [N][64] FP16).
// N is 64 (hidden) or kGuideOutPad; outputs go back to act (FP16, after ReLU) or to out32.
template <int N, bool LAST>
__device__ void warpLayer(const __half* W, const float* bias, __half* act, float* out32) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    float acc[2][N / 8][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        const int k0 = kt * 16 + tig * 2;
        uint32_t a[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const __half* r0 = act + (mt * 16 + gid) * kActStride;
            const __half* r1 = r0 + 8 * kActStride;
            a[mt][0] = pack2(r0 + k0);
            a[mt][1] = pack2(r1 + k0);
            a[mt][2] = pack2(r0 + k0 + 8);
            a[mt][3] = pack2(r1 + k0 + 8);
        }
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            const __half* wr = W + (nt * 8 + gid) * kActStride;
            const uint32_t b0 = pack2(wr + k0), b1 = pack2(wr + k0 + 8);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma16816(acc[mt][nt], a[mt][0], a[mt][1], a[mt][2], a[mt][3], b0, b1);
        }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {  // h = 0: row gid, h = 1: row gid + 8
                const int row = mt * 16 + gid + 8 * h, col = nt * 8 + tig * 2;
                float v0 = acc[mt][nt][2 * h] + bias[col], v1 = acc[mt][nt][2 * h + 1] + bias[col + 1];
                if (LAST) {
                    if (col < kGuideOut) out32[row * kGuideOut + col] = v0;
                    if (col + 1 < kGuideOut) out32[row * kGuideOut + col + 1] = v1;
                } else {
                    v0 = fmaxf(v0, 0.0f);
                    v1 = fmaxf(v1, 0.0f);
                    act[row * kActStride + col] = __float2half_rn(v0);
                    act[row * kActStride + col + 1] = __float2half_rn(v1);
                }
            }
    __syncwarp();
}

// Loads the FP16 weights (row stride kActStride) and FP32 biases into shared memory.
__device__ void loadNet(const GuideNetDev& net, __half* sW, float* sB) {
    for (int i = threadIdx.x; i < kWeightRows * kGuideIn; i += blockDim.x) {
        const int r = i / kGuideIn, c = i % kGuideIn;
        sW[r * kActStride + c] = net.w16[r * kGuideIn + c];
    }
    for (int i = threadIdx.x; i < kGParams - kGWCount; i += blockDim.x) sB[i] = __half2float(net.w16[kGWCount + i]);
    __syncthreads();
}

// Row i's features: from an explicit array (features != nullptr) or from a traced path.
struct InferRows {
    const float* features;       // [n][9], or nullptr
    const uint32_t* queue;       // path indices (when features == nullptr)
    const uint32_t* queueCount;  // device count of the queue
    uint64_t n;                  // rows when features != nullptr
    // path inputs
    const float4* rayO;
    const float4* rayD;
    const float* hitT;
    const uint32_t* hitTri;
    const float4* triNg;
    V3 lo, inv;
    float* out;                  // [row or path][kGuideOut]
};

__device__ bool rowFeatures(const InferRows& R, uint64_t i, float f[kGuideFeatures], uint64_t& outRow) {
    if (R.features) {
        for (int k = 0; k < kGuideFeatures; ++k) f[k] = R.features[i * kGuideFeatures + k];
        outRow = i;
        return true;
    }
    const uint32_t path = R.queue[i];
    outRow = path;
    const uint32_t tri = R.hitTri[path];
    if (tri == kNoTriangle) return false;
    const float4 o = R.rayO[path], d = R.rayD[path];
    const float t = R.hitT[path];
    const V3 p{o.x + t * d.x, o.y + t * d.y, o.z + t * d.z};
    const float4 ng = R.triNg[tri];
    f[0] = (p.x - R.lo.x) * R.inv.x; f[1] = (p.y - R.lo.y) * R.inv.y; f[2] = (p.z - R.lo.z) * R.inv.z;
    f[3] = -d.x; f[4] = -d.y; f[5] = -d.z;
    f[6] = ng.x; f[7] = ng.y; f[8] = ng.z;
    return true;
}

__global__ void __launch_bounds__(32 * kInferWarps) k_guide_infer(GuideNetDev net, InferRows R) {
    extern __shared__ __align__(16) unsigned char smem[];
    __half* sW = reinterpret_cast<__half*>(smem);
    float* sB = reinterpret_cast<float*>(sW + kWeightRows * kActStride);
    __half* sAct = reinterpret_cast<__half*>(sB + (kGParams - kGWCount));
    float* sOut = reinterpret_cast<float*>(sAct + kInferWarps * 32 * kActStride);
    loadNet(net, sW, sB);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __half* act = sAct + warp * 32 * kActStride;
    float* out = sOut + warp * 32 * kGuideOut;
    const uint64_t rows = R.features ? R.n : *R.queueCount;
    for (uint64_t base = (blockIdx.x * static_cast<uint64_t>(kInferWarps) + warp) * 32; base < rows;
         base += static_cast<uint64_t>(gridDim.x) * kInferWarps * 32) {
        const uint64_t i = base + lane;
        float f[kGuideFeatures] = {};
        uint64_t outRow = 0;
        const bool valid = i < rows && rowFeatures(R, i, f, outRow);
        float x[kGuideIn];
        guideEncode(f, x);
        for (int c = 0; c < kGuideIn; ++c) act[lane * kActStride + c] = __float2half_rn(valid ? x[c] : 0.0f);
        __syncwarp();
        warpLayer<kGuideWidth, false>(sW + kGW1 / kGuideIn * kActStride, sB + (kGB1 - kGWCount), act, nullptr);
        warpLayer<kGuideWidth, false>(sW + kGW2 / kGuideIn * kActStride, sB + (kGB2 - kGWCount), act, nullptr);
        warpLayer<kGuideWidth, false>(sW + kGW3 / kGuideIn * kActStride, sB + (kGB3 - kGWCount), act, nullptr);
        warpLayer<kGuideOutPad, true>(sW + kGW4 / kGuideIn * kActStride, sB + (kGB4 - kGWCount), act, out);
        if (valid)
            for (int c = 0; c < kGuideOut; ++c) R.out[outRow * kGuideOut + c] = out[lane * kGuideOut + c];
        __syncwarp();
    }
}

// d(-log q(dir))/d(outputs) for one sample; returns -log q.
__device__ float mixtureGrad(const float* out, V3 dir, float* g) {
    float lp[kGuideLobes], lf[kGuideLobes], mxl = -1e30f;
    float kap[kGuideLobes], mlen[kGuideLobes], cosv[kGuideLobes];
    V3 mu[kGuideLobes];
    for (int j = 0; j < kGuideLobes; ++j) mxl = fmaxf(mxl, out[5 * j]);
    float zs = 0;
    for (int j = 0; j < kGuideLobes; ++j) zs += expf(out[5 * j] - mxl);
    const float logZ = mxl + logf(zs);
    float mx = -1e30f;
    for (int j = 0; j < kGuideLobes; ++j) {
        lp[j] = out[5 * j] - logZ;  // log pi_j
        const float lk = fminf(fmaxf(out[5 * j + 1], kLogKappaMin), kLogKappaMax);
        kap[j] = expf(lk);
        const V3 raw{out[5 * j + 2], out[5 * j + 3], out[5 * j + 4]};
        mlen[j] = sqrtf(dot(raw, raw));
        mu[j] = mlen[j] > 1e-12f ? raw * (1.0f / mlen[j]) : V3{0, 0, 1};
        cosv[j] = dot(mu[j], dir);
        lf[j] = lp[j] + vmfLogPdf(mu[j], kap[j], dir);
        mx = fmaxf(mx, lf[j]);
    }
    float s = 0;
    for (int j = 0; j < kGuideLobes; ++j) s += expf(lf[j] - mx);
    const float logq = mx + logf(s);
    for (int j = 0; j < kGuideLobes; ++j) {
        const float r = expf(lf[j] - logq), pi = expf(lp[j]);
        g[5 * j] = pi - r;
        const float lk = out[5 * j + 1];
        const float k = kap[j];
        // d log vMF / d log k = 1 - 2k / (e^2k - 1) + k (c - 1)
        const float dlk = 1 - (k > 1e-4f ? 2 * k / expm1f(2 * k) : 1.0f) + k * (cosv[j] - 1);
        g[5 * j + 1] = (lk > kLogKappaMin && lk < kLogKappaMax) ? -r * dlk : 0.0f;
        const float sc = mlen[j] > 1e-12f ? -r * k / mlen[j] : 0.0f;  // d/dm = -r k (dir - c mu) / |m|
        g[5 * j + 2] = sc * (dir.x - cosv[j] * mu[j].x);
        g[5 * j + 3] = sc * (dir.y - cosv[j] * mu[j].y);
        g[5 * j + 4] = sc * (dir.z - cosv[j] * mu[j].z);
    }
    return -logq;
}

// ---- training on the tensor cores ------------------------------------------------------------
// A block of kTrainWarps warps takes kTrainRows samples, 32 rows per warp. Every layer of the
// forward pass, every back-propagated delta and every weight gradient is a GEMM on the tensor
// cores: mma.sync.m16n8k8 on TF32 operands in split precision (warpGemm) with FP32
// accumulation, operands in shared memory (FP32, row stride kTS). Forward: H = act(X W^T + b),
// with the FP16-rounded weights inference uses. The loss gradient dL/d(outputs) of each sample
// is computed by its own lane in FP32 (mixtureGrad). Backward: dX = (dY W) * relu'(X) per warp,
// and dW += dY^T X, db += column sums of dY over the block's rows, added to the global gradient
// once per block.
constexpr int kTrainWarps = 4;
constexpr int kTrainThreads = 32 * kTrainWarps;
constexpr int kTrainRows = kTrainThreads;
constexpr int kTS = 68;  // FP32 row stride: fragment loads of 8 rows x 4 columns hit 32 banks

__device__ __forceinline__ uint32_t tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void mma1688(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                        uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// An FP32 value as the sum of two TF32 values (hi: x rounded to TF32, lo: the rest rounded).
struct Split { uint32_t hi, lo; };
__device__ __forceinline__ Split split(float x) {
    const uint32_t hi = tf32(x);
    return Split{hi, tf32(x - __uint_as_float(hi))};
}
// One warp: acc[MT][NT] (16 x 8 tiles) += A (MT*16 x KT*8) times B (KT*8 x NT*8), the operands
// read through a(m, k) and b(k, n). Each product is taken in split precision, a_hi b_hi +
// a_hi b_lo + a_lo b_hi (three TF32 MMAs; the dropped a_lo b_lo is ~2^-22 of the product), so
// the result has FP32 accuracy. Fragments (PTX m16n8k8, g = lane / 4, t = lane % 4):
// A: (g, t), (g + 8, t), (g, t + 4), (g + 8, t + 4); B: (t, g), (t + 4, g);
// C: (g, 2t), (g, 2t + 1), (g + 8, 2t), (g + 8, 2t + 1).
// BEXACT: every B value is exactly a TF32 value (an FP16 weight), so its lo part is zero and
// the a_hi b_lo product is left out.
template <int MT, int NT, int KT, bool BEXACT = false, class FA, class FB>
__device__ __forceinline__ void warpGemm(float (&acc)[MT][NT][4], FA a, FB b) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
        const int k = kt * 8 + t;
        Split af[MT][4];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int m = mt * 16 + g;
            af[mt][0] = split(a(m, k));
            af[mt][1] = split(a(m + 8, k));
            af[mt][2] = split(a(m, k + 4));
            af[mt][3] = split(a(m + 8, k + 4));
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int n = nt * 8 + g;
            const Split b0 = split(b(k, n)), b1 = split(b(k + 4, n));
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const Split(&A)[4] = af[mt];
                mma1688(acc[mt][nt], A[0].lo, A[1].lo, A[2].lo, A[3].lo, b0.hi, b1.hi);
                if (!BEXACT) mma1688(acc[mt][nt], A[0].hi, A[1].hi, A[2].hi, A[3].hi, b0.lo, b1.lo);
                mma1688(acc[mt][nt], A[0].hi, A[1].hi, A[2].hi, A[3].hi, b0.hi, b1.hi);
            }
        }
    }
}
template <int MT, int NT>
__device__ __forceinline__ void zero(float (&acc)[MT][NT][4]) {
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
}
// Visits the accumulator's elements: f(row, col, value).
template <int MT, int NT, class F>
__device__ __forceinline__ void forTile(const float (&acc)[MT][NT][4], F f) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) f(mt * 16 + g + 8 * (e >> 1), nt * 8 + 2 * t + (e & 1), acc[mt][nt][e]);
}

// One warp's forward layer: Y = act(X W^T + b), X and Y 32 rows (stride kTS), W [N][64] FP16
// (stride kActStride).
template <int N, bool RELU>
__device__ void fwdLayer(const float* X, const __half* W, const float* bias, float* Y) {
    float acc[2][N / 8][4];
    zero(acc);
    warpGemm<2, N / 8, kGuideIn / 8, true>(acc, [&](int m, int k) { return X[m * kTS + k]; },
                                           [&](int k, int n) { return __half2float(W[n * kActStride + k]); });
    forTile(acc, [&](int r, int c, float v) {
        v += bias[c];
        Y[r * kTS + c] = RELU ? fmaxf(v, 0.0f) : v;
    });
    __syncwarp();
}
// One warp's delta through a layer: dX = (dY W) * relu'(Xact), dY 32 x NOUT, W [NOUT][64].
template <int NOUT>
__device__ void backLayer(const float* dY, const __half* W, const float* Xact, float* dX) {
    float acc[2][kGuideWidth / 8][4];
    zero(acc);
    warpGemm<2, kGuideWidth / 8, NOUT / 8, true>(acc, [&](int m, int k) { return dY[m * kTS + k]; },
                                                 [&](int k, int n) { return __half2float(W[k * kActStride + n]); });
    forTile(acc, [&](int r, int c, float v) { dX[r * kTS + c] = Xact[r * kTS + c] > 0 ? v : 0.0f; });
    __syncwarp();
}
// The block's weight and bias gradients of one layer: dW[n][k] += sum over the block's rows of
// dY[row][n] X[row][k], db[n] += sum dY[row][n]. The warps split the output rows (16-row tiles).
// Buffer b of warp w's activation space, and its row r.
constexpr int kTrainBufs = 5;
constexpr int kBuf = 32 * kTS;
__device__ __forceinline__ float* rowOf(float* acts, int w, int b, int r) {
    return acts + (w * kTrainBufs + b) * kBuf + r * kTS;
}
template <int NOUT>
__device__ void weightGrad(float* acts, int dYbuf, int Xbuf, float* grad, int wOff, int bOff) {
    constexpr int MT = NOUT / 16;
    const int warp = threadIdx.x >> 5;
    for (int mt0 = warp; mt0 < MT; mt0 += kTrainWarps) {
        float acc[1][kGuideIn / 8][4];
        zero(acc);
        warpGemm<1, kGuideIn / 8, kTrainRows / 8>(
            acc, [&](int m, int k) { return rowOf(acts, k >> 5, dYbuf, k & 31)[mt0 * 16 + m]; },
            [&](int k, int n) { return rowOf(acts, k >> 5, Xbuf, k & 31)[n]; });
        forTile(acc, [&](int r, int c, float v) {
            if (v != 0.0f) atomicAdd(&grad[wOff + (mt0 * 16 + r) * kGuideIn + c], v);
        });
    }
    for (int n = threadIdx.x; n < NOUT; n += kTrainThreads) {
        float a = 0;
        for (int row = 0; row < kTrainRows; ++row) a += rowOf(acts, row >> 5, dYbuf, row & 31)[n];
        if (a != 0.0f) atomicAdd(&grad[bOff + n], a);
    }
}

// samples: features (9), dir (3), weight. grad += d(sum_i scale * w_i * -log q_i).
// Per warp five activation buffers A..E (32 rows each): forward X -> A, H1 -> B, H2 -> C,
// H3 -> D, outputs -> E; the loss gradient -> A; deltas: layer 4 -> E, layer 3 -> A, layer 2
// -> E; the inputs X are encoded again into A for the first layer's weight gradient.
__global__ void __launch_bounds__(kTrainThreads) k_guide_grad(GuideNetDev net, const GuideSample* samples, uint64_t n,
                                                              float scale, float* grad, double* loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    __half* sW = reinterpret_cast<__half*>(smem);                              // [kWeightRows][kActStride]
    float* sB = reinterpret_cast<float*>(sW + kWeightRows * kActStride);      // biases
    float* acts = sB + (kGParams - kGWCount);                                 // kTrainWarps x kTrainBufs x 32 rows
    for (int e = threadIdx.x; e < kWeightRows * kGuideIn; e += blockDim.x)
        sW[(e / kGuideIn) * kActStride + e % kGuideIn] = net.w16[e];
    for (int e = threadIdx.x; e < kGParams - kGWCount; e += blockDim.x) sB[e] = net.w32[kGWCount + e];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    enum { A = 0, B = 1, C = 2, D = 3, E = 4 };
    float* buf[kTrainBufs];
    for (int b = 0; b < kTrainBufs; ++b) buf[b] = rowOf(acts, warp, b, 0);
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(kTrainRows) + threadIdx.x;
    const bool valid = i < n;
    float f[kGuideFeatures] = {};
    V3 dir{0, 0, 1};
    float w = 0;
    if (valid) {
        const GuideSample smp = samples[i];
        for (int k = 0; k < kGuideFeatures; ++k) f[k] = smp.feat[k];
        dir = V3{smp.dir[0], smp.dir[1], smp.dir[2]};
        w = smp.weight * scale;
    }
    auto encodeInto = [&](float* X) {
        float x[kGuideIn];
        guideEncode(f, x);
        for (int k = 0; k < kGuideIn; ++k) X[lane * kTS + k] = x[k];
    };
    encodeInto(buf[A]);
    __syncthreads();  // weights and every warp's inputs in place
    const __half* W1 = sW + (kGW1 / kGuideIn) * kActStride;
    const __half* W2 = sW + (kGW2 / kGuideIn) * kActStride;
    const __half* W3 = sW + (kGW3 / kGuideIn) * kActStride;
    const __half* W4 = sW + (kGW4 / kGuideIn) * kActStride;
    fwdLayer<kGuideWidth, true>(buf[A], W1, sB + (kGB1 - kGWCount), buf[B]);
    fwdLayer<kGuideWidth, true>(buf[B], W2, sB + (kGB2 - kGWCount), buf[C]);
    fwdLayer<kGuideWidth, true>(buf[C], W3, sB + (kGB3 - kGWCount), buf[D]);
    fwdLayer<kGuideOutPad, false>(buf[D], W4, sB + (kGB4 - kGWCount), buf[E]);
    // the loss gradient of the lane's own sample, as the delta of the output layer
    {
        float o[kGuideOutPad], g[kGuideOutPad];
        for (int k = 0; k < kGuideOutPad; ++k) { o[k] = buf[E][lane * kTS + k]; g[k] = 0.0f; }
        float nll = 0;
        if (valid && w > 0) {
            nll = mixtureGrad(o, dir, g);
            for (int k = 0; k < kGuideOut; ++k) g[k] *= w;
        }
        if (valid) atomicAdd(loss, static_cast<double>(w * nll));
        for (int k = 0; k < kGuideOutPad; ++k) buf[A][lane * kTS + k] = g[k];
    }
    __syncthreads();
    // layer 4: delta A (48 columns), input H3 = D
    weightGrad<kGuideOutPad>(acts, A, D, grad, kGW4, kGB4);
    backLayer<kGuideOutPad>(buf[A], W4, buf[D], buf[E]);
    __syncthreads();
    // layer 3: delta E, input H2 = C
    weightGrad<kGuideWidth>(acts, E, C, grad, kGW3, kGB3);
    backLayer<kGuideWidth>(buf[E], W3, buf[C], buf[A]);
    __syncthreads();
    // layer 2: delta A, input H1 = B
    weightGrad<kGuideWidth>(acts, A, B, grad, kGW2, kGB2);
    backLayer<kGuideWidth>(buf[A], W2, buf[B], buf[E]);
    __syncthreads();  // every warp is done with A
    encodeInto(buf[A]);
    __syncthreads();
    // layer 1: delta E, input X = A
    weightGrad<kGuideWidth>(acts, E, A, grad, kGW1, kGB1);
}

__global__ void k_guide_adam(float* p, float* g, float* m, float* v, __half* p16, float* p32, int count, float lr,
                             float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi, vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
        p[i] = pi;
        const __half h = __float2half_rn(pi);
        p16[i] = h;
        p32[i] = __half2float(h);
        g[i] = 0.0f;
    }
}

__global__ void k_guide_refresh(const float* p, __half* p16, float* p32, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const __half h = __float2half_rn(p[i]);
        p16[i] = h;
        p32[i] = __half2float(h);
    }
}

constexpr size_t kInferSmem = kWeightRows * kActStride * sizeof(__half) + (kGParams - kGWCount) * sizeof(float) +
                              kInferWarps * 32 * kActStride * sizeof(__half) + kInferWarps * 32 * kGuideOut * sizeof(float);
constexpr size_t kTrainSmem = kWeightRows * kActStride * sizeof(__half) +
                              ((kGParams - kGWCount) + kTrainWarps * kTrainBufs * 32 * kTS) * sizeof(float);
static_assert(kTrainSmem <= 227 * 1024, "training block's shared memory");

}  // namespace crg

struct cr_guide {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevAlloc mem;
    float* p = nullptr;    // FP32 masters
    float* g = nullptr;    // gradient
    float* m = nullptr;
    float* v = nullptr;
    __half* p16 = nullptr;
    float* p32 = nullptr;  // FP16-rounded values as FP32
    double* loss = nullptr;
    uint64_t step = 0;
    int inferGrid = 0;
    DevAlloc scratch;      // caller data for the test entry points
    size_t scratchBytes = 0;
    void* scratchPtr = nullptr;

    GuideNetDev net() const { return GuideNetDev{p16, p32}; }
    void* ensureScratch(size_t bytes) {
        if (bytes > scratchBytes) {
            scratch.release();
            scratchPtr = nullptr;  // until the larger block exists (its allocation may fail)
            scratchBytes = 0;
            scratchPtr = scratch.alloc<unsigned char>(bytes);
            scratchBytes = bytes;
        }
        return scratchPtr;
    }
    ~cr_guide() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        mem.release();
        scratch.release();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace crg {

void guideAttributes() {
    static bool done = false;
    if (done) return;
    CR_CUDA(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kInferSmem)));
    CR_CUDA(cudaFuncSetAttribute(k_guide_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTrainSmem)));
    done = true;
}

// Inference over a traced path queue (guided renders): out[path][40] for the paths of `queue`.
void guideInferPaths(cr_guide* gd, cudaStream_t s, const uint32_t* queue, const uint32_t* queueCount, uint32_t maxRows,
                     const PathSoA& st, const float* hitT, const DevScene& S, V3 lo, V3 inv, float* out) {
    guideAttributes();
    InferRows R{};
    R.queue = queue; R.queueCount = queueCount;
    R.rayO = st.ray_o; R.rayD = st.ray_d; R.hitT = hitT; R.hitTri = st.hit_tri; R.triNg = S.tri_ng;
    R.lo = lo; R.inv = inv; R.out = out;
    const uint32_t rowsPerBlock = 32 * kInferWarps;
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(static_cast<uint32_t>(gd->inferGrid),
                                                                     (maxRows + rowsPerBlock - 1) / rowsPerBlock));
    k_guide_infer<<<blocks, 32 * kInferWarps, kInferSmem, s>>>(gd->net(), R);
    CR_CUDA(cudaGetLastError());
}

__global__ void k_guide_weight_sum(const GuideSample* samples, uint64_t n, double* sum) {
    double a = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        a += samples[i].weight;
    for (int o = 16; o; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, a);
}

// Adam steps on device-resident samples: `steps` mini-batches of `batch` consecutive samples
// (wrapping around), loss weights normalised by the collection's mean weight.
float guideTrain(cr_guide* gd, cudaStream_t s, const GuideSample* samples, uint64_t n, uint32_t steps, uint32_t batch,
                 float lr, double weightMean) {
    guideAttributes();
    if (n == 0 || steps == 0) return 0.0f;
    if (weightMean <= 0) {
        CR_CUDA(cudaMemsetAsync(gd->loss, 0, sizeof(double), s));
        k_guide_weight_sum<<<256, 256, 0, s>>>(samples, n, gd->loss);
        double sum = 0;
        CR_CUDA(cudaMemcpyAsync(&sum, gd->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        weightMean = sum / static_cast<double>(n);
    }
    const uint64_t b = std::min<uint64_t>(batch, n);
    const float scale = static_cast<float>(1.0 / (static_cast<double>(b) * (weightMean > 0 ? weightMean : 1.0)));
    double lossHost = 0;
    uint64_t at = 0;
    for (uint32_t k = 0; k < steps; ++k) {
        const uint64_t count = std::min<uint64_t>(b, n - at);
        CR_CUDA(cudaMemsetAsync(gd->loss, 0, sizeof(double), s));
        k_guide_grad<<<static_cast<unsigned>((count + kTrainRows - 1) / kTrainRows), kTrainThreads, kTrainSmem, s>>>(
            gd->net(), samples + at, count, scale, gd->g, gd->loss);
        ++gd->step;
        const float bc1 = 1.0f - std::pow(0.9f, static_cast<float>(gd->step));
        const float bc2 = 1.0f - std::pow(0.999f, static_cast<float>(gd->step));
        k_guide_adam<<<64, 256, 0, s>>>(gd->p, gd->g, gd->m, gd->v, gd->p16, gd->p32, kGParams, lr, bc1, bc2);
        CR_CUDA(cudaGetLastError());
        at = (at + count) % n;
    }
    CR_CUDA(cudaMemcpyAsync(&lossHost, gd->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    return static_cast<float>(lossHost);
}

}  // namespace crg

extern "C" {

uint32_t cr_guide_parameter_count(void) { return kGParams; }

cr_status cr_guide_create(int device, uint64_t seed, cr_guide** out) {
    try {
        if (!out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        CR_CUDA(cudaSetDevice(device));
        auto gd = std::make_unique<cr_guide>();
        gd->device = device;
        CR_CUDA(cudaStreamCreateWithFlags(&gd->stream, cudaStreamNonBlocking));
        gd->p = gd->mem.alloc<float>(kGParams);
        gd->g = gd->mem.alloc<float>(kGParams);
        gd->m = gd->mem.alloc<float>(kGParams);
        gd->v = gd->mem.alloc<float>(kGParams);
        gd->p16 = gd->mem.alloc<__half>(kGParams);
        gd->p32 = gd->mem.alloc<float>(kGParams);
        gd->loss = gd->mem.alloc<double>(1);
        // He-uniform hidden layers, a small output layer: lobes start broad (kappa 1), equally
        // weighted, with means along seeded random directions.
        std::vector<float> h(kGParams, 0.0f);
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<float> uni(-1.0f, 1.0f);
        const float lim = std::sqrt(6.0f / kGuideIn);
        for (int i = kGW1; i < kGW4; ++i) h[i] = lim * uni(rng);
        for (int r = 0; r < kGuideOut; ++r)
            for (int k = 0; k < kGuideIn; ++k) h[kGW4 + r * kGuideIn + k] = 1e-3f * uni(rng);
        for (int j = 0; j < kGuideLobes; ++j) {
            std::normal_distribution<float> nd;
            float a = nd(rng), b = nd(rng), c = nd(rng);
            const float l = std::sqrt(a * a + b * b + c * c) + 1e-12f;
            h[kGB4 + 5 * j + 2] = a / l; h[kGB4 + 5 * j + 3] = b / l; h[kGB4 + 5 * j + 4] = c / l;
        }
        CR_CUDA(cudaMemcpyAsync(gd->p, h.data(), kGParams * sizeof(float), cudaMemcpyHostToDevice, gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->g, 0, kGParams * sizeof(float), gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->m, 0, kGParams * sizeof(float), gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->v, 0, kGParams * sizeof(float), gd->stream));
        k_guide_refresh<<<64, 256, 0, gd->stream>>>(gd->p, gd->p16, gd->p32, kGParams);
        CR_CUDA(cudaGetLastError());
        CR_CUDA(cudaStreamSynchronize(gd->stream));
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        gd->inferGrid = sms * 2;
        guideAttributes();
        *out = gd.release();
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_guide_destroy(cr_guide* gd) {
    delete gd;
    return CR_OK;
}

cr_status cr_guide_get_parameters(cr_guide* gd, float* out) {
    try {
        if (!gd || !out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        CR_CUDA(cudaSetDevice(gd->device));
        CR_CUDA(cudaMemcpyAsync(out, gd->p, kGParams * sizeof(float), cudaMemcpyDeviceToHost, gd->stream));
        CR_CUDA(cudaStreamSynchronize(gd->stream));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_guide_set_parameters(cr_guide* gd, const float* in) {
    try {
        if (!gd || !in) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        CR_CUDA(cudaSetDevice(gd->device));
        CR_CUDA(cudaMemcpyAsync(gd->p, in, kGParams * sizeof(float), cudaMemcpyHostToDevice, gd->stream));
        k_guide_refresh<<<64, 256, 0, gd->stream>>>(gd->p, gd->p16, gd->p32, kGParams);
        CR_CUDA(cudaGetLastError());
        CR_CUDA(cudaStreamSynchronize(gd->stream));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_guide_evaluate(cr_guide* gd, const float* features, uint64_t n, float* out) {
    try {
        if (!gd || !features || !out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        if (n == 0) return CR_OK;
        CR_CUDA(cudaSetDevice(gd->device));
        const size_t inBytes = n * kGuideFeatures * sizeof(float), outBytes = n * kGuideOut * sizeof(float);
        unsigned char* buf = static_cast<unsigned char*>(gd->ensureScratch(inBytes + outBytes + 256));
        float* dIn = reinterpret_cast<float*>(buf);
        float* dOut = reinterpret_cast<float*>(buf + (inBytes + 255) / 256 * 256);
        CR_CUDA(cudaMemcpyAsync(dIn, features, inBytes, cudaMemcpyHostToDevice, gd->stream));
        InferRows R{};
        R.features = dIn; R.n = n; R.out = dOut;
        const uint64_t blocks = std::min<uint64_t>(static_cast<uint64_t>(gd->inferGrid), (n + 127) / 128);
        k_guide_infer<<<static_cast<unsigned>(std::max<uint64_t>(1, blocks)), 32 * kInferWarps, kInferSmem, gd->stream>>>(gd->net(), R);
        CR_CUDA(cudaGetLastError());
        CR_CUDA(cudaMemcpyAsync(out, dOut, outBytes, cudaMemcpyDeviceToHost, gd->stream));
        CR_CUDA(cudaStreamSynchronize(gd->stream));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

// samples: n x 13 floats (features 9, direction 3, weight). grad receives
// d/dparams of sum_i w_i * -log q_i(dir_i); *loss that sum.
cr_status cr_guide_gradients(cr_guide* gd, const float* samples, uint64_t n, float* grad, double* loss) {
    try {
        if (!gd || !samples || !grad || !loss) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        CR_CUDA(cudaSetDevice(gd->device));
        static_assert(sizeof(GuideSample) == 13 * sizeof(float), "GuideSample is 13 floats");
        GuideSample* d = static_cast<GuideSample*>(gd->ensureScratch(n * sizeof(GuideSample) + 16));
        CR_CUDA(cudaMemcpyAsync(d, samples, n * sizeof(GuideSample), cudaMemcpyHostToDevice, gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->g, 0, kGParams * sizeof(float), gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->loss, 0, sizeof(double), gd->stream));
        k_guide_grad<<<static_cast<unsigned>((n + kTrainRows - 1) / kTrainRows), kTrainThreads, kTrainSmem, gd->stream>>>(
            gd->net(), d, n, 1.0f, gd->g, gd->loss);
        CR_CUDA(cudaGetLastError());
        CR_CUDA(cudaMemcpyAsync(grad, gd->g, kGParams * sizeof(float), cudaMemcpyDeviceToHost, gd->stream));
        CR_CUDA(cudaMemcpyAsync(loss, gd->loss, sizeof(double), cudaMemcpyDeviceToHost, gd->stream));
        CR_CUDA(cudaMemsetAsync(gd->g, 0, kGParams * sizeof(float), gd->stream));
        CR_CUDA(cudaStreamSynchronize(gd->stream));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

// Adam on caller samples (host memory): `steps` mini-batches of `batch`; *loss receives the
// last batch's normalised loss.
cr_status cr_guide_train(cr_guide* gd, const float* samples, uint64_t n, uint32_t steps, uint32_t batch, float lr,
                         float* loss) {
    try {
        if (!gd || !samples || n == 0) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        CR_CUDA(cudaSetDevice(gd->device));
        GuideSample* d = static_cast<GuideSample*>(gd->ensureScratch(n * sizeof(GuideSample) + 16));
        CR_CUDA(cudaMemcpyAsync(d, samples, n * sizeof(GuideSample), cudaMemcpyHostToDevice, gd->stream));
        double mean = 0;
        for (uint64_t i = 0; i < n; ++i) mean += samples[13 * i + 12];
        mean /= static_cast<double>(n);
        const float l = guideTrain(gd, gd->stream, d, n, steps, batch, lr, mean);
        if (loss) *loss = l;
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"
