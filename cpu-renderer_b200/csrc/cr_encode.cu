// Device-side output encoding of a linear RGB film: the pixels io::writePng hands to its PNG
// codec (filmic curve + sRGB + 8 bits, src/io/image.cpp:116-124, 193-212), the RGBE quads and
// the complete Radiance file io::writeHdr writes (image.cpp:216-230) through stb_image_write
// 1.16 (third_party/stb_image_write.h: stbiw__linear_to_rgbe, stbiw__write_hdr_scanline,
// stbi_write_hdr_core), restated here from the codec's published algorithm.
//
// Kernels (all HBM-bound byte work, grid-stride over the film):
//   k_check      validateOutput (image.cpp:100-113): first non-finite/negative pixel and, for
//                RGBE, first pixel at or above 2^127, as atomic minima of the pixel index.
//   k_srgb8      one pixel per thread: the display byte of each channel by binary search in a
//                256-entry threshold table (built on the host with the reference's own
//                arithmetic, crh::display_thresholds), so bytes equal displayChannel's.
//   k_rgbe       one pixel per thread: shared-exponent quad.
//   k_rle        one (scanline, component) per thread: the codec's greedy run-length coding.
//   k_row_scan   one block: exclusive scan of scanline sizes.
//   k_gather     one block per scanline: scanline header + four component segments.
#include "cr_encode.h"

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cr_gpu.h"
#include "cr_host.h"

namespace crg {
namespace {

#define ENC_CUDA(x)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) throw crh::Error(CR_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

constexpr unsigned long long kNone = ~0ull;
constexpr float kRgbeLimit = 1.70141183460469231731687303715884105728e38f;  // 2^127, image.cpp:109

struct Check {
    unsigned long long badValue;  // first pixel not finite or negative
    unsigned long long badRange;  // first (otherwise valid) pixel at or above 2^127
    unsigned long long rowBytes;  // total scanline bytes (k_row_scan)
};

__global__ void k_check(const float* __restrict__ film, uint64_t n, int hdr, Check* chk) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const float r = film[3 * i], g = film[3 * i + 1], b = film[3 * i + 2];
        if (!(isfinite(r) && isfinite(g) && isfinite(b)) || r < 0 || g < 0 || b < 0)
            atomicMin(&chk->badValue, static_cast<unsigned long long>(i));
        else if (hdr && fmaxf(r, fmaxf(g, b)) >= kRgbeLimit)
            atomicMin(&chk->badRange, static_cast<unsigned long long>(i));
    }
}

__global__ void __launch_bounds__(256) k_srgb8(const float* __restrict__ film, uint64_t n, const float* __restrict__ thresholds,
                                               unsigned char* __restrict__ out) {
    __shared__ float T[256];
    T[threadIdx.x] = thresholds[threadIdx.x];
    __syncthreads();
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < 3 * n; i += uint64_t(gridDim.x) * blockDim.x) {
        const float v = film[i];
        int k = 0;
#pragma unroll
        for (int step = 128; step; step >>= 1)
            if (T[k + step] <= v) k += step;  // largest k with T[k] <= v: displayChannel(v)
        out[i] = static_cast<unsigned char>(k);
    }
}

// stbiw__linear_to_rgbe. The float-to-byte conversions go through int, as x86-64 code for
// the codec does, so a product that rounds up to 256.0 wraps the same way.
__device__ __forceinline__ uchar4 rgbe(float r, float g, float b) {
    const float gb = g > b ? g : b;
    const float m = r > gb ? r : gb;
    if (m < 1e-32f) return make_uchar4(0, 0, 0, 0);
    int e;
    const float mant = frexpf(m, &e);
    const float normalize = mant * 256.0f / m;
    return make_uchar4(static_cast<unsigned char>(static_cast<int>(r * normalize)),
                       static_cast<unsigned char>(static_cast<int>(g * normalize)),
                       static_cast<unsigned char>(static_cast<int>(b * normalize)),
                       static_cast<unsigned char>(e + 128));
}

__global__ void k_rgbe(const float* __restrict__ film, uint64_t n, uchar4* __restrict__ out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = rgbe(film[3 * i], film[3 * i + 1], film[3 * i + 2]);
}

// stbiw__write_hdr_scanline's run-length coding of one component of one scanline: find the
// next run of three equal bytes, dump the bytes before it in pieces of at most 128 (count
// byte, then the bytes), then the run in pieces of at most 127 (128 + count, then the byte).
__global__ void k_rle(const uchar4* __restrict__ quads, int width, int height, unsigned char* __restrict__ seg,
                      uint32_t segCap, uint32_t* __restrict__ segLen) {
    const uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (t >= 4ull * height) return;
    const int y = static_cast<int>(t >> 2), c = static_cast<int>(t & 3);
    const unsigned char* row = reinterpret_cast<const unsigned char*>(quads + static_cast<uint64_t>(y) * width) + c;
    auto comp = [&](int x) { return row[4 * x]; };
    unsigned char* o = seg + t * segCap;
    uint32_t len = 0;
    int x = 0;
    while (x < width) {
        int r = x;
        while (r + 2 < width) {
            const unsigned char a = comp(r);
            if (a == comp(r + 1) && a == comp(r + 2)) break;
            ++r;
        }
        if (r + 2 >= width) r = width;
        while (x < r) {
            const int n = min(r - x, 128);
            o[len++] = static_cast<unsigned char>(n);
            for (int k = 0; k < n; ++k) o[len++] = comp(x + k);
            x += n;
        }
        if (r + 2 < width) {
            const unsigned char v = comp(x);
            while (r < width && comp(r) == v) ++r;
            while (x < r) {
                const int n = min(r - x, 127);
                o[len++] = static_cast<unsigned char>(n + 128);
                o[len++] = v;
                x += n;
            }
        }
    }
    segLen[t] = len;
}

// Exclusive scan of the scanline sizes (4 + the four segments) by one 1024-thread block.
__global__ void __launch_bounds__(1024) k_row_scan(const uint32_t* __restrict__ segLen, int height,
                                                   unsigned long long* __restrict__ rowOff, Check* chk) {
    __shared__ unsigned long long part[1024];
    const int per = (height + 1023) / 1024;
    const int y0 = threadIdx.x * per, y1 = min(height, y0 + per);
    unsigned long long sum = 0;
    for (int y = y0; y < y1; ++y)
        sum += 4ull + segLen[4 * y] + segLen[4 * y + 1] + segLen[4 * y + 2] + segLen[4 * y + 3];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
        const unsigned long long v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int y = y0; y < y1; ++y) {
        rowOff[y] = run;
        run += 4ull + segLen[4 * y] + segLen[4 * y + 1] + segLen[4 * y + 2] + segLen[4 * y + 3];
    }
    if (threadIdx.x == 1023) chk->rowBytes = part[1023];
}

__global__ void k_gather(const unsigned char* __restrict__ seg, uint32_t segCap, const uint32_t* __restrict__ segLen,
                         const unsigned long long* __restrict__ rowOff, int width, unsigned char* __restrict__ out) {
    const int y = blockIdx.x;
    unsigned char* o = out + rowOff[y];
    if (threadIdx.x == 0) {
        o[0] = 2; o[1] = 2;
        o[2] = static_cast<unsigned char>((width & 0xff00) >> 8);
        o[3] = static_cast<unsigned char>(width & 0xff);
    }
    uint64_t at = 4;
    for (int c = 0; c < 4; ++c) {
        const uint64_t t = 4ull * y + c;
        const uint32_t n = segLen[t];
        const unsigned char* src = seg + t * segCap;
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) o[at + k] = src[k];
        at += n;
    }
}

}  // namespace

// Device buffers of one device, grown on demand and kept for later calls.
struct EncodeCache {
    std::mutex encodeMutex;  // the device buffers below
    std::mutex filmMutex;    // film and stream
    unsigned char* body = nullptr; uint64_t bodyCap = 0;
    unsigned char* seg = nullptr; uint64_t segBytes = 0;
    uint32_t* segLen = nullptr; uint64_t segCount = 0;
    unsigned long long* rowOff = nullptr; uint64_t rows = 0;
    float* thresholds = nullptr;
    Check* check = nullptr;
    Check* hostCheck = nullptr;  // pinned
    int grid = 0;
    float* film = nullptr; uint64_t filmFloats = 0;  // a caller's film (cr_gpu_encode)
    cudaStream_t stream = nullptr;
};

EncodeCache& cacheFor(int device) {
    static std::mutex registry;
    static std::vector<EncodeCache*> caches;
    std::lock_guard<std::mutex> lock(registry);
    if (device >= static_cast<int>(caches.size())) caches.resize(device + 1, nullptr);
    if (!caches[device]) caches[device] = new EncodeCache();  // lives until the process exits
    return *caches[device];
}

template <class T>
void grow(T*& p, uint64_t& cap, uint64_t need) {
    if (need <= cap) return;
    if (p) ENC_CUDA(cudaFree(p));
    p = nullptr;
    cap = 0;
    crh::count_allocation();
    if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        throw crh::Error(CR_ERR_OUT_OF_MEMORY, "device allocation for output encoding failed");
    }
    cap = need;
}

uint64_t encode_film(const float* dFilm, int width, int height, int format, float exposure, cudaStream_t s,
                     void* out, uint64_t capacity) {
    const bool png = format == CR_ENCODE_SRGB8;
    const bool hdrFile = format == CR_ENCODE_HDR_FILE;
    if (!png && format != CR_ENCODE_RGBE && !hdrFile) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "unknown encode format");
    const std::string label = png ? "PNG output" : "HDR output";
    crh::check_image_dims(width, height, label);
    float thresholds[256];
    std::string exposureError;  // io::writePng checks the exposure after the pixels
    if (png) {
        try {
            crh::display_thresholds(exposure, thresholds);
        } catch (const crh::Error& e) {
            exposureError = e.what();
        }
    }
    const uint64_t n = static_cast<uint64_t>(width) * height;
    int device = 0;
    ENC_CUDA(cudaGetDevice(&device));
    EncodeCache& E = cacheFor(device);
    std::lock_guard<std::mutex> lock(E.encodeMutex);
    if (!E.check) {
        // E.check is set last: until every buffer exists the next call sets them up again
        for (int k = 0; k < 3; ++k) crh::count_allocation();
        if (!E.thresholds) ENC_CUDA(cudaMalloc(&E.thresholds, 256 * sizeof(float)));
        if (!E.hostCheck) ENC_CUDA(cudaMallocHost(&E.hostCheck, sizeof(Check)));
        int sms = 0;
        ENC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        E.grid = sms * 8;
        Check* check = nullptr;
        ENC_CUDA(cudaMalloc(&check, sizeof(Check)));
        E.check = check;
    }
    const Check init{kNone, kNone, 0};
    ENC_CUDA(cudaMemcpyAsync(E.check, &init, sizeof(Check), cudaMemcpyHostToDevice, s));
    k_check<<<E.grid, 256, 0, s>>>(dFilm, n, png ? 0 : 1, E.check);
    ENC_CUDA(cudaGetLastError());

    const bool rle = hdrFile && width >= 8 && width < 32768;  // stbiw__write_hdr_scanline
    const std::string header = hdrFile ? crh::hdr_header(width, height) : std::string();
    const uint64_t quadBytes = 4 * n;
    uint64_t bodyBytes = png ? 3 * n : quadBytes;
    uint64_t segCap = 0;
    if (png && exposureError.empty()) {
        grow(E.body, E.bodyCap, 3 * n);
        ENC_CUDA(cudaMemcpyAsync(E.thresholds, thresholds, sizeof(thresholds), cudaMemcpyHostToDevice, s));
        k_srgb8<<<E.grid, 256, 0, s>>>(dFilm, n, E.thresholds, E.body);
    } else if (!png) {
        // quads first; scanline segments (at most 2 bytes per input byte) and the body after
        segCap = rle ? 2ull * width + 2 : 0;
        const uint64_t segTotal = rle ? 4ull * height * segCap : 0;
        grow(E.seg, E.segBytes, quadBytes + segTotal + 16);
        k_rgbe<<<E.grid, 256, 0, s>>>(dFilm, n, reinterpret_cast<uchar4*>(E.seg));
        if (rle) {
            grow(E.segLen, E.segCount, 4ull * height);
            grow(E.rowOff, E.rows, static_cast<uint64_t>(height));
            unsigned char* segs = E.seg + (quadBytes + 15) / 16 * 16;
            k_rle<<<static_cast<unsigned>((4ull * height + 127) / 128), 128, 0, s>>>(
                reinterpret_cast<const uchar4*>(E.seg), width, height, segs, static_cast<uint32_t>(segCap), E.segLen);
            k_row_scan<<<1, 1024, 0, s>>>(E.segLen, height, E.rowOff, E.check);
            grow(E.body, E.bodyCap, static_cast<uint64_t>(height) * (4 + 4 * segCap));
            k_gather<<<height, 128, 0, s>>>(segs, static_cast<uint32_t>(segCap), E.segLen, E.rowOff, width, E.body);
        }
    }
    ENC_CUDA(cudaGetLastError());
    ENC_CUDA(cudaMemcpyAsync(E.hostCheck, E.check, sizeof(Check), cudaMemcpyDeviceToHost, s));
    ENC_CUDA(cudaStreamSynchronize(s));
    const Check c = *E.hostCheck;
    if (c.badValue != kNone && (c.badRange == kNone || c.badValue < c.badRange))
        throw crh::Error(CR_ERR_INVALID_ARGUMENT, label + ": pixels must contain finite, nonnegative linear radiance");
    if (c.badRange != kNone)
        throw crh::Error(CR_ERR_INVALID_ARGUMENT, label + ": radiance exceeds the Radiance RGBE exponent range");
    if (!exposureError.empty()) throw crh::Error(CR_ERR_INVALID_ARGUMENT, exposureError);
    if (rle) bodyBytes = c.rowBytes;
    const uint64_t total = header.size() + bodyBytes;
    if (!out || capacity < total) return total;
    unsigned char* o = static_cast<unsigned char*>(out);
    std::memcpy(o, header.data(), header.size());
    const unsigned char* src = png || rle ? E.body : E.seg;
    ENC_CUDA(cudaMemcpyAsync(o + header.size(), src, bodyBytes, cudaMemcpyDeviceToHost, s));
    ENC_CUDA(cudaStreamSynchronize(s));
    return total;
}

}  // namespace crg

extern "C" cr_status cr_gpu_encode(const float* film_rgb, int width, int height, int format, float exposure, int device,
                                   void* out, uint64_t capacity, uint64_t* size) {
    try {
        if (!film_rgb || !size) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        crh::check_image_dims(width, height, format == CR_ENCODE_SRGB8 ? "PNG output" : "HDR output");
        ENC_CUDA(cudaSetDevice(device));
        crg::EncodeCache& E = crg::cacheFor(device);
        std::lock_guard<std::mutex> lock(E.filmMutex);
        if (!E.stream) ENC_CUDA(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
        const uint64_t floats = 3ull * width * height;
        crg::grow(E.film, E.filmFloats, floats);
        ENC_CUDA(cudaMemcpyAsync(E.film, film_rgb, floats * sizeof(float), cudaMemcpyHostToDevice, E.stream));
        const uint64_t n = crg::encode_film(E.film, width, height, format, exposure, E.stream, out, capacity);
        *size = n;
        if (out && capacity < n)
            return crh::set_last_error(CR_ERR_OUT_OF_RANGE, "output buffer holds " + std::to_string(capacity) +
                                                                " bytes; the encoding needs " + std::to_string(n));
        return CR_OK;
    } catch (const crh::Error& e) {
        return crh::set_last_error(e.status, e.what());
    } catch (const std::exception& e) {
        return crh::set_last_error(CR_ERR_CUDA, e.what());
    }
}
