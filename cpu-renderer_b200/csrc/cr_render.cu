// Wavefront path tracer for sm_100a: kernels and the host driver behind include/cr_gpu.h.
//
// One render (cr::render, render.cpp:352-456) runs a pool of path slots. Camera samples are
// numbered sample-major (id = sample * pixels + pixel) and issued in order to free slots, a
// chunk of ids at a time (by default one pool's worth: every slot starts a sample at the
// chunk's first iteration and the chunk drains). Every iteration runs these launches:
//
//   k_regen   free slots take the next sample ids: jitter + camera ray   (render.cpp:396-401)
//   k_trace   closest hit for the live queue (Bvh::intersect, geometry.cpp:554) and any hit for
//             the shadow rays queued by the previous iteration, in one launch
//   k_shade   one trace() iteration per live path (render.cpp:240-344), one launch per
//             material class -> next live queue, shadow queue, free queue (warp ballots)
//
// Warps take 32-entry batches of a queue from a counter, so a launch ends when its work does.
// Scenes without alpha masks, textures or punctual lights run instantiations compiled without
// that code. Each path keeps the reference's order of random draws and radiance sums, so a
// camera sample consumes the same SplitMix stream as on the CPU. Every sample's radiance is
// stored by id; at the end of a chunk of ids, k_accumulate adds each pixel's samples in index
// order into FP64 sums (render.cpp:388-415), so the film does not depend on scheduling.
// Precision replay (render.cpp:403-412) resets a failing path to its camera ray with split
// origins and runs it again in the same pool.
#include "cr_kernels.cuh"
#include "cr_driver.h"
#include "cr_encode.h"
#include "cr_host.h"

#include <atomic>
#include <chrono>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

// =============================================================================================
// Host driver
// =============================================================================================
using namespace crg;
using namespace crd;

namespace crd {

cr_status fail(const std::exception& e) {
    if (const auto* x = dynamic_cast<const crh::Error*>(&e)) return crh::set_last_error(x->status, x->what());
    if (dynamic_cast<const std::bad_alloc*>(&e)) return crh::set_last_error(CR_ERR_OUT_OF_MEMORY, "host allocation failed");
    return crh::set_last_error(CR_ERR_CUDA, e.what());
}

cr_gpu_tuning defaults(const cr_gpu_tuning* t) {
    cr_gpu_tuning d{};
    if (t) d = *t;
    return d;
}

RenderParams makeParams(const cr_camera& camera, const cr_render_options& o, const cr_gpu_tuning& t) {
    RenderParams P{};
    P.width = o.width; P.height = o.height; P.samples = o.samples; P.bounces = o.bounces;
    P.seed = o.seed; P.nee = o.next_event_estimation != 0; P.rr = o.russian_roulette != 0;
    P.env_alias = t.env_alias; P.exact_traversal = t.exact_traversal;
    crh::camera_setup(camera, o.width, o.height, P.camera);
    return P;
}

int referenceWorkers(const cr_render_options& o) {  // render.cpp:361-363
    constexpr int tileSize = 16;
    const int tilesX = (o.width + tileSize - 1) / tileSize, tilesY = (o.height + tileSize - 1) / tileSize, tiles = tilesX * tilesY;
    const int automatic = static_cast<int>(std::max(1u, std::thread::hardware_concurrency() / 2));
    return std::min(tiles, o.threads ? o.threads : automatic);
}

}  // namespace crd

// Render work buffers of one device: the path pool, its queues, the chunk's per-sample
// radiance and the host staging words. Kept for the life of the process and shared by every
// scene on the device (a render holds the mutex), so a new scene does not pay for fresh
// multi-gigabyte allocations.
struct Workspace {
    int device = 0;
    std::mutex mutex;
    DevAlloc work, outAlloc, packedAlloc;
    size_t capacity = 0, outCapacity = 0, packedCapacity = 0;
    PathSoA st{};
    Queues q{};
    uint32_t* counts = nullptr;
    unsigned long long* stats = nullptr;
    DevError* detail = nullptr;
    float* packed = nullptr;
    uint32_t* hostCounts = nullptr;           // pinned
    unsigned long long* hostStats = nullptr;  // pinned
    int gridTrace = 0, gridShade = 0, gridShadeLight = 0, gridShadeMiss = 0, gridRegen = 0, gridSmall = 0;
    int gridShadeLean = 0, gridShadeLightLean = 0, gridShadeMissLean = 0, gridTraceNoAlpha = 0;
    int gridShadeCond = 0, gridShadeCondLean = 0;
    std::vector<cudaEvent_t> events;
    // more streams for the shading launches that run beside the generic one
    static constexpr int kSide = 3;
    cudaStream_t side[kSide] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[kSide] = {nullptr, nullptr, nullptr};

    // Each handle is taken only once it exists, so a creation that fails part-way is completed
    // by the next call instead of leaving a null stream (the legacy default stream) or event.
    void ensureSideStreams() {
        if (!fork) {
            cudaEvent_t e = nullptr;
            CR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            fork = e;
        }
        for (int k = 0; k < kSide; ++k) {
            if (!side[k]) {
                cudaStream_t st = nullptr;
                CR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                side[k] = st;
            }
            if (!join[k]) {
                cudaEvent_t e = nullptr;
                CR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                join[k] = e;
            }
        }
    }

    cudaEvent_t event(size_t i) {
        while (events.size() <= i) {
            cudaEvent_t e;
            CR_CUDA(cudaEventCreate(&e));
            events.push_back(e);
        }
        return events[i];
    }
    void ensureWork(size_t paths) {
        if (paths <= capacity) return;
        work.release();
        capacity = 0;
        const size_t n = paths;
        allocPaths(work, n, st, q);
        counts = q.counts;
        stats = work.alloc<unsigned long long>(kStatWords);
        detail = work.alloc<DevError>(1);
        capacity = n;
    }
    void ensureOut(size_t samples) {
        if (samples <= outCapacity) return;
        outAlloc.release();
        outCapacity = 0;
        st.out = outAlloc.alloc<float4>(samples);
        outCapacity = samples;
    }
    void ensurePacked(size_t samples) {
        if (samples <= packedCapacity) return;
        packedAlloc.release();
        packedCapacity = 0;
        packed = packedAlloc.alloc<float>(3 * samples);
        packedCapacity = samples;
    }
    uint64_t bytes() const { return work.bytes + outAlloc.bytes + packedAlloc.bytes; }
};

// One workspace per device, created on first use and intentionally never destroyed (process
// exit reclaims device memory; destroying after the CUDA runtime has shut down would fail).
Workspace& workspaceFor(int device) {
    static std::mutex m;
    static Workspace* ws[64] = {};
    if (device < 0 || device >= 64) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(m);
    if (!ws[device]) { ws[device] = new Workspace; ws[device]->device = device; }
    return *ws[device];
}


namespace {

template <class T> struct ArrayView {
    const T* p;
    size_t n;
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
    const T& operator[](size_t i) const { return p[i]; }
};

// One host block for the arrays a scene upload builds (page-locked when that can be had, so
// their copies run asynchronously). The destructor waits for the stream's copies before the
// block goes back to the cache.
class Staging {
  public:
    Staging(cudaStream_t s, size_t bytes) : s_(s) {
        auto [q, have] = PinnedCache::get().take(bytes);
        if (q) { p_ = static_cast<unsigned char*>(q); size_ = have; pinned_ = true; }
        else { fallback_.reset(new unsigned char[bytes]); p_ = fallback_.get(); size_ = bytes; }
    }
    Staging(const Staging&) = delete;
    Staging& operator=(const Staging&) = delete;
    ~Staging() {
        cudaStreamSynchronize(s_);
        if (pinned_) PinnedCache::get().give(p_, size_);
    }
    static size_t bytesFor(size_t bytes) { return (bytes + 255) / 256 * 256; }
    template <class T> T* carve(size_t count) {
        T* r = reinterpret_cast<T*>(p_ + used_);
        used_ += bytesFor(count * sizeof(T));
        if (used_ > size_) throw std::logic_error("staging block too small");
        return r;
    }

  private:
    cudaStream_t s_;
    unsigned char* p_ = nullptr;
    size_t size_ = 0, used_ = 0;
    bool pinned_ = false;
    std::unique_ptr<unsigned char[]> fallback_;
};

// Copies host memory (the caller's, pageable) to the device through page-locked chunks: a few
// host threads fill one chunk while the chunks before it are in transfer, so the copy runs near
// the host's memcpy rate rather than the driver's pageable path (~9 GB/s measured). Returns when
// the copy is complete.
void stagedUpload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    constexpr size_t kChunk = size_t{16} << 20;
    constexpr int kRing = 3;
    if (bytes < kChunk) {
        CR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaStreamSynchronize(s));
        return;
    }
    auto [block, have] = PinnedCache::get().take(kRing * kChunk);
    if (!block) {  // no page-locked memory to be had: the driver's own path
        CR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaStreamSynchronize(s));
        return;
    }
    struct Ring {
        void* block;
        size_t size;
        cudaStream_t s;
        cudaEvent_t done[kRing] = {};
        ~Ring() {
            cudaStreamSynchronize(s);
            for (cudaEvent_t e : done) if (e) cudaEventDestroy(e);
            PinnedCache::get().give(block, size);
        }
    } ring{block, have, s};
    for (auto& e : ring.done) CR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    unsigned char* const base = static_cast<unsigned char*>(block);
    const unsigned char* const from = static_cast<const unsigned char*>(src);
    for (size_t off = 0, i = 0; off < bytes; off += kChunk, ++i) {
        const size_t len = std::min(kChunk, bytes - off);
        const int k = static_cast<int>(i % kRing);
        unsigned char* const buf = base + k * kChunk;
        if (i >= kRing) CR_CUDA(cudaEventSynchronize(ring.done[k]));  // the slot's last transfer is done
        crh::parallel_for(len, [&](uint64_t b, uint64_t e) { std::memcpy(buf + b, from + off + b, e - b); }, size_t{4} << 20);
        CR_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, buf, len, cudaMemcpyHostToDevice, s));
        CR_CUDA(cudaEventRecord(ring.done[k], s));
    }
    CR_CUDA(cudaStreamSynchronize(s));
}

// Parts of a scene upload that run on host threads beside the caller's: task k runs on its
// own thread with the scene's device current and copies on stream(k); join(k) waits for the
// task and its copies and rethrows its exception. The destructor joins whatever is left.
class SideWork {
  public:
    static constexpr int kTasks = 2;
    explicit SideWork(int device) : device_(device) {
        for (int k = 0; k < kTasks; ++k) {
            const cudaError_t e = cudaStreamCreateWithFlags(&streams_[k], cudaStreamNonBlocking);
            if (e != cudaSuccess) {
                cudaGetLastError();
                for (int j = 0; j < k; ++j) cudaStreamDestroy(streams_[j]);
                throw CudaError(e, "cudaStreamCreateWithFlags");
            }
        }
    }
    SideWork(const SideWork&) = delete;
    SideWork& operator=(const SideWork&) = delete;
    cudaStream_t stream(int k) const { return streams_[k]; }
    void run(int k, std::function<void()> fn) {
        threads_[k] = std::thread([this, k, fn = std::move(fn)] {
            try {
                CR_CUDA(cudaSetDevice(device_));
                fn();
                CR_CUDA(cudaStreamSynchronize(streams_[k]));
            } catch (...) {
                errors_[k] = std::current_exception();
            }
        });
    }
    void join(int k) {
        if (threads_[k].joinable()) threads_[k].join();
        if (errors_[k]) std::rethrow_exception(errors_[k]);
    }
    ~SideWork() {
        for (auto& t : threads_) if (t.joinable()) t.join();
        for (auto st : streams_) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
    }

  private:
    int device_;
    cudaStream_t streams_[kTasks] = {};
    std::thread threads_[kTasks];
    std::exception_ptr errors_[kTasks];
};

// Build the device scene: geometry in leaf order, node pairs, materials, lights, environment.
void uploadScene(cr_gpu_scene& g, const cr_scene_desc& d, const cr_environment_desc& env) {
    const uint64_t n = d.triangle_count;
    if (n && !d.triangles) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "triangles is NULL");
    if (d.material_count && !d.materials) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "materials is NULL");
    {
        std::atomic<bool> bad{false};
        crh::parallel_for(n, [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i)
                if (d.triangles[i].material >= d.material_count) bad = true;
        });
        if (bad) throw crh::Error(CR_ERR_OUT_OF_RANGE, "Triangle material index out of range");
    }
    for (uint32_t m = 0; m < d.material_count; ++m) {
        const cr_material& mat = d.materials[m];
        const cr_texture_slot* s[5] = {&mat.base_color_texture, &mat.metallic_roughness_texture, &mat.normal_texture,
                                       &mat.emissive_texture, &mat.transmission_texture};
        for (auto* slot : s) {
            if (slot->texture == -1) continue;
            if (slot->texture < 0 || static_cast<uint32_t>(slot->texture) >= d.texture_count)
                throw crh::Error(CR_ERR_OUT_OF_RANGE, "Texture slot index out of range");
            if (slot->texcoord < 0 || slot->texcoord > 1) throw crh::Error(CR_ERR_OUT_OF_RANGE, "Only TEXCOORD_0 and TEXCOORD_1 are supported");
            const cr_texture& t = d.textures[slot->texture];
            if (t.image < 0 || static_cast<uint32_t>(t.image) >= d.image_count) throw crh::Error(CR_ERR_OUT_OF_RANGE, "Texture image index out of range");
            const cr_image& im = d.images[t.image];
            if (im.width <= 0 || im.height <= 0 || !im.pixels) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "Texture image dimensions do not match its pixels");
        }
    }
    // The triangle records go to the device unchanged: that copy (the largest, from the caller's
    // memory) starts on a helper thread, and the environment tables are built and copied on
    // another, while this thread prepares the geometry. Errors keep their order: the helpers
    // are joined where their step stood in the sequential upload.
    cudaStream_t s = g.stream;
    DevScene& S = g.dev;
    S = DevScene{};
    crh::EnvTables& E = g.env;
    DevAlloc envMem;  // the environment thread's blocks, handed to the scene when it is done
    struct AdoptBlocks {
        DevAlloc& from;
        DevAlloc& to;
        ~AdoptBlocks() {
            to.blocks.insert(to.blocks.end(), from.blocks.begin(), from.blocks.end());
            to.bytes += from.bytes;
            from.blocks.clear();
            from.bytes = 0;
        }
    } adopt{envMem, g.geometry};
    SideWork side(g.device);
    S.tris = g.geometry.alloc<cr_triangle>(n);
    side.run(0, [&, dst = const_cast<cr_triangle*>(S.tris)] {
        if (n) stagedUpload(dst, d.triangles, n * sizeof(cr_triangle), side.stream(0));
    });
    side.run(1, [&] {
        crh::build_environment(env, E);
        if (E.hasImage) {
            const cudaStream_t es = side.stream(1);
            const size_t px = static_cast<size_t>(E.width) * E.height;
            float4* pixels = envMem.alloc<float4>(px);
            stagedUpload(pixels, env.pixels, px * sizeof(float4), es);
            S.env_pixels = pixels;
            double* cdf = envMem.alloc<double>(E.cdf.size());
            stagedUpload(cdf, E.cdf.data(), E.cdf.size() * sizeof(double), es);
            S.env_cdf = cdf;
            float* pdf = envMem.alloc<float>(E.pdf.size());
            stagedUpload(pdf, E.pdf.data(), E.pdf.size() * sizeof(float), es);
            S.env_pdf = pdf;
            S.env_row_cos = envMem.upload(E.rowCos.data(), E.rowCos.size(), es);
            S.env_coarse = envMem.upload(E.coarse.data(), E.coarse.size(), es);
        }
    });
    // BVH: the caller's (the reference's own node array, read in place) or ours.
    std::vector<cr_bvh_node> ownNodes;
    std::vector<uint32_t> ownIndices;
    if (d.bvh_index_count && !d.bvh_indices) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "bvh_indices is NULL");
    const bool callerBvh = d.bvh_nodes && d.bvh_node_count;
    if (!callerBvh) crh::build_bvh(d.triangles, n, ownNodes, ownIndices);
    const ArrayView<cr_bvh_node> nodes = callerBvh ? ArrayView<cr_bvh_node>{d.bvh_nodes, d.bvh_node_count}
                                                   : ArrayView<cr_bvh_node>{ownNodes.data(), ownNodes.size()};
    const ArrayView<uint32_t> indices = callerBvh ? ArrayView<uint32_t>{d.bvh_indices, d.bvh_index_count}
                                                  : ArrayView<uint32_t>{ownIndices.data(), ownIndices.size()};
    // Structure checks: adjacent children at odd indices, leaf ranges inside indices.
    {
        std::atomic<int> bad{0};
        crh::parallel_for(nodes.size(), [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i) {
                const cr_bvh_node& nd = nodes[i];
                if (nd.count) {
                    if (static_cast<uint64_t>(nd.first) + nd.count > indices.size()) bad = 1;
                } else if ((nd.first & 1u) == 0 || static_cast<uint64_t>(nd.first) + 1 >= nodes.size() || nd.first <= i) {
                    bad = 2;
                }
            }
        });
        if (bad == 1) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "BVH leaf range outside its index array");
        if (bad == 2) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "BVH interior node does not reference an adjacent child pair");
        crh::parallel_for(indices.size(), [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i) if (indices[i] >= n) bad = 3;
        });
        if (bad == 3) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "BVH index outside the triangle array");
    }

    S.triangle_count = n;
    g.triangleCount = n;
    // The arrays built here go into one staging block and are copied as soon as each is done.
    const size_t ngCount = n ? n : 1;
    const size_t posCount = 3 * (indices.empty() ? 1 : indices.size());
    const size_t pairCount = nodes.size() > 1 ? (nodes.size() - 1) / 2 : 0;
    const size_t pairSlots = pairCount ? pairCount : 1;
    Staging stage(s, Staging::bytesFor(ngCount * sizeof(float4)) + Staging::bytesFor(posCount * sizeof(float4)) +
                         Staging::bytesFor(pairSlots * sizeof(NodePair)));
    float4* ng = stage.carve<float4>(ngCount);
    float4* pos = stage.carve<float4>(posCount);
    NodePair* pairs = stage.carve<NodePair>(pairSlots);
    // per-triangle flags and geometric normals (Scene::accepts, geometry.cpp:282-290)
    std::unique_ptr<uint32_t[]> flags(new uint32_t[ngCount]);
    flags[0] = 0;
    ng[0] = make_float4(0, 0, 0, 0);
    std::atomic<uint32_t> anyMaskA{0};
    std::atomic<bool> texturedEmitterA{false};
    crh::parallel_for(n, [&](uint64_t b, uint64_t e) {
        uint32_t localMask = 0;
        bool localEmitter = false;
        for (uint64_t i = b; i < e; ++i) {
            const cr_triangle& t = d.triangles[i];
            const cr_material& m = d.materials[t.material];
            uint32_t f = 0;
            if (!m.double_sided && m.transmission <= 0) f |= kTriCull;
            if (m.alpha_mode == CR_ALPHA_MASK) { f |= kTriAlphaMask; localMask = 1; }
            // bsdf.cpp:171-179: smooth, and the diffuse weight (1-metallic)(1-transmission) is zero
            if (m.roughness <= 0.001f && m.metallic_roughness_texture.texture < 0 &&
                (m.metallic == 1.0f || (m.transmission == 1.0f && m.transmission_texture.texture < 0)))
                f |= kTriNeeNull;
            else if (m.metallic == 1.0f && m.transmission == 0.0f && m.metallic_roughness_texture.texture < 0 &&
                     m.transmission_texture.texture < 0)
                f |= kTriConductor;  // a rough GGX conductor: its BSDF has no diffuse or transmission lobe
            const bool textured = m.base_color_texture.texture >= 0 || m.metallic_roughness_texture.texture >= 0 ||
                                  m.normal_texture.texture >= 0 || m.emissive_texture.texture >= 0 ||
                                  m.transmission_texture.texture >= 0;
            if (textured && (m.emission[0] > 0 || m.emission[1] > 0 || m.emission[2] > 0)) localEmitter = true;
            flags[i] = f;
            float gx = t.geometric_normal[0], gy = t.geometric_normal[1], gz = t.geometric_normal[2];
            if (gx == 0 && gy == 0 && gz == 0) {  // geometry.cpp:284
                const double ax = static_cast<double>(t.v[1].position[0]) - t.v[0].position[0];
                const double ay = static_cast<double>(t.v[1].position[1]) - t.v[0].position[1];
                const double az = static_cast<double>(t.v[1].position[2]) - t.v[0].position[2];
                const double bx = static_cast<double>(t.v[2].position[0]) - t.v[0].position[0];
                const double by = static_cast<double>(t.v[2].position[1]) - t.v[0].position[1];
                const double bz = static_cast<double>(t.v[2].position[2]) - t.v[0].position[2];
                const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
                const double sq = cx * cx + cy * cy + cz * cz;
                if (sq > 0 && std::isfinite(sq)) {
                    const double inv = 1 / std::sqrt(sq);
                    gx = static_cast<float>(cx * inv); gy = static_cast<float>(cy * inv); gz = static_cast<float>(cz * inv);
                }
            }
            float fw;
            std::memcpy(&fw, &f, 4);
            ng[i] = make_float4(gx, gy, gz, fw);
        }
        if (localMask) anyMaskA = 1;
        if (localEmitter) texturedEmitterA = true;
    });
    const uint32_t anyMask = anyMaskA;
    const bool texturedEmitter = texturedEmitterA;
    float4* devNg = g.geometry.alloc<float4>(ngCount);
    CR_CUDA(cudaMemcpyAsync(devNg, ng, ngCount * sizeof(float4), cudaMemcpyHostToDevice, s));
    S.tri_ng = devNg;
    for (int k = 0; k < 3; ++k) pos[k] = make_float4(0, 0, 0, 0);
    crh::parallel_for(indices.size(), [&](uint64_t b, uint64_t e) {
        for (uint64_t slot = b; slot < e; ++slot) {
            const uint32_t idx = indices[slot];
            const cr_triangle& t = d.triangles[idx];
            float w0, w1;
            std::memcpy(&w0, &idx, 4);
            std::memcpy(&w1, &flags[idx], 4);
            pos[3 * slot] = make_float4(t.v[0].position[0], t.v[0].position[1], t.v[0].position[2], w0);
            pos[3 * slot + 1] = make_float4(t.v[1].position[0], t.v[1].position[1], t.v[1].position[2], w1);
            pos[3 * slot + 2] = make_float4(t.v[2].position[0], t.v[2].position[1], t.v[2].position[2], 0.0f);
        }
    });
    float4* devPos = g.geometry.alloc<float4>(posCount);
    CR_CUDA(cudaMemcpyAsync(devPos, pos, posCount * sizeof(float4), cudaMemcpyHostToDevice, s));
    S.tri_pos = devPos;
    pairs[0] = NodePair{};
    auto childRef = [&](const cr_bvh_node& c, uint32_t& ref, uint32_t& cnt) {
        if (c.count) { ref = c.first; cnt = c.count; } else { ref = (c.first - 1) / 2; cnt = 0; }
    };
    crh::parallel_for(pairCount, [&](uint64_t b, uint64_t e) {
        for (uint64_t p = b; p < e; ++p) {
            const cr_bvh_node& c0 = nodes[2 * p + 1];
            const cr_bvh_node& c1 = nodes[2 * p + 2];
            NodePair& np = pairs[p];
            np.a = make_float4(c0.lo[0], c0.lo[1], c0.lo[2], c0.hi[0]);
            np.b = make_float4(c0.hi[1], c0.hi[2], c1.lo[0], c1.lo[1]);
            np.c = make_float4(c1.lo[2], c1.hi[0], c1.hi[1], c1.hi[2]);
            childRef(c0, np.d.x, np.d.y);
            childRef(c1, np.d.z, np.d.w);
        }
    });
    if (!nodes.empty()) {
        S.has_root = 1;
        for (int k = 0; k < 3; ++k) { S.root_lo[k] = nodes[0].lo[k]; S.root_hi[k] = nodes[0].hi[k]; }
        childRef(nodes[0], S.root_ref, S.root_count);
    }
    NodePair* devPairs = g.geometry.alloc<NodePair>(pairSlots);
    CR_CUDA(cudaMemcpyAsync(devPairs, pairs, pairSlots * sizeof(NodePair), cudaMemcpyHostToDevice, s));
    S.pairs = devPairs;
    // the triangle half of the light table, while the helpers finish
    const crh::LightScan lightScan = crh::scan_lights(d.triangles, n, d.materials);
    side.join(0);  // the triangle records
    S.any_alpha_mask = anyMask;
    // A textured emitter's light sample evaluates textures, which can fail; keep it then.
    S.nee_skip = texturedEmitter ? 0u : 1u;
    // materials and textures
    S.materials = g.geometry.upload(d.materials, d.material_count, s);
    S.material_count = d.material_count;
    std::vector<double2> trig(5 * (d.material_count ? d.material_count : 1));
    for (uint32_t m = 0; m < d.material_count; ++m) {
        const cr_material& mat = d.materials[m];
        const cr_texture_slot* sl[5] = {&mat.base_color_texture, &mat.metallic_roughness_texture, &mat.normal_texture,
                                        &mat.emissive_texture, &mat.transmission_texture};
        for (int k = 0; k < 5; ++k) {
            const double r = static_cast<double>(sl[k]->rotation);
            trig[5 * m + k] = make_double2(std::cos(r), std::sin(r));
        }
    }
    S.slot_trig = g.geometry.upload(trig.data(), trig.size(), s);
    std::vector<DevImage> images(d.image_count ? d.image_count : 1);
    for (uint32_t i = 0; i < d.image_count; ++i) {
        images[i].width = d.images[i].width; images[i].height = d.images[i].height;
        const size_t px = static_cast<size_t>(d.images[i].width) * d.images[i].height;
        images[i].pixels = g.geometry.upload(reinterpret_cast<const float4*>(d.images[i].pixels), px, s);
    }
    S.images = g.geometry.upload(images.data(), images.size(), s);
    S.image_count = d.image_count;
    S.textures = g.geometry.upload(d.textures, d.texture_count, s);
    S.texture_count = d.texture_count;
    // environment (tables and copies from the helper thread)
    side.join(1);
    S.env_has_image = E.hasImage;
    for (int k = 0; k < 3; ++k) S.env_constant[k] = E.constant[k];
    if (E.hasImage) {
        S.env_width = E.width; S.env_height = E.height;
        S.env_coarse_count = static_cast<uint32_t>(E.coarse.size());
        S.alias_threshold = nullptr;  // built on the first render that asks for alias sampling
        S.alias_index = nullptr;
    }
    S.env_weight_sum = E.weightSum;
    S.env_rotation = E.rotation;
    S.env_intensity = E.intensity;
    // lights
    crh::LightTables L;
    crh::build_lights(lightScan, d.lights, d.light_count, E.integral, L);
    S.light_entries = g.geometry.upload(L.entries.data(), L.entries.size(), s);
    S.light_entry_count = static_cast<uint32_t>(L.entries.size());
    S.tri_light_probability = g.geometry.upload(L.triangleProbability.data(), L.triangleProbability.size(), s);
    S.env_probability = L.environmentProbability;
    std::vector<DevPunctual> punctual(d.light_count ? d.light_count : 1);
    for (uint32_t i = 0; i < d.light_count; ++i) {
        const cr_punctual_light& l = d.lights[i];
        DevPunctual& p = punctual[i];
        p.type = l.type;
        for (int k = 0; k < 3; ++k) { p.position[k] = l.position[k]; p.direction[k] = l.direction[k]; p.color[k] = l.color[k]; }
        p.intensity = l.intensity; p.range = l.range;
        p.cos_outer = std::cos(l.outer_cone);  // render.cpp:203 (float std::cos)
        p.cos_inner = std::cos(l.inner_cone);
    }
    S.punctual = g.geometry.upload(punctual.data(), punctual.size(), s);
    S.punctual_count = d.light_count;
    CR_CUDA(cudaStreamSynchronize(s));
}



// Progressive output: after every `every` samples per pixel, the film so far, encoded.
struct Frames {
    uint32_t every = 0;  // 0: no frames
    int format = CR_ENCODE_SRGB8;
    float exposure = 0;
    cr_frame_fn fn = nullptr;
    void* user = nullptr;
};

// A guided render: the network, its online training during the first trainSamples samples per
// pixel, and the mixture's share of the sampled directions.
struct GuideRun {
    cr_guide* gd = nullptr;
    uint32_t trainSamples = 32;
    float probability = 0.5f;
    uint32_t batch = 16384;
    uint32_t epochs = 4;
};

// The alias-table sampler's tables, built and uploaded on the first request (scene with an
// environment image only).
void ensureAlias(cr_gpu_scene& g) {
    if (!g.dev.env_has_image || g.dev.alias_threshold) return;
    crh::build_alias(g.env);
    // The scene takes the tables only once all three exist: a failed upload leaves it without
    // them (and the next request builds them again), never with some of them.
    const auto* threshold = reinterpret_cast<const unsigned long long*>(
        g.aliasAlloc.upload(g.env.aliasThreshold.data(), g.env.aliasThreshold.size(), g.stream));
    const auto* index = g.aliasAlloc.upload(g.env.aliasIndex.data(), g.env.aliasIndex.size(), g.stream);
    const float* pdf = g.aliasAlloc.upload(g.env.aliasPdf.data(), g.env.aliasPdf.size(), g.stream);
    g.dev.alias_index = index;
    g.aliasPdf = pdf;
    g.dev.alias_threshold = threshold;
}

// The whole render. filmHost may be NULL (film stays on the device).
void renderImpl(cr_gpu_scene& g, const cr_camera& camera, const cr_render_options& o, cr_progress_fn progress,
                void* user, float* filmHost, cr_render_stats* stats, const cr_gpu_tuning& tuning, float* perSample,
                const Frames& frames = Frames{}, const GuideRun* guide = nullptr, const TraceDump* dump = nullptr) {
    const auto start = std::chrono::steady_clock::now();
    crh::validate_options(o);
    const uint64_t pixels = static_cast<uint64_t>(o.width) * o.height;
    const uint64_t total = pixels * static_cast<uint64_t>(o.samples);
    RenderParams P;
    try {
        P = makeParams(camera, o, tuning);
    } catch (const crh::Error& e) {
        // The reference throws these from Camera::generate inside the first sample.
        throw crh::Error(CR_ERR_RENDER, std::string("Pixel (0,0), sample 0: ") + e.what());
    }
    CR_CUDA(cudaSetDevice(g.device));
    // Pool of path slots and chunk of sample ids held in device memory at once. By default a
    // chunk is one pool's worth of samples: every path slot starts a camera sample at the
    // chunk's first iteration and the chunk drains without refilling freed slots. On the
    // 1M-triangle 1080p workload that measured faster than refilling (regeneration) at every
    // pool/chunk ratio tried (212 vs 200 Msamples/s at its best, 2x pool), and a larger pool
    // amortises the drain tail over more samples (132.7 M samples at 1080p x 64 spp: 2^24 slots
    // 526 ms, 2^25 508 ms, 2^26 499 ms, 2^27 494 ms). With pixel-major chunks 2^27 slots take
    // all 64 samples of a 1080p frame in one chunk, one drain instead of two: 316.7 -> 320.8
    // Msamples/s, for ~33 GB of path state (248 bytes per slot) on a 180 GB device.
    uint64_t pool = tuning.paths_per_wave > 0 ? static_cast<uint64_t>(tuning.paths_per_wave)
                                              : (uint64_t{1} << (guide ? 23 : 27));
    pool = std::max<uint64_t>(1024, std::min<uint64_t>(pool, total));
    const uint64_t chunkBudget = uint64_t{1} << 28;  // 268 M samples = 4 GiB of float4 radiance
    if (tuning.chunk_log2 && (tuning.chunk_log2 < 16 || tuning.chunk_log2 > 28))
        throw crh::Error(CR_ERR_INVALID_ARGUMENT, "chunk_log2 must be 0 or in [16, 28]");
    uint64_t chunk = tuning.chunk_log2 ? std::max<uint64_t>(pool, uint64_t{1} << tuning.chunk_log2) : pool;
    chunk = std::min<uint64_t>(total, std::min<uint64_t>(chunk, chunkBudget));
    std::vector<unsigned char> frameBuf;
    if (frames.every) {
        // a chunk ends exactly where samples [0, every) of every pixel are done
        if (static_cast<uint64_t>(frames.every) * pixels > chunkBudget)
            throw crh::Error(CR_ERR_INVALID_ARGUMENT, "progressive frames need every_samples*width*height <= 268435456");
        if (frames.format != CR_ENCODE_SRGB8 && frames.format != CR_ENCODE_RGBE && frames.format != CR_ENCODE_HDR_FILE)
            throw crh::Error(CR_ERR_INVALID_ARGUMENT, "unknown encode format");
        crh::check_image_dims(o.width, o.height, frames.format == CR_ENCODE_SRGB8 ? "PNG output" : "HDR output");
        if (frames.format == CR_ENCODE_SRGB8) { float t[256]; crh::display_thresholds(frames.exposure, t); }
        chunk = std::min<uint64_t>(total, static_cast<uint64_t>(frames.every) * pixels);
        frameBuf.resize(frames.format == CR_ENCODE_SRGB8 ? 3 * pixels
                        : frames.format == CR_ENCODE_RGBE ? 4 * pixels
                        : crh::hdr_header(o.width, o.height).size() + static_cast<uint64_t>(o.height) * (4 + 8ull * o.width + 8));
    }
    // Chunks of whole samples per pixel (where one fits the pool) issue their ids pixel-major
    // (see Chunk): the default chunk is the most whole samples of every pixel the pool holds.
    if (!tuning.chunk_log2 && !frames.every && !guide && chunk >= pixels) chunk = chunk / pixels * pixels;
    // a pool never needs more slots than one chunk has samples
    pool = std::min<uint64_t>(pool, chunk);
    pool = (pool + 127) / 128 * 128;
    Workspace& W = workspaceFor(g.device);
    std::lock_guard<std::mutex> wsLock(W.mutex);
    W.ensureWork(static_cast<size_t>(pool));
    W.ensureSideStreams();
    W.ensureOut(static_cast<size_t>(chunk));
    g.ensureFilm(pixels);
    if (perSample) W.ensurePacked(static_cast<size_t>(chunk));
    // Guided renders: per-path network outputs and hit distances for the pool, records and the
    // training-sample store for the training chunks (one sample per pixel each).
    DevAlloc guideMem;
    struct ReleaseAtEnd {
        DevAlloc& m;
        cudaStream_t s;
        ~ReleaseAtEnd() { cudaStreamSynchronize(s); m.release(); }
    } releaseGuide{guideMem, g.stream};
    PathSoA st = W.st;  // after the workspace buffers above exist
    if (dump) st.dump = *dump;  // recorded by the counting traversal kernels
    const uint64_t trainTotal = guide ? std::min<uint64_t>(total, static_cast<uint64_t>(guide->trainSamples) * pixels) : 0;
    float* guideOut = nullptr;
    GuideSample* guideSamples = nullptr;
    uint64_t guideCapacity = 0;
    if (guide) {
        guideOut = guideMem.alloc<float>(pool * kGuideOut);
        st.guide.mixture = guideOut;
        st.guide.hitT = guideMem.alloc<float>(pool);
        const uint64_t trainPool = std::min<uint64_t>(pool, pixels);
        st.guide.records = guideMem.alloc<GuideRecord>(trainPool * kGuideRecords);
        st.guide.count = guideMem.alloc<uint32_t>(trainPool);
        guideCapacity = std::min<uint64_t>(uint64_t{1} << 22, pixels * kGuideRecords);
        guideSamples = guideMem.alloc<GuideSample>(guideCapacity);
        st.guide.samples = guideSamples;
        st.guide.sampleCount = guideMem.alloc<unsigned long long>(1);
        st.guide.sampleCapacity = guideCapacity;
        for (int k = 0; k < 3; ++k) {
            const float lo = g.dev.root_lo[k], ext = g.dev.root_hi[k] - lo;
            st.guide.lo[k] = lo;
            st.guide.inv[k] = ext > 0 ? 1.0f / ext : 0.0f;
        }
        st.guide.guideProbability = guide->probability;
        st.guide.record = 1;
        CR_CUDA(cudaMemsetAsync(st.guide.sampleCount, 0, sizeof(unsigned long long), g.stream));
    }
    if (!W.hostCounts) { crh::count_allocation(); CR_CUDA(cudaMallocHost(&W.hostCounts, kCountWords * sizeof(uint32_t))); }
    if (!W.hostStats) { crh::count_allocation(); CR_CUDA(cudaMallocHost(&W.hostStats, kStatWords * sizeof(unsigned long long))); }
    cudaStream_t s = g.stream;
    if (!W.gridTrace) {
        W.gridTrace = occupancyGrid(reinterpret_cast<const void*>(k_trace<false>), 128, g.device);
        W.gridShade = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeGeneric>), 128, g.device);
        W.gridShadeLight = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeNeeNull>), 128, g.device);
        W.gridShadeMiss = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeMiss>), 128, g.device);
        W.gridTraceNoAlpha = occupancyGrid(reinterpret_cast<const void*>(k_trace<false, false, true>), 128, g.device);
        W.gridShadeLean = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeGeneric, false, false, true>), 128, g.device);
        W.gridShadeLightLean = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeNeeNull, false, false, true>), 128, g.device);
        W.gridShadeMissLean = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeMiss, false, false, true>), 128, g.device);
        W.gridShadeCond = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeConductor>), 128, g.device);
        W.gridShadeCondLean = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeConductor, false, false, true>), 128, g.device);
        W.gridRegen = occupancyGrid(reinterpret_cast<const void*>(k_regen<false>), 128, g.device);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
        W.gridSmall = sms * 8;
    }
    if (tuning.env_alias) ensureAlias(g);
    // The scene as this render's kernels see it: alias sampling reads the alias sampler's own
    // texel densities (for light samples and MIS weights alike); the diagnostic switch
    // generic_shading sends every hit through the generic shading kernel.
    DevScene dev = g.dev;
    if (tuning.env_alias && g.dev.env_has_image) dev.env_pdf = g.aliasPdf;
    if (tuning.generic_shading) dev.nee_skip = 0;
    // rough conductors take their own kernel (guided renders shade them in the guided generic one)
    dev.conductor_class = !guide && !tuning.generic_shading ? 1u : 0u;
    CR_CUDA(cudaMemsetAsync(g.acc, 0, 3 * pixels * sizeof(double), s));
    CR_CUDA(cudaMemsetAsync(W.stats, 0, kStatWords * sizeof(unsigned long long), s));
    const unsigned long long noError = ~0ull;
    CR_CUDA(cudaMemcpyAsync(W.stats + kStatErrorKey, &noError, sizeof(noError), cudaMemcpyHostToDevice, s));
    const ErrSink E{W.stats + kStatErrorKey, nullptr};

    const bool timePhases = tuning.time_phases != 0;
    double traceMs = 0, shadeMs = 0, regenMs = 0;
    uint64_t launches = 0;
    int iterations = 0, chunks = 0;
    cudaEvent_t t0 = W.event(0), t1 = W.event(1);
    CR_CUDA(cudaEventRecord(t0, s));
    auto lastProgress = start;
    bool errored = false;
    const int batch = 8;
    uint64_t step = chunk;
    for (uint64_t c0 = 0; c0 < total && !errored; c0 += step) {
        // guided renders train between one-sample-per-pixel chunks, then render in full chunks
        const bool training = guide && c0 < trainTotal;
        step = training ? std::min<uint64_t>(pixels, trainTotal - c0) : chunk;
        if (guide && !training && st.guide.count) {  // training is over: stop recording
            st.guide.count = nullptr;
            st.guide.records = nullptr;
            st.guide.record = 0;
        }
        Chunk C{c0, std::min<uint64_t>(total, c0 + step), pixels};
        if (c0 % pixels == 0 && (C.c1 - c0) % pixels == 0) {  // whole samples: pixel-major
            C.spp = static_cast<uint32_t>((C.c1 - c0) / pixels);
            C.s0 = static_cast<uint32_t>(c0 / pixels);
        }
        ++chunks;
        // the chunk's ids are issued from c0
        CR_CUDA(cudaMemsetAsync(W.counts, 0, kCountWords * sizeof(uint32_t), s));
        const unsigned long long issuedStart = c0;
        CR_CUDA(cudaMemcpyAsync(W.stats + kStatIssued, &issuedStart, sizeof(issuedStart), cudaMemcpyHostToDevice, s));
        // a training chunk uses only as many slots as it has samples: its paths' records cover them
        const uint64_t chunkPool = training ? std::min<uint64_t>(pool, step) : pool;
        k_pool_init<<<W.gridSmall, 128, 0, s>>>(W.q, static_cast<uint32_t>(chunkPool));
        ++launches;
        const uint64_t maxIterations = ((C.c1 - C.c0) / chunkPool + 3) * 2 * static_cast<uint64_t>(o.bounces + 2) + 16;
        // scenes without textures, punctual lights or alpha masks take the lean shading kernels
        const bool lean = g.dev.texture_count == 0 && g.dev.punctual_count == 0 && !g.dev.any_alpha_mask;
        // no launch needs more blocks than the chunk's pool has 128-path batches (warps take
        // their batches from a counter, so a smaller grid only spares the launch its idle blocks)
        const int poolBlocks = static_cast<int>(std::min<uint64_t>((chunkPool + 127) / 128, 1u << 30));
        auto cap = [&](int grid) { return std::max(1, std::min(grid, poolBlocks)); };
        const bool noAlpha = !g.dev.any_alpha_mask;
        uint64_t iter = 0;
        int cur = 0;
        std::vector<std::pair<size_t, int>> timed;
        size_t ev = 2;
        for (;;) {
            timed.clear();
            ev = 2;
            for (int b = 0; b < batch; ++b) {
                auto rec = [&](int phase, auto&& launch) {
                    if (timePhases) CR_CUDA(cudaEventRecord(W.event(ev), s));
                    launch();
                    if (timePhases) { CR_CUDA(cudaEventRecord(W.event(ev + 1), s)); timed.push_back({ev, phase}); ev += 2; }
                    ++launches;
                };
                rec(2, [&] { k_regen<false><<<cap(W.gridRegen), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}, 1); });
                rec(0, [&] {
                    if (tuning.count_traversal) k_trace<true><<<cap(W.gridTrace), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                    else if (noAlpha) k_trace<false, false, true><<<cap(W.gridTraceNoAlpha), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                    else k_trace<false><<<cap(W.gridTrace), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                });
                // shading: the lean instantiations when the scene allows them. The classes'
                // queues are independent, so without phase timing or guiding the miss and
                // NEE-null launches run on two more streams beside the generic one, and each
                // fills the device while the others drain.
                if (!timePhases && !guide) {
                    CR_CUDA(cudaEventRecord(W.fork, s));
                    for (int k = 0; k < Workspace::kSide; ++k) CR_CUDA(cudaStreamWaitEvent(W.side[k], W.fork, 0));
                    if (lean) {
                        k_shade<kShadeMiss, false, false, true><<<cap(W.gridShadeMissLean), 128, 0, W.side[0]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeNeeNull, false, false, true><<<cap(W.gridShadeLightLean), 128, 0, W.side[1]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeConductor, false, false, true><<<cap(W.gridShadeCondLean), 128, 0, W.side[2]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeGeneric, false, false, true><<<cap(W.gridShadeLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                    } else {
                        k_shade<kShadeMiss><<<cap(W.gridShadeMiss), 128, 0, W.side[0]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeNeeNull><<<cap(W.gridShadeLight), 128, 0, W.side[1]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeConductor><<<cap(W.gridShadeCond), 128, 0, W.side[2]>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                        k_shade<kShadeGeneric><<<cap(W.gridShade), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{});
                    }
                    for (int k = 0; k < Workspace::kSide; ++k) {
                        CR_CUDA(cudaEventRecord(W.join[k], W.side[k]));
                        CR_CUDA(cudaStreamWaitEvent(s, W.join[k], 0));
                    }
                    launches += 4;
                } else {
                if (lean) {
                    rec(1, [&] { k_shade<kShadeMiss, false, false, true><<<cap(W.gridShadeMissLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                    rec(1, [&] { k_shade<kShadeNeeNull, false, false, true><<<cap(W.gridShadeLightLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                    if (dev.conductor_class)
                        rec(1, [&] { k_shade<kShadeConductor, false, false, true><<<cap(W.gridShadeCondLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                } else {
                    rec(1, [&] { k_shade<kShadeMiss><<<cap(W.gridShadeMiss), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                    rec(1, [&] { k_shade<kShadeNeeNull><<<cap(W.gridShadeLight), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                    if (dev.conductor_class)
                        rec(1, [&] { k_shade<kShadeConductor><<<cap(W.gridShadeCond), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                }
                if (guide) {
                    rec(1, [&] {
                        guideInferPaths(guide->gd, s, W.q.shade[kShadeGeneric], W.q.counts + kCountShade0 + kShadeGeneric,
                                        static_cast<uint32_t>(pool), st, st.guide.hitT, dev,
                                        V3{st.guide.lo[0], st.guide.lo[1], st.guide.lo[2]},
                                        V3{st.guide.inv[0], st.guide.inv[1], st.guide.inv[2]}, guideOut);
                    });
                    if (lean) rec(1, [&] { k_shade<kShadeGeneric, false, true, true><<<cap(W.gridShadeLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                    else rec(1, [&] { k_shade<kShadeGeneric, false, true><<<cap(W.gridShade), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                } else if (lean) {
                    rec(1, [&] { k_shade<kShadeGeneric, false, false, true><<<cap(W.gridShadeLean), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                } else {
                    rec(1, [&] { k_shade<kShadeGeneric><<<cap(W.gridShade), 128, 0, s>>>(dev, P, st, W.q, cur, C, E, W.stats, JobTable{}); });
                }
                }
                cur ^= 1;
                ++iter;
                ++iterations;
            }
            CR_CUDA(cudaMemcpyAsync(W.hostCounts, W.counts, kCountWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaMemcpyAsync(W.hostStats, W.stats, kStatWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaStreamSynchronize(s));
            CR_CUDA(cudaGetLastError());
            for (auto& te : timed) {
                float ms = 0;
                CR_CUDA(cudaEventElapsedTime(&ms, W.event(te.first), W.event(te.first + 1)));
                (te.second == 0 ? traceMs : te.second == 1 ? shadeMs : regenMs) += ms;
            }
            // after the last shade: live = next live queue + queued shadow rays
            const uint64_t live = W.hostCounts[kCountExtend0 + cur] + W.hostCounts[kCountShadow0 + (cur ^ 1)];
            const bool issuedAll = W.hostStats[kStatIssued] >= C.c1;
            if (W.hostStats[kStatErrorKey] != ~0ull) { errored = true; break; }
            if (issuedAll && live == 0) break;
            if (iter > maxIterations) throw crh::Error(CR_ERR_DEVICE_TIMEOUT, "paths still live after the iteration bound");
            if (progress) {
                const auto now = std::chrono::steady_clock::now();
                if (now - lastProgress >= std::chrono::seconds(2)) {
                    lastProgress = now;
                    const uint64_t issued = std::min<uint64_t>(W.hostStats[kStatIssued], C.c1);
                    const uint64_t done = issued > live ? issued - live : 0;
                    progress(done, total, std::chrono::duration<double>(now - start).count(), user);
                }
            }
        }
        if (errored) break;
        k_accumulate<<<W.gridSmall, 128, 0, s>>>(st.out, C, g.acc);
        ++launches;
        if (training) {  // Adam over this chunk's samples; the next chunk uses the new weights
            unsigned long long collected = 0;
            CR_CUDA(cudaMemcpyAsync(&collected, st.guide.sampleCount, sizeof(collected), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaStreamSynchronize(s));
            const uint64_t n = std::min<uint64_t>(collected, guideCapacity);
            if (n) {
                const uint32_t steps = static_cast<uint32_t>(guide->epochs * ((n + guide->batch - 1) / guide->batch));
                guideTrain(guide->gd, s, guideSamples, n, steps, guide->batch, 1e-3f, -1.0);
                launches += 2ull * steps + 1;
            }
            CR_CUDA(cudaMemsetAsync(st.guide.sampleCount, 0, sizeof(unsigned long long), s));
        }
        if (frames.every) {
            const uint32_t done = static_cast<uint32_t>(C.c1 / pixels);
            k_film<<<W.gridSmall, 128, 0, s>>>(g.acc, g.film, pixels, done);
            ++launches;
            const uint64_t size = crg::encode_film(g.film, o.width, o.height, frames.format, frames.exposure, s,
                                                   frameBuf.data(), frameBuf.size());
            if (size > frameBuf.size()) throw crh::Error(CR_ERR_CUDA, "progressive frame larger than its bound");
            if (frames.fn) frames.fn(done, frameBuf.data(), size, frames.user);
        }
        if (perSample) {
            const uint64_t n = C.c1 - C.c0;
            k_pack_samples<<<W.gridSmall, 128, 0, s>>>(st.out, C, W.packed);
            CR_CUDA(cudaMemcpyAsync(perSample + 3 * C.c0, W.packed, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaStreamSynchronize(s));
        }
    }
    if (errored) {
        // Re-run the first failing sample alone to recover the reference's message.
        const unsigned long long key = W.hostStats[kStatErrorKey];
        const uint32_t sample = static_cast<uint32_t>(key & ((1ull << 21) - 1));
        const uint64_t rank = key >> 21;
        const uint64_t tilesX = (static_cast<uint64_t>(o.width) + 15) / 16;
        const uint64_t tile = rank / 256, within = rank % 256;
        const uint32_t x = static_cast<uint32_t>((tile % tilesX) * 16 + within % 16);
        const uint32_t y = static_cast<uint32_t>((tile / tilesX) * 16 + within / 16);
        DevError host{};
        CR_CUDA(cudaStreamSynchronize(s));
        CR_CUDA(cudaMemsetAsync(W.detail, 0, sizeof(DevError), s));
        CR_CUDA(cudaMemsetAsync(W.stats, 0, 2 * sizeof(unsigned long long), s));
        k_trace_one<<<1, 32, 0, s>>>(dev, P, W.st, y * static_cast<uint32_t>(o.width) + x, sample, W.detail, W.stats, W.stats + 1);
        CR_CUDA(cudaMemcpyAsync(&host, W.detail, sizeof(DevError), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        if (!host.code) { host.code = -1; host.x = static_cast<int32_t>(x); host.y = static_cast<int32_t>(y); host.sample = static_cast<int32_t>(sample); }
        throw crh::Error(CR_ERR_RENDER, crh::sample_error_message(host));
    }
    k_film<<<W.gridSmall, 128, 0, s>>>(g.acc, g.film, pixels, o.samples);
    ++launches;
    g.filmWidth = o.width;
    g.filmHeight = o.height;
    CR_CUDA(cudaEventRecord(t1, s));
    if (filmHost) CR_CUDA(cudaMemcpyAsync(filmHost, g.film, 3 * pixels * sizeof(float), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(W.hostStats, W.stats, kStatWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    float deviceMs = 0;
    CR_CUDA(cudaEventElapsedTime(&deviceMs, t0, t1));
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->seconds = seconds;
        stats->device_ms = deviceMs;
        stats->trace_ms = traceMs; stats->shade_ms = shadeMs; stats->regen_ms = regenMs;
        stats->workers = referenceWorkers(o);
        stats->chunks = chunks;
        stats->iterations = static_cast<uint64_t>(iterations);
        stats->camera_samples = total;
        stats->boundary_retries = W.hostStats[kStatRetries];
        stats->extend_rays = W.hostStats[kStatExtendRays];
        stats->shadow_rays = W.hostStats[kStatShadowRays];
        stats->kernel_launches = launches;
        stats->extend_pairs = W.hostStats[kStatPairs];
        stats->extend_triangles = W.hostStats[kStatTris];
        stats->shadow_pairs = W.hostStats[kStatShadowPairs];
        stats->shadow_triangles = W.hostStats[kStatShadowTris];
    }
    if (progress) progress(total, total, seconds, user);
}

// ---- allocation-free render ----------------------------------------------------------------
// cr_gpu_render_noalloc renders through the same kernels as cr_gpu_render, but every buffer a
// render needs beyond the scene (path pool, queues, per-sample radiance, FP64 sums, film,
// counters) is carved out of one fixed array in device memory, so the call never allocates.
// Every GPU that loads this library holds the array until the process exits.
constexpr size_t kNoAllocBytes = size_t{32} << 20;          // 32 MiB per device
constexpr uint32_t kNoAllocPool = 32768;                   // path slots
constexpr uint64_t kNoAllocChunk = uint64_t{1} << 19;      // sample ids per chunk
constexpr uint64_t kNoAllocMaxPixels = 512 * 512;          // largest width*height
static __device__ __align__(256) unsigned char g_noallocScratch[kNoAllocBytes];

struct NoAllocLayout {
    PathSoA st;
    Queues q;
    unsigned long long* stats;
    DevError* detail;
    double* acc;
    float* film;
};
// Lays the workspace out from `base`; returns the bytes used (the same for every call).
size_t layoutNoAlloc(unsigned char* base, NoAllocLayout& L) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base ? base + off : nullptr;
        off = (off + bytes + 255) / 256 * 256;
        return static_cast<void*>(p);
    };
    const size_t n = kNoAllocPool;
    PathSoA& st = L.st;
    st.ray_o = static_cast<float4*>(take(16 * n)); st.ray_d = static_cast<float4*>(take(16 * n));
    st.ray_lo = static_cast<float4*>(take(16 * n)); st.hit_tri = static_cast<uint32_t*>(take(4 * n));
    st.thr = static_cast<float4*>(take(16 * n)); st.rad = static_cast<float4*>(take(16 * n));
    st.last_pos = static_cast<float4*>(take(16 * n)); st.absorb = static_cast<float4*>(take(16 * n));
    st.flags = static_cast<uint32_t*>(take(4 * n)); st.rng = static_cast<uint64_t*>(take(8 * n));
    st.prev_tri = static_cast<uint32_t*>(take(4 * n)); st.pixel = static_cast<uint32_t*>(take(4 * n));
    st.sample = static_cast<uint32_t*>(take(4 * n)); st.depth = static_cast<uint32_t*>(take(4 * n));
    st.sh_o = static_cast<float4*>(take(16 * n)); st.sh_d = static_cast<float4*>(take(16 * n));
    st.sh_lo = static_cast<float4*>(take(16 * n)); st.sh_c = static_cast<float4*>(take(16 * n));
    st.out = static_cast<float4*>(take(16 * kNoAllocChunk));
    for (int k = 0; k < 2; ++k) {
        L.q.extend[k] = static_cast<uint32_t*>(take(4 * n));
        L.q.shadow[k] = static_cast<uint32_t*>(take(4 * n));
        L.q.free[k] = static_cast<uint32_t*>(take(4 * n));
    }
    for (int c = 0; c < kShadeClasses; ++c) L.q.shade[c] = static_cast<uint32_t*>(take(4 * n));
    L.q.counts = static_cast<uint32_t*>(take(4 * kCountWords));
    L.stats = static_cast<unsigned long long*>(take(8 * kStatWords));
    L.detail = static_cast<DevError*>(take(sizeof(DevError)));
    L.acc = static_cast<double*>(take(24 * kNoAllocMaxPixels));
    L.film = static_cast<float*>(take(12 * kNoAllocMaxPixels));
    return off;
}

// Per-device set-up of the allocation-free render: the workspace's device address, looked up
// once per device (cudaGetSymbolAddress) with that device current (the host-side name of the
// array is not a device address), and two timing events. The address is cached for the life of
// the process: a host that calls cudaDeviceReset would invalidate it, and must not call
// cr_gpu_render_noalloc on that device afterwards.
struct NoAllocDevice {
    unsigned char* base = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
};
const NoAllocDevice& noallocDevice(int device) {
    static std::mutex m;
    static NoAllocDevice dev[64];
    if (device < 0 || device >= 64) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(m);
    NoAllocDevice& d = dev[device];
    if (!d.base) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) throw CudaError(e, "cudaGetSymbolAddress(g_noallocScratch)");
        CR_CUDA(cudaEventCreate(&d.start));
        CR_CUDA(cudaEventCreate(&d.stop));
        d.base = static_cast<unsigned char*>(p);
    }
    return d;
}

void renderNoAlloc(cr_gpu_scene& g, const cr_camera& camera, const cr_render_options& o, float* filmHost,
                   cr_render_stats* stats) {
    const auto start = std::chrono::steady_clock::now();
    crh::validate_options(o);
    const uint64_t pixels = static_cast<uint64_t>(o.width) * o.height;
    if (pixels > kNoAllocMaxPixels)
        throw crh::Error(CR_ERR_INVALID_ARGUMENT, "cr_gpu_render_noalloc: width*height " + std::to_string(pixels) +
                                                      " exceeds its fixed workspace limit of 262144 pixels (512x512)");
    const uint64_t total = pixels * static_cast<uint64_t>(o.samples);
    const cr_gpu_tuning tuning{};
    RenderParams P;
    try {
        P = makeParams(camera, o, tuning);
    } catch (const crh::Error& e) {
        throw crh::Error(CR_ERR_RENDER, std::string("Pixel (0,0), sample 0: ") + e.what());
    }
    CR_CUDA(cudaSetDevice(g.device));
    NoAllocLayout L;
    if (layoutNoAlloc(nullptr, L) > kNoAllocBytes) throw crh::Error(CR_ERR_LOGIC, "no-alloc workspace layout exceeds its array");
    const NoAllocDevice& D = noallocDevice(g.device);
    layoutNoAlloc(D.base, L);
    cudaStream_t s = g.stream;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device);
    // the kernel variants cr_gpu_render picks for this scene (host-side choices only): the
    // traversal without the alpha test when no triangle is alpha-masked, the lean shading
    // kernels without textures, punctual lights or alpha masks
    const bool noAlpha = !g.dev.any_alpha_mask;
    const bool lean = g.dev.texture_count == 0 && g.dev.punctual_count == 0 && !g.dev.any_alpha_mask;
    const void* traceK = noAlpha ? reinterpret_cast<const void*>(k_trace<false, false, true>) : reinterpret_cast<const void*>(k_trace<false>);
    // (the scene's own tables route rough conductors to the generic kernel: three classes here)
    constexpr int kClasses = 3;
    const void* shadeK[kClasses] = {
        lean ? reinterpret_cast<const void*>(k_shade<kShadeMiss, false, false, true>) : reinterpret_cast<const void*>(k_shade<kShadeMiss>),
        lean ? reinterpret_cast<const void*>(k_shade<kShadeNeeNull, false, false, true>) : reinterpret_cast<const void*>(k_shade<kShadeNeeNull>),
        lean ? reinterpret_cast<const void*>(k_shade<kShadeGeneric, false, false, true>) : reinterpret_cast<const void*>(k_shade<kShadeGeneric>)};
    const int gridRegen = occupancyGrid(reinterpret_cast<const void*>(k_regen<false>), 128, g.device);
    const int gridTrace = occupancyGrid(traceK, 128, g.device);
    int gridShadeK[kClasses];
    for (int c = 0; c < kClasses; ++c) gridShadeK[c] = occupancyGrid(shadeK[c], 128, g.device);
    const int gridSmall = sms * 8;
    // The workspace keeps the previous call's contents: clear what must start at zero.
    CR_CUDA(cudaMemsetAsync(L.acc, 0, 3 * pixels * sizeof(double), s));
    CR_CUDA(cudaMemsetAsync(L.stats, 0, kStatWords * sizeof(unsigned long long), s));
    const unsigned long long noError = ~0ull;
    CR_CUDA(cudaMemcpyAsync(L.stats + kStatErrorKey, &noError, sizeof(noError), cudaMemcpyHostToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    const ErrSink E{L.stats + kStatErrorKey, nullptr};
    uint32_t hostCounts[kCountWords];
    unsigned long long hostStats[kStatWords];
    const uint64_t pool = std::min<uint64_t>(kNoAllocPool, total);
    const uint64_t chunk = std::min<uint64_t>(total, kNoAllocChunk);
    uint64_t iterations = 0, launches = 0;
    bool errored = false;
    // no launch needs more blocks than the pool has 128-path batches
    const int poolBlocks = static_cast<int>((pool + 127) / 128);
    auto cap = [&](int grid) { return std::max(1, std::min(grid, poolBlocks)); };
    CR_CUDA(cudaEventRecord(D.start, s));
    for (uint64_t c0 = 0; c0 < total && !errored; c0 += chunk) {
        const Chunk C{c0, std::min<uint64_t>(total, c0 + chunk), pixels};
        CR_CUDA(cudaMemsetAsync(L.q.counts, 0, kCountWords * sizeof(uint32_t), s));
        const unsigned long long issuedStart = c0;
        CR_CUDA(cudaMemcpyAsync(L.stats + kStatIssued, &issuedStart, sizeof(issuedStart), cudaMemcpyHostToDevice, s));
        k_pool_init<<<gridSmall, 128, 0, s>>>(L.q, static_cast<uint32_t>(pool));
        ++launches;
        const uint64_t maxIterations = ((C.c1 - C.c0) / pool + 3) * 2 * static_cast<uint64_t>(o.bounces + 2) + 16;
        uint64_t iter = 0;
        int cur = 0;
        for (;;) {
            for (int b = 0; b < 8; ++b) {
                k_regen<false><<<cap(gridRegen), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{}, 1);
                if (noAlpha) k_trace<false, false, true><<<cap(gridTrace), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                else k_trace<false><<<cap(gridTrace), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                if (lean) {
                    k_shade<kShadeMiss, false, false, true><<<cap(gridShadeK[0]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                    k_shade<kShadeNeeNull, false, false, true><<<cap(gridShadeK[1]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                    k_shade<kShadeGeneric, false, false, true><<<cap(gridShadeK[2]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                } else {
                    k_shade<kShadeMiss><<<cap(gridShadeK[0]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                    k_shade<kShadeNeeNull><<<cap(gridShadeK[1]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                    k_shade<kShadeGeneric><<<cap(gridShadeK[2]), 128, 0, s>>>(g.dev, P, L.st, L.q, cur, C, E, L.stats, JobTable{});
                }
                launches += 5;
                cur ^= 1;
                ++iter;
                ++iterations;
            }
            CR_CUDA(cudaMemcpyAsync(hostCounts, L.q.counts, sizeof(hostCounts), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaMemcpyAsync(hostStats, L.stats, sizeof(hostStats), cudaMemcpyDeviceToHost, s));
            CR_CUDA(cudaStreamSynchronize(s));
            CR_CUDA(cudaGetLastError());
            const uint64_t live = hostCounts[kCountExtend0 + cur] + hostCounts[kCountShadow0 + (cur ^ 1)];
            if (hostStats[kStatErrorKey] != ~0ull) { errored = true; break; }
            if (hostStats[kStatIssued] >= C.c1 && live == 0) break;
            if (iter > maxIterations) throw crh::Error(CR_ERR_DEVICE_TIMEOUT, "paths still live after the iteration bound");
        }
        if (errored) break;
        k_accumulate<<<gridSmall, 128, 0, s>>>(L.st.out, C, L.acc);
        ++launches;
    }
    if (errored) {
        const unsigned long long key = hostStats[kStatErrorKey];
        const uint32_t sample = static_cast<uint32_t>(key & ((1ull << 21) - 1));
        const uint64_t rank = key >> 21, tilesX = (static_cast<uint64_t>(o.width) + 15) / 16;
        const uint64_t tile = rank / 256, within = rank % 256;
        const uint32_t x = static_cast<uint32_t>((tile % tilesX) * 16 + within % 16);
        const uint32_t y = static_cast<uint32_t>((tile / tilesX) * 16 + within / 16);
        DevError host{};
        CR_CUDA(cudaMemsetAsync(L.detail, 0, sizeof(DevError), s));
        CR_CUDA(cudaMemsetAsync(L.stats, 0, 2 * sizeof(unsigned long long), s));
        k_trace_one<<<1, 32, 0, s>>>(g.dev, P, L.st, y * static_cast<uint32_t>(o.width) + x, sample, L.detail, L.stats, L.stats + 1);
        CR_CUDA(cudaMemcpyAsync(&host, L.detail, sizeof(DevError), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        if (!host.code) { host.code = -1; host.x = static_cast<int32_t>(x); host.y = static_cast<int32_t>(y); host.sample = static_cast<int32_t>(sample); }
        throw crh::Error(CR_ERR_RENDER, crh::sample_error_message(host));
    }
    k_film<<<gridSmall, 128, 0, s>>>(L.acc, L.film, pixels, o.samples);
    ++launches;
    CR_CUDA(cudaEventRecord(D.stop, s));
    if (filmHost) CR_CUDA(cudaMemcpyAsync(filmHost, L.film, 3 * pixels * sizeof(float), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(hostStats, L.stats, sizeof(hostStats), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    float deviceMs = 0;
    CR_CUDA(cudaEventElapsedTime(&deviceMs, D.start, D.stop));
    if (stats) {
        // as cr_gpu_render fills them, except trace_ms/shade_ms/regen_ms (no phase timing here)
        std::memset(stats, 0, sizeof(*stats));
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        stats->device_ms = deviceMs;
        stats->extend_pairs = hostStats[kStatPairs];
        stats->extend_triangles = hostStats[kStatTris];
        stats->shadow_pairs = hostStats[kStatShadowPairs];
        stats->shadow_triangles = hostStats[kStatShadowTris];
        stats->workers = referenceWorkers(o);
        stats->chunks = static_cast<int32_t>((total + chunk - 1) / chunk);
        stats->camera_samples = total;
        stats->boundary_retries = hostStats[kStatRetries];
        stats->extend_rays = hostStats[kStatExtendRays];
        stats->shadow_rays = hostStats[kStatShadowRays];
        stats->kernel_launches = launches;
        stats->iterations = iterations;
    }
}


}  // namespace

extern "C" {

cr_status cr_gpu_allocation_count(uint64_t* count) {
    if (!count) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "count is NULL");
    *count = crh::allocation_count();
    return CR_OK;
}

cr_status cr_gpu_debug_fail_allocation(int64_t nth) {
    crh::inject_allocation_failure(nth);
    return CR_OK;
}

cr_status cr_gpu_device_count(int* count) {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { n = 0; cudaGetLastError(); }
    if (count) *count = n;
    return CR_OK;
}

cr_status cr_gpu_scene_create(const cr_scene_desc* scene, const cr_environment_desc* environment, int device, cr_gpu_scene** out) {
    try {
        if (!scene || !out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "scene or out is NULL");
        *out = nullptr;
        cr_environment_desc black{};
        const cr_environment_desc& env = environment ? *environment : black;
        auto g = std::make_unique<cr_gpu_scene>();
        g->device = device;
        CR_CUDA(cudaSetDevice(device));
        CR_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        uploadScene(*g, *scene, env);
        *out = g.release();
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_scene_destroy(cr_gpu_scene* scene) {
    delete scene;
    return CR_OK;
}

cr_status cr_gpu_scene_bytes(const cr_gpu_scene* scene, uint64_t* bytes) {
    if (!scene || !bytes) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "scene or bytes is NULL");
    *bytes = scene->geometry.bytes + scene->aliasAlloc.bytes + scene->filmAlloc.bytes + workspaceFor(scene->device).bytes();
    return CR_OK;
}

cr_status cr_gpu_intersect(cr_gpu_scene* g, const cr_ray* rays, uint64_t count, int any, uint32_t ignore,
                           cr_hit* hits, uint8_t* found, const cr_gpu_tuning* tuning) {
    try {
        if (!g) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "scene is NULL");
        if (count == 0) return CR_OK;
        if (!rays || !hits || !found) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "rays, hits or found is NULL");
        std::lock_guard<std::mutex> lock(g->mutex);
        const cr_gpu_tuning t = defaults(tuning);
        CR_CUDA(cudaSetDevice(g->device));
        cudaStream_t s = g->stream;
        DevAlloc tmp;
        cr_ray* dr = tmp.upload(rays, count, s);
        cr_hit* dh = tmp.upload(hits, count, s);
        uint8_t* df = tmp.alloc<uint8_t>(count);
        unsigned long long* de = tmp.alloc<unsigned long long>(1);
        const unsigned long long none = ~0ull;
        CR_CUDA(cudaMemcpyAsync(de, &none, sizeof(none), cudaMemcpyHostToDevice, s));
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
        k_intersect_batch<<<sms * 8, 128, 0, s>>>(g->dev, dr, dh, df, count, any, ignore, t.exact_traversal, de);
        CR_CUDA(cudaGetLastError());
        unsigned long long errIndex = 0;
        CR_CUDA(cudaMemcpyAsync(hits, dh, count * sizeof(cr_hit), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(found, df, count, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(&errIndex, de, sizeof(errIndex), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        tmp.release();
        if (errIndex != ~0ull) return crh::set_last_error(CR_ERR_LOGIC, "BVH traversal exceeded its bounded stack");
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_camera_rays(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options, uint32_t sample, cr_ray* rays) {
    try {
        if (!g || !camera || !options || !rays) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        crh::validate_options(*options);
        const cr_gpu_tuning t{};
        RenderParams P = makeParams(*camera, *options, t);
        CR_CUDA(cudaSetDevice(g->device));
        cudaStream_t s = g->stream;
        const uint64_t pixels = static_cast<uint64_t>(options->width) * options->height;
        DevAlloc tmp;
        cr_ray* dr = tmp.alloc<cr_ray>(pixels);
        unsigned long long* de = tmp.alloc<unsigned long long>(1);
        const unsigned long long none = ~0ull;
        CR_CUDA(cudaMemcpyAsync(de, &none, sizeof(none), cudaMemcpyHostToDevice, s));
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
        k_camera_rays<<<sms * 8, 128, 0, s>>>(P, sample, dr, de);
        CR_CUDA(cudaGetLastError());
        unsigned long long key = 0;
        CR_CUDA(cudaMemcpyAsync(rays, dr, pixels * sizeof(cr_ray), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(&key, de, sizeof(key), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        tmp.release();
        if (key != ~0ull) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "Unrepresentable perspective ray");
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options, cr_progress_fn progress,
                        void* user, float* film_rgb, cr_render_stats* stats, const cr_gpu_tuning* tuning) {
    try {
        if (!g || !camera || !options) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        renderImpl(*g, *camera, *options, progress, user, film_rgb, stats, defaults(tuning), nullptr);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render_resident(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options,
                                 cr_render_stats* stats, const cr_gpu_tuning* tuning, float* per_sample_rgb) {
    try {
        if (!g || !camera || !options) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        renderImpl(*g, *camera, *options, nullptr, nullptr, nullptr, stats, defaults(tuning), per_sample_rgb);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

static_assert(sizeof(cr_traced_ray) == 96, "cr_traced_ray layout");

cr_status cr_gpu_environment_sample(cr_gpu_scene* g, int alias, uint64_t seed, uint64_t count, uint32_t* texels,
                                    float* densities) {
    try {
        if (!g || (count && (!texels || !densities))) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        if (!g->dev.env_has_image) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "the scene has no environment image");
        CR_CUDA(cudaSetDevice(g->device));
        if (alias) ensureAlias(*g);
        DevScene dev = g->dev;
        if (alias) dev.env_pdf = g->aliasPdf;
        DevAlloc mem;
        struct Release {
            DevAlloc& m;
            cudaStream_t s;
            ~Release() { cudaStreamSynchronize(s); m.release(); }
        } release{mem, g->stream};
        const uint64_t batch = std::min<uint64_t>(std::max<uint64_t>(count, 1), uint64_t{1} << 26);
        uint32_t* dTex = mem.alloc<uint32_t>(batch);
        float* dPdf = mem.alloc<float>(batch);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
        for (uint64_t b = 0; b < count; b += batch) {  // sample i of the call uses stream i
            const uint64_t m = std::min<uint64_t>(batch, count - b);
            k_env_samples<<<sms * 8, 128, 0, g->stream>>>(dev, alias, seed, b, m, dTex, dPdf);
            CR_CUDA(cudaGetLastError());
            CR_CUDA(cudaMemcpyAsync(texels + b, dTex, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
            CR_CUDA(cudaMemcpyAsync(densities + b, dPdf, m * sizeof(float), cudaMemcpyDeviceToHost, g->stream));
            CR_CUDA(cudaStreamSynchronize(g->stream));
        }
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render_trace_dump(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options,
                                   const cr_gpu_tuning* tuning, cr_traced_ray* rays, uint64_t capacity, uint64_t* count) {
    try {
        if (!g || !camera || !options || !count || (capacity && !rays))
            return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        CR_CUDA(cudaSetDevice(g->device));
        cr_gpu_tuning t = defaults(tuning);
        t.count_traversal = 1;  // the counting kernels record the rays
        DevAlloc mem;
        struct Release {
            DevAlloc& m;
            cudaStream_t s;
            ~Release() { cudaStreamSynchronize(s); m.release(); }
        } release{mem, g->stream};
        TraceDump d;
        d.capacity = capacity;
        d.rays = mem.alloc<cr_traced_ray>(capacity ? capacity : 1);
        d.count = mem.alloc<unsigned long long>(1);
        CR_CUDA(cudaMemsetAsync(d.count, 0, sizeof(unsigned long long), g->stream));
        renderImpl(*g, *camera, *options, nullptr, nullptr, nullptr, nullptr, t, nullptr, Frames{}, nullptr, &d);
        unsigned long long n = 0;
        CR_CUDA(cudaMemcpyAsync(&n, d.count, sizeof(n), cudaMemcpyDeviceToHost, g->stream));
        CR_CUDA(cudaStreamSynchronize(g->stream));
        const uint64_t copy = std::min<uint64_t>(n, capacity);
        if (copy) CR_CUDA(cudaMemcpyAsync(rays, d.rays, copy * sizeof(cr_traced_ray), cudaMemcpyDeviceToHost, g->stream));
        CR_CUDA(cudaStreamSynchronize(g->stream));
        *count = n;
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render_noalloc(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options,
                                float* film_rgb, cr_render_stats* stats) {
    try {
        if (!g || !camera || !options) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        renderNoAlloc(*g, *camera, *options, film_rgb, stats);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render_progressive(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options,
                                    uint32_t every_samples, int format, float exposure, cr_frame_fn on_frame, void* user,
                                    float* film_rgb, cr_render_stats* stats, const cr_gpu_tuning* tuning) {
    try {
        if (!g || !camera || !options) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        if (every_samples == 0) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "every_samples must be positive");
        std::lock_guard<std::mutex> lock(g->mutex);
        Frames f;
        f.every = every_samples; f.format = format; f.exposure = exposure; f.fn = on_frame; f.user = user;
        renderImpl(*g, *camera, *options, nullptr, nullptr, film_rgb, stats, defaults(tuning), nullptr, f);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_render_guided(cr_gpu_scene* g, const cr_camera* camera, const cr_render_options* options, cr_guide* guide,
                               const cr_guide_options* gopt, float* film_rgb, cr_render_stats* stats, const cr_gpu_tuning* tuning) {
    try {
        if (!g || !camera || !options || !guide) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        GuideRun run;
        run.gd = guide;
        if (gopt) {
            run.trainSamples = gopt->train_samples;
            if (gopt->guide_probability > 0) run.probability = std::min(gopt->guide_probability, 0.95f);
            if (gopt->batch) run.batch = gopt->batch;
            if (gopt->epochs) run.epochs = gopt->epochs;
        }
        renderImpl(*g, *camera, *options, nullptr, nullptr, film_rgb, stats, defaults(tuning), nullptr, Frames{}, &run);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_film_encode(cr_gpu_scene* g, int format, float exposure, void* out, uint64_t capacity, uint64_t* size) {
    try {
        if (!g || !size) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        if (!g->filmWidth) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "the scene has no film: render first");
        CR_CUDA(cudaSetDevice(g->device));
        const uint64_t n = crg::encode_film(g->film, g->filmWidth, g->filmHeight, format, exposure, g->stream, out, capacity);
        *size = n;
        if (out && capacity < n)
            return crh::set_last_error(CR_ERR_OUT_OF_RANGE, "output buffer holds " + std::to_string(capacity) +
                                                                " bytes; the encoding needs " + std::to_string(n));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_film_download(cr_gpu_scene* g, float* film_rgb, uint64_t floats) {
    try {
        if (!g || !film_rgb) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(g->mutex);
        if (floats > 3 * g->filmPixels) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "film request larger than the last render");
        CR_CUDA(cudaSetDevice(g->device));
        CR_CUDA(cudaMemcpyAsync(film_rgb, g->film, floats * sizeof(float), cudaMemcpyDeviceToHost, g->stream));
        CR_CUDA(cudaStreamSynchronize(g->stream));
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

}  // extern "C"
