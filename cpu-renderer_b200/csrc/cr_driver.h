// Host-side pieces shared by the single-render driver (cr_render.cu) and the multi-job engine
// (cr_engine.cu): CUDA error mapping, device allocations, the scene handle.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cr_gpu.h"
#include "cr_host.h"
#include "cr_internal.h"

namespace crd {

struct CudaError : crh::Error {
    CudaError(cudaError_t e, const char* what)
        : crh::Error(e == cudaErrorMemoryAllocation ? CR_ERR_OUT_OF_MEMORY : CR_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e)) {}
};
#define CR_CUDA(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) throw crd::CudaError(e_, #call); } while (0)

// Device allocation owned by a scene.
// Device blocks given back by DevAlloc::release are kept per device for reuse, up to
// kBlockCacheBytes: handing large blocks back to the driver (cudaFree) occasionally stalls for
// hundreds of milliseconds, and a scene created again with the same array sizes then reuses its
// blocks at once. A block is reused for requests of at least half its size. An allocation that
// fails empties the device's cache and tries again.
class BlockCache {
  public:
    static constexpr size_t kBlockCacheBytes = size_t{48} << 30;
    static BlockCache& get() {
        static BlockCache* c = new BlockCache();  // lives until the process exits
        return *c;
    }
    // A cached block of at least `bytes` (and at most twice that), with its own size; or null.
    std::pair<void*, size_t> take(int device, size_t bytes) {
        std::lock_guard<std::mutex> lock(m_);
        auto& bin = blocks_[device];
        auto it = bin.lower_bound(bytes);
        if (it == bin.end() || it->first > 2 * bytes) return {nullptr, 0};
        const std::pair<void*, size_t> b{it->second, it->first};
        held_[device] -= it->first;
        bin.erase(it);
        return b;
    }
    void give(int device, void* p, size_t bytes) {
        {
            std::lock_guard<std::mutex> lock(m_);
            if (held_[device] + bytes <= kBlockCacheBytes) {
                blocks_[device].emplace(bytes, p);
                held_[device] += bytes;
                return;
            }
        }
        cudaFree(p);
    }
    void flush(int device) {
        std::lock_guard<std::mutex> lock(m_);
        for (auto& b : blocks_[device]) cudaFree(b.second);
        blocks_[device].clear();
        held_[device] = 0;
    }

  private:
    std::mutex m_;
    std::map<int, std::multimap<size_t, void*>> blocks_;
    std::map<int, size_t> held_;
};

// Page-locked host blocks kept for reuse by scene uploads: copies from page-locked memory run
// asynchronously at the link's full rate, and pinning fresh memory for every upload would cost
// more than the copy itself. At most kHeld bytes stay cached; blocks live until process exit.
class PinnedCache {
  public:
    static PinnedCache& get() {
        static PinnedCache* c = new PinnedCache;  // never destroyed: outlives the CUDA runtime's users
        return *c;
    }
    // A block of at least `bytes` (the cached block's own size is returned), or {nullptr, 0}
    // when page-locked memory cannot be had.
    std::pair<void*, size_t> take(size_t bytes) {
        {
            std::lock_guard<std::mutex> lock(m_);
            auto it = free_.lower_bound(bytes);
            if (it != free_.end()) {
                const std::pair<void*, size_t> r{it->second, it->first};
                held_ -= it->first;
                free_.erase(it);
                return r;
            }
        }
        void* p = nullptr;
        crh::count_allocation();
        if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return {nullptr, 0};
        }
        return {p, bytes};
    }
    void give(void* p, size_t bytes) {
        std::lock_guard<std::mutex> lock(m_);
        free_.insert({bytes, p});
        held_ += bytes;
        while (held_ > kHeld && !free_.empty()) {
            auto it = free_.begin();
            cudaFreeHost(it->second);
            held_ -= it->first;
            free_.erase(it);
        }
    }

  private:
    static constexpr size_t kHeld = size_t{1} << 31;
    std::mutex m_;
    std::multimap<size_t, void*> free_;
    size_t held_ = 0;
};

struct DevAlloc {
    std::vector<std::pair<void*, size_t>> blocks;
    uint64_t bytes = 0;
    template <class T> T* alloc(size_t count) {
        if (count == 0) count = 1;
        const size_t want = count * sizeof(T);
        int device = 0;
        CR_CUDA(cudaGetDevice(&device));
        crh::count_allocation();
        if (crh::injected_allocation_failure()) throw CudaError(cudaErrorMemoryAllocation, "device allocation (injected failure)");
        auto [p, have] = BlockCache::get().take(device, want);
        if (!p) {
            if (cudaMalloc(&p, want) != cudaSuccess) {
                cudaGetLastError();
                BlockCache::get().flush(device);
                CR_CUDA(cudaMalloc(&p, want));
            }
            have = want;
        }
        blocks.push_back({p, have});
        bytes += want;
        return static_cast<T*>(p);
    }
    template <class T> T* upload(const T* src, size_t count, cudaStream_t s) {
        T* d = alloc<T>(count);
        if (count) CR_CUDA(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
        return d;
    }
    // The caller has finished every use of the blocks (its streams are synchronised).
    void release() {
        int device = 0;
        cudaGetDevice(&device);
        for (auto& b : blocks) BlockCache::get().give(device, b.first, b.second);
        blocks.clear();
        bytes = 0;
    }
};

inline int occupancyGrid(const void* kernel, int block, int device) {
    int sms = 0, perSm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, block, 0);
    if (perSm < 1) perSm = 1;
    return sms * perSm;
}


// The path pool's state arrays and queues for n slots.
inline void allocPaths(DevAlloc& work, size_t n, crg::PathSoA& st, crg::Queues& q) {
    using namespace crg;
    st.ray_o = work.alloc<float4>(n); st.ray_d = work.alloc<float4>(n); st.ray_lo = work.alloc<float4>(n);
    st.hit_tri = work.alloc<uint32_t>(n);
    st.thr = work.alloc<float4>(n); st.rad = work.alloc<float4>(n); st.last_pos = work.alloc<float4>(n);
    st.absorb = work.alloc<float4>(n); st.flags = work.alloc<uint32_t>(n);
    st.rng = work.alloc<uint64_t>(n); st.prev_tri = work.alloc<uint32_t>(n);
    st.pixel = work.alloc<uint32_t>(n); st.sample = work.alloc<uint32_t>(n); st.depth = work.alloc<uint32_t>(n);
    st.sh_o = work.alloc<float4>(n); st.sh_d = work.alloc<float4>(n); st.sh_lo = work.alloc<float4>(n);
    st.sh_c = work.alloc<float4>(n);
    for (int k = 0; k < 2; ++k) {
        q.extend[k] = work.alloc<uint32_t>(n);
        q.shadow[k] = work.alloc<uint32_t>(n);
        q.free[k] = work.alloc<uint32_t>(n);
    }
    for (int c = 0; c < kShadeClasses; ++c) q.shade[c] = work.alloc<uint32_t>(n);
    q.counts = work.alloc<uint32_t>(kCountWords);
}

cr_status fail(const std::exception& e);
cr_gpu_tuning defaults(const cr_gpu_tuning* t);
crg::RenderParams makeParams(const cr_camera& camera, const cr_render_options& o, const cr_gpu_tuning& t);
int referenceWorkers(const cr_render_options& o);

}  // namespace crd

struct cr_gpu_scene {
    int device = 0;
    cudaStream_t stream = nullptr;
    crd::DevAlloc geometry;  // scene data
    crg::DevScene dev{};
    uint64_t triangleCount = 0;
    crh::EnvTables env;  // host copy, for the alias table built on demand
    crd::DevAlloc aliasAlloc;
    const float* aliasPdf = nullptr;  // the alias sampler's texel densities (device), once built
    // film of the last render: FP64 sums and the float film
    double* acc = nullptr;
    float* film = nullptr;
    size_t filmPixels = 0;
    int filmWidth = 0, filmHeight = 0;  // of the last render's film (0: none yet)
    crd::DevAlloc filmAlloc;
    std::mutex mutex;

    ~cr_gpu_scene() {
        if (device >= 0) cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        geometry.release();
        aliasAlloc.release();
        filmAlloc.release();
        if (stream) cudaStreamDestroy(stream);
    }

    void ensureFilm(size_t pixels) {
        if (pixels <= filmPixels) return;
        CR_CUDA(cudaStreamSynchronize(stream));
        filmAlloc.release();
        // The last film went back with its blocks (a failed allocation below may even hand them
        // to the driver): until a render completes in the new ones there is no film to read.
        acc = nullptr;
        film = nullptr;
        filmPixels = 0;
        filmWidth = filmHeight = 0;
        acc = filmAlloc.alloc<double>(3 * pixels);
        film = filmAlloc.alloc<float>(3 * pixels);
        filmPixels = pixels;
    }
};

