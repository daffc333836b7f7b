// Multi-job engine: many renders in one path pool (cr_gpu_render_batch, cr_server_*).
//
// The pool and kernels are the single render's (cr_kernels.cuh) in their MULTI form: a path's
// job comes from the issue range it was started from. The host side here keeps the issue
// list and the jobs:
//
//   admit     a job gets a slot in the device job tables (its scene's DevScene and its
//             RenderParams), FP64 pixel sums and a film, if the memory budget allows
//   issue     the jobs' remaining samples are cut into ranges (at most range_samples: blocks
//             of pixels with all their samples, or for a progressive job whole samples of
//             every pixel, never across a frame boundary) and appended to the issue list, each to
//             the job with the fewest samples per pixel issued, while the per-sample
//             radiance arena has room and the pool is not already fed a pool's worth ahead
//   run       iterations_per_step iterations of k_regen / k_trace / k_shade x3 (one CUDA
//             graph per kernel variant when use_graphs), k_regen refilling freed slots every
//             refill_interval; the variant drops the alpha test and the texture and punctual
//             light code when no active job's scene needs them
//   complete  finished-sample counters are read back; a job's ranges are summed into its
//             pixel sums strictly in order (k_accumulate), so the film is the ordered FP64
//             sum of its samples exactly as in a single render; frames and results go out
//
// A job whose sample fails stops taking new ranges; once its issued ranges have drained, the
// failing sample is re-run alone to recover the reference's message, as a single render does.
// In a batch, jobs that fill the pool on their own render alone through the single-render
// entry points, on a helper thread beside the pool (runBatch).
#include "cr_kernels.cuh"
#include "cr_driver.h"
#include "cr_encode.h"
#include "cr_host.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace crg;
using namespace crd;

namespace {

constexpr uint32_t kMaxJobSlots = 1024;
constexpr uint32_t kMaxRanges = 1u << 18;
constexpr unsigned long long kNoKey = ~0ull;

struct EngineConfig {
    uint64_t pool = uint64_t{1} << 24;
    uint64_t rangeSamples = uint64_t{1} << 22;
    uint64_t outSamples = 0;
    uint32_t refill = 1;
    uint32_t refillPercent = 0;
    uint32_t iters = 8;
    bool graphs = true;
    int policy = 0;  // 1: jobs in order, 2: fewest samples per pixel first
    uint64_t budget = 150ull << 30;
    int block = 128;  // threads per block of the pool's traversal and shading kernels
};

EngineConfig makeConfig(const cr_engine_tuning* t, int defaultPolicy) {
    EngineConfig c;
    c.policy = defaultPolicy;
    if (t) {
        if (t->pool_paths) c.pool = t->pool_paths;
        if (t->range_samples) c.rangeSamples = t->range_samples;
        if (t->refill_interval) c.refill = t->refill_interval;
        c.refillPercent = std::min<uint32_t>(100, t->refill_free_percent);
        if (t->iterations_per_step) c.iters = t->iterations_per_step;
        c.graphs = t->use_graphs != 0;
        if (t->issue_policy == 1 || t->issue_policy == 2) c.policy = t->issue_policy;
        if (t->memory_budget) c.budget = t->memory_budget;
        if (t->block_size == 64 || t->block_size == 256) c.block = static_cast<int>(t->block_size);
    }
    c.pool = std::max<uint64_t>(1024, (c.pool + 127) / 128 * 128);
    c.rangeSamples = std::max<uint64_t>(1024, c.rangeSamples);
    c.iters = std::max<uint32_t>(2, (c.iters + 1) / 2 * 2);  // even: each step starts at parity 0
    c.outSamples = std::max<uint64_t>(2 * c.pool, 4 * c.rangeSamples);
    return c;
}

// First-fit spans of the per-sample radiance arena.
class Arena {
  public:
    explicit Arena(uint64_t size) { free_[0] = size; }
    bool take(uint64_t n, uint64_t& at) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            at = it->first;
            const uint64_t rest = it->second - n, next = it->first + n;
            free_.erase(it);
            if (rest) free_[next] = rest;
            return true;
        }
        return false;
    }
    void give(uint64_t at, uint64_t n) {
        auto it = free_.emplace(at, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
        }
    }

  private:
    std::map<uint64_t, uint64_t> free_;
};

struct Active {
    cr_job* job = nullptr;
    uint64_t ticket = 0;
    uint32_t slot = 0;
    DevAlloc buffers;
    double* acc = nullptr;
    float* film = nullptr;
    RenderParams P{};
    uint64_t pixels = 0, total = 0, frameSamples = 0;  // frameSamples: every * pixels (0: none)
    uint64_t issued = 0, accumulated = 0, bytes = 0, chunks = 0;
    std::deque<uint32_t> ranges;  // issued, not yet summed, in sample order
    bool failed = false;
    unsigned long long errKey = kNoKey;
    uint64_t admitStep = 0;  // the engine step that admitted the job
    std::vector<unsigned char> frame;
};

class Engine {
  public:
    Engine(int device, const cr_engine_tuning* tuning, int defaultPolicy)
        : device_(device), cfg_(makeConfig(tuning, defaultPolicy)), arena_(0) {
        try {
            setUp();
        } catch (...) {
            releaseAll();  // a constructor that throws runs no destructor
            throw;
        }
    }
    ~Engine() { releaseAll(); }

  private:
    void setUp() {
        CR_CUDA(cudaSetDevice(device_));
        CR_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
        start_ = std::chrono::steady_clock::now();
        arena_ = Arena(cfg_.outSamples);
        allocPaths(pool_, cfg_.pool, st_, q_);
        st_.out = pool_.alloc<float4>(cfg_.outSamples);
        slotOf_ = pool_.alloc<uint2>(cfg_.pool);
        stats_ = pool_.alloc<unsigned long long>(kStatWords);
        errKeys_ = pool_.alloc<unsigned long long>(kMaxJobSlots);
        retries_ = pool_.alloc<unsigned long long>(kMaxJobSlots);
        scenes_ = pool_.alloc<DevScene>(kMaxJobSlots);
        params_ = pool_.alloc<RenderParams>(kMaxJobSlots);
        ranges_ = pool_.alloc<IssueRange>(kMaxRanges);
        done_ = pool_.alloc<unsigned long long>(kMaxRanges);
        // [0] issue end, [1] range count, [2..3] issued, [4..5] free-ring head, [6] free-ring tail
        // (host staging hCtl_: [0..1] and [2..3] alternate for the issue end and range count)
        ctl_ = pool_.alloc<unsigned long long>(8);
        allocPaths(scratchAlloc_, 1, one_, oneQ_);
        one_.out = scratchAlloc_.alloc<float4>(1);
        oneDetail_ = scratchAlloc_.alloc<DevError>(1);
        oneStats_ = scratchAlloc_.alloc<unsigned long long>(2);
        for (int k = 0; k < 2 + 2 * 5; ++k) crh::count_allocation();
        CR_CUDA(cudaMallocHost(&hRanges_, kMaxRanges * sizeof(IssueRange)));
        CR_CUDA(cudaMallocHost(&hCtl_, 8 * sizeof(unsigned long long)));
        for (Mirror& M : mirrors_) {
            CR_CUDA(cudaMallocHost(&M.done, kMaxRanges * sizeof(unsigned long long)));
            CR_CUDA(cudaMallocHost(&M.ctl, 4 * sizeof(unsigned long long)));
            CR_CUDA(cudaMallocHost(&M.err, kMaxJobSlots * sizeof(unsigned long long)));
            CR_CUDA(cudaMallocHost(&M.counts, kCountWords * sizeof(uint32_t)));
            CR_CUDA(cudaMallocHost(&M.stats, kStatWords * sizeof(unsigned long long)));
            CR_CUDA(cudaEventCreateWithFlags(&M.ready, cudaEventDisableTiming));
        }
        hDone_ = mirrors_[0].done;
        hErr_ = mirrors_[0].err;
        CR_CUDA(cudaMemsetAsync(ctl_, 0, 8 * sizeof(unsigned long long), s_));
        CR_CUDA(cudaMemsetAsync(done_, 0, kMaxRanges * sizeof(unsigned long long), s_));
        CR_CUDA(cudaMemsetAsync(stats_, 0, kStatWords * sizeof(unsigned long long), s_));
        CR_CUDA(cudaMemsetAsync(q_.counts, 0, kCountWords * sizeof(uint32_t), s_));
        switch (cfg_.block) {
            case 64: setGrids<64>(); break;
            case 256: setGrids<256>(); break;
            default: setGrids<128>(); break;
        }
        gridRegen_ = occupancyGrid(reinterpret_cast<const void*>(k_regen<true>), 128, device_);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
        gridSmall_ = sms * 8;
        k_pool_init<<<gridSmall_, 128, 0, s_>>>(q_, static_cast<uint32_t>(cfg_.pool));  // the ring: every slot
        CR_CUDA(cudaGetLastError());
        hCtl_[6] = cfg_.pool;
        CR_CUDA(cudaMemcpyAsync(ctl_ + 6, hCtl_ + 6, sizeof(unsigned long long), cudaMemcpyHostToDevice, s_));
        CR_CUDA(cudaStreamSynchronize(s_));
        for (uint32_t i = 0; i < kMaxJobSlots; ++i) freeSlots_.push_back(kMaxJobSlots - 1 - i);
        hScenes_.resize(kMaxJobSlots);
        hParams_.resize(kMaxJobSlots);
        J_.scenes = scenes_; J_.params = params_; J_.ranges = ranges_; J_.ctl = ctl_; J_.issued = ctl_ + 2;
        J_.done = done_; J_.errKeys = errKeys_; J_.retries = retries_; J_.slot = slotOf_;
        J_.refillMin = static_cast<uint32_t>(cfg_.pool * cfg_.refillPercent / 100);
        J_.ring = q_.free[1];
        J_.head = ctl_ + 4;
        J_.tail = ctl_ + 6;
        J_.poolSize = cfg_.pool;
    }

    // Everything the engine holds; also what a failed set-up had taken so far.
    void releaseAll() {
        cudaSetDevice(device_);
        if (s_) cudaStreamSynchronize(s_);
        for (auto& g : graph_) if (g) cudaGraphExecDestroy(g);
        for (auto& a : active_) a.buffers.release();
        pool_.release();
        scratchAlloc_.release();
        cudaFreeHost(hRanges_); cudaFreeHost(hCtl_);
        for (Mirror& M : mirrors_) {
            cudaFreeHost(M.done); cudaFreeHost(M.ctl); cudaFreeHost(M.err); cudaFreeHost(M.counts); cudaFreeHost(M.stats);
            if (M.ready) cudaEventDestroy(M.ready);
        }
        if (s_) cudaStreamDestroy(s_);
    }

  public:
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count(); }

    uint64_t submit(cr_job* j) {
        std::lock_guard<std::mutex> lock(mutex_);
        j->submitted_at = now();
        j->started_at = j->first_frame_at = j->finished_at = 0;
        j->status = CR_OK;
        j->error[0] = 0;
        std::memset(&j->stats, 0, sizeof(j->stats));
        const uint64_t t = ++lastTicket_;
        pending_.push_back({j, t});
        cv_.notify_all();
        return t;
    }

    // One step: admit, issue, run, then complete the previous step. The counters a step's
    // graph leaves are copied to one of two host mirrors behind it, and are read after the next
    // step's graph has been queued: the device works on step k+1 while the host completes step
    // k (issue() sees finished ranges one step late, which only delays reuse of their space).
    // Returns false when there is nothing to do.
    bool step() {
        CR_CUDA(cudaSetDevice(device_));
        ++stepCount_;
        admit();
        if (active_.empty()) {
            drainPoll();
            return false;
        }
        const auto t0 = std::chrono::steady_clock::now();
        issue();
        run();
        enqueuePoll(mirror_);
        if (pollPending_) {
            processPoll(mirror_ ^ 1);
            complete();
        }
        pollPending_ = true;
        mirror_ ^= 1;
        std::lock_guard<std::mutex> lock(mutex_);
        busySeconds_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return true;
    }

    bool idle() {
        std::lock_guard<std::mutex> lock(mutex_);
        return pending_.empty() && active_.empty();
    }

    // Server side: waits for work or stop; true when there may be work.
    bool waitForWork(const std::atomic<bool>& stop) {
        std::unique_lock<std::mutex> lock(mutex_);
        cv_.wait(lock, [&] { return stop.load() || !pending_.empty(); });
        return !pending_.empty();
    }
    void wake() { cv_.notify_all(); }

    cr_status wait(uint64_t ticket, double timeout) {
        std::unique_lock<std::mutex> lock(mutex_);
        auto ready = [&] { return ended_.count(ticket) != 0; };
        if (timeout < 0) cv_.wait(lock, ready);
        else if (!cv_.wait_for(lock, std::chrono::duration<double>(timeout), ready)) return CR_ERR_DEVICE_TIMEOUT;
        return ended_[ticket];
    }

    // Ends every job that has not ended (engine failure).
    void failAll(cr_status status, const std::string& message) {
        std::vector<std::pair<cr_job*, uint64_t>> victims;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            for (auto& p : pending_) victims.push_back(p);
            pending_.clear();
        }
        // the jobs' buffers go back once nothing queued can still write them (after a CUDA
        // error the wait returns at once)
        if (s_) cudaStreamSynchronize(s_);
        cudaGetLastError();
        for (auto& a : active_) {
            victims.push_back({a.job, a.ticket});
            a.buffers.release();
        }
        active_.clear();
        usedBytes_ = 0;
        for (auto& v : victims) endJob(v.first, v.second, status, message);
    }

    cr_engine_stats stats() {
        std::lock_guard<std::mutex> lock(mutex_);
        cr_engine_stats s = stats_host_;
        s.seconds = busySeconds_;
        s.extend_rays += solo_.extend_rays;
        s.shadow_rays += solo_.shadow_rays;
        return s;
    }

    // Registers a job that will render alone (it never enters the pending queue): its ticket.
    uint64_t registerSolo(cr_job* j) {
        std::lock_guard<std::mutex> lock(mutex_);
        j->submitted_at = now();
        j->started_at = j->first_frame_at = j->finished_at = 0;
        j->status = CR_OK;
        j->error[0] = 0;
        std::memset(&j->stats, 0, sizeof(j->stats));
        return ++lastTicket_;
    }

    // A batch job that fills the pool on its own renders alone through the single-render entry
    // points: its rays then stay in its own sample order (the pool holds no other job's paths)
    // and the kernels can be the lean variants its scene allows. Its times, status and stats
    // are kept as for a pooled job. Runs on its own host thread beside step().
    void runSolo(cr_job* j, uint64_t ticket) {
        j->started_at = now();
        struct Hook {
            Engine* e;
            cr_job* j;
            static void frame(uint32_t spp, const void* data, uint64_t size, void* user) {
                Hook* h = static_cast<Hook*>(user);
                if (!h->j->first_frame_at) h->j->first_frame_at = h->e->now();
                if (h->j->on_frame) h->j->on_frame(spp, data, size, h->j->user);
            }
        } hook{this, j};
        const cr_status st = j->every_samples
            ? cr_gpu_render_progressive(j->scene, &j->camera, &j->options, j->every_samples, j->format, j->exposure,
                                        &Hook::frame, &hook, j->film_rgb, &j->stats, nullptr)
            : cr_gpu_render(j->scene, &j->camera, &j->options, nullptr, nullptr, j->film_rgb, &j->stats, nullptr);
        char message[sizeof(j->error)] = {0};
        if (st != CR_OK) cr_gpu_last_error(message, sizeof(message));
        endJob(j, ticket, st, message);
        std::lock_guard<std::mutex> lock(mutex_);
        if (st == CR_OK) stats_host_.camera_samples += j->stats.camera_samples;
        stats_host_.iterations += j->stats.iterations;
        stats_host_.launches += j->stats.kernel_launches;
        solo_.extend_rays += j->stats.extend_rays;
        solo_.shadow_rays += j->stats.shadow_rays;
    }
    int device() const { return device_; }

  private:
    void endJob(cr_job* j, uint64_t ticket, cr_status status, const std::string& message) {
        j->status = status;
        std::snprintf(j->error, sizeof(j->error), "%s", message.c_str());
        j->finished_at = now();
        std::lock_guard<std::mutex> lock(mutex_);
        if (status == CR_OK) ++stats_host_.jobs_done; else ++stats_host_.jobs_failed;
        ended_[ticket] = status;
        cv_.notify_all();
    }

    void admit() {
        for (;;) {
            std::pair<cr_job*, uint64_t> next;
            {
                std::lock_guard<std::mutex> lock(mutex_);
                if (pending_.empty()) return;
                next = pending_.front();
            }
            cr_job* j = next.first;
            Active a;
            a.job = j;
            a.ticket = next.second;
            try {
                if (!j->scene) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "job scene is NULL");
                if (j->scene->device != device_) throw crh::Error(CR_ERR_INVALID_ARGUMENT, "job scene lives on another device");
                crh::validate_options(j->options);
                const cr_gpu_tuning t{};
                try {
                    a.P = makeParams(j->camera, j->options, t);
                } catch (const crh::Error& e) {
                    throw crh::Error(CR_ERR_RENDER, std::string("Pixel (0,0), sample 0: ") + e.what());
                }
                a.pixels = static_cast<uint64_t>(j->options.width) * j->options.height;
                a.total = a.pixels * static_cast<uint64_t>(j->options.samples);
                if (j->every_samples) {
                    if (j->format != CR_ENCODE_SRGB8 && j->format != CR_ENCODE_RGBE && j->format != CR_ENCODE_HDR_FILE)
                        throw crh::Error(CR_ERR_INVALID_ARGUMENT, "unknown encode format");
                    crh::check_image_dims(j->options.width, j->options.height,
                                          j->format == CR_ENCODE_SRGB8 ? "PNG output" : "HDR output");
                    if (j->format == CR_ENCODE_SRGB8) { float th[256]; crh::display_thresholds(j->exposure, th); }
                    a.frameSamples = static_cast<uint64_t>(j->every_samples) * a.pixels;
                    a.frame.resize(j->format == CR_ENCODE_SRGB8 ? 3 * a.pixels
                                   : j->format == CR_ENCODE_RGBE ? 4 * a.pixels
                                   : crh::hdr_header(j->options.width, j->options.height).size() +
                                         static_cast<uint64_t>(j->options.height) * (4 + 8ull * j->options.width + 8));
                }
                a.bytes = a.pixels * (3 * sizeof(double) + 3 * sizeof(float));
                if (a.bytes > cfg_.budget)
                    throw crh::Error(CR_ERR_OUT_OF_MEMORY, "job needs " + std::to_string(a.bytes) +
                                                               " bytes of buffers, more than the memory budget");
            } catch (const crh::Error& e) {
                popPending();
                endJob(j, a.ticket, e.status, e.what());
                continue;
            }
            if (freeSlots_.empty() || (usedBytes_ + a.bytes > cfg_.budget && !active_.empty())) return;  // wait
            try {
                a.acc = a.buffers.alloc<double>(3 * a.pixels);
                a.film = a.buffers.alloc<float>(3 * a.pixels);
            } catch (const crh::Error& e) {
                a.buffers.release();
                cudaGetLastError();
                if (!active_.empty()) return;  // retry when running jobs have freed memory
                popPending();
                endJob(j, a.ticket, CR_ERR_OUT_OF_MEMORY, e.what());
                continue;
            }
            popPending();
            a.slot = freeSlots_.back();
            freeSlots_.pop_back();
            hScenes_[a.slot] = j->scene->dev;
            hScenes_[a.slot].conductor_class = 1;  // the pool runs the conductor shading kernel
            hParams_[a.slot] = a.P;
            CR_CUDA(cudaMemsetAsync(a.acc, 0, 3 * a.pixels * sizeof(double), s_));
            CR_CUDA(cudaMemcpyAsync(scenes_ + a.slot, &hScenes_[a.slot], sizeof(DevScene), cudaMemcpyHostToDevice, s_));
            CR_CUDA(cudaMemcpyAsync(params_ + a.slot, &hParams_[a.slot], sizeof(RenderParams), cudaMemcpyHostToDevice, s_));
            CR_CUDA(cudaMemsetAsync(errKeys_ + a.slot, 0xff, sizeof(unsigned long long), s_));
            CR_CUDA(cudaMemsetAsync(retries_ + a.slot, 0, sizeof(unsigned long long), s_));
            usedBytes_ += a.bytes;
            a.admitStep = stepCount_;
            j->started_at = now();
            active_.push_back(std::move(a));
            std::lock_guard<std::mutex> lock(mutex_);
            stats_host_.peak_jobs = std::max<uint32_t>(stats_host_.peak_jobs, static_cast<uint32_t>(active_.size()));
        }
    }

    void popPending() {
        std::lock_guard<std::mutex> lock(mutex_);
        pending_.pop_front();
    }

    void issue() {
        // With nothing in flight the issue list starts over (positions, ranges, counters). The
        // counters still in flight describe the old list: they are taken first, and the test
        // made again on them.
        if (openRanges_ == 0 && live_ == 0 && rangeCount_ > 0 && pollPending_) {
            processPoll(mirror_ ^ 1);
            complete();
            pollPending_ = false;
        }
        if (openRanges_ == 0 && live_ == 0 && rangeCount_ > 0) {
            CR_CUDA(cudaMemsetAsync(done_, 0, rangeCount_ * sizeof(unsigned long long), s_));
            CR_CUDA(cudaMemsetAsync(ctl_ + 2, 0, 2 * sizeof(unsigned long long), s_));
            rangeCount_ = 0;
            uploaded_ = 0;
            issueEnd_ = 0;
            issuedPos_ = 0;
            firstOpen_ = 0;
            closed_.clear();
        }
        // Next range: policy 1 feeds the earliest admitted job to its end before the next, so the
        // pool's paths stay on few scenes (their BVHs stay in cache); policy 2 feeds the job with
        // the fewest samples per pixel issued (ties: the earliest admitted), so a job that just
        // arrived gets its first frame's samples ahead of the later frames of running jobs.
        while (issueEnd_ - issuedPos_ < cfg_.pool && rangeCount_ < kMaxRanges) {
            Active* best = nullptr;
            for (auto& a : active_) {
                if (a.failed || a.issued >= a.total) continue;
                if (cfg_.policy == 1) { best = &a; break; }  // the earliest admitted job with samples left
                // a.issued / a.pixels < best->issued / best->pixels, without division
                if (!best || static_cast<long double>(a.issued) * best->pixels <
                                 static_cast<long double>(best->issued) * a.pixels)
                    best = &a;
            }
            if (!best) return;
            Active& a = *best;
            uint64_t n = std::min<uint64_t>(cfg_.rangeSamples, a.total - a.issued);
            if (a.frameSamples) n = std::min<uint64_t>(n, (a.issued / a.frameSamples + 1) * a.frameSamples - a.issued);
            // Ranges are issued pixel-major, so a warp's paths start samples of one pixel (as in a
            // single render's chunks). A job without progressive frames whose samples per pixel
            // fit a range is cut into blocks of pixels that each range holds every sample of (a
            // warp: min(32, spp) samples of one pixel); otherwise into whole samples of every
            // pixel where a range holds at least one.
            uint32_t spp = 0, s0 = 0, p0 = 0;
            const uint64_t perPixel = a.total / a.pixels;
            if (!a.frameSamples && perPixel <= cfg_.rangeSamples && a.pixels <= UINT32_MAX && a.issued % perPixel == 0) {
                const uint64_t first = a.issued / perPixel;
                const uint64_t count = std::min<uint64_t>(std::max<uint64_t>(1, cfg_.rangeSamples / perPixel), a.pixels - first);
                n = count * perPixel;
                spp = static_cast<uint32_t>(perPixel);
                p0 = static_cast<uint32_t>(first);
            } else if (a.pixels <= n && a.issued % a.pixels == 0) {
                n = n / a.pixels * a.pixels;
                spp = static_cast<uint32_t>(n / a.pixels);
                s0 = static_cast<uint32_t>(a.issued / a.pixels);
            }
            uint64_t at = 0;
            if (!arena_.take(n, at)) return;
            IssueRange& R = hRanges_[rangeCount_];
            R.start = issueEnd_;
            R.c0 = a.issued;
            R.c1 = a.issued + n;
            R.outBase = at;
            R.pixels = a.pixels;
            R.job = a.slot;
            R.spp = spp;
            R.s0 = s0;
            R.p0 = p0;
            a.ranges.push_back(rangeCount_);
            closed_.push_back(false);
            ++a.chunks;
            ++rangeCount_;
            ++openRanges_;
            issueEnd_ += n;
            a.issued += n;
        }
    }

    void run() {
        if (rangeCount_ > uploaded_) {
            CR_CUDA(cudaMemcpyAsync(ranges_ + uploaded_, hRanges_ + uploaded_, (rangeCount_ - uploaded_) * sizeof(IssueRange),
                                    cudaMemcpyHostToDevice, s_));
            uploaded_ = rangeCount_;
        }
        // The staging words alternate with the mirrors: the copy queued two steps ago has run
        // (its step's counters were waited for), the one queued last step may not have.
        unsigned long long* stage = hCtl_ + 2 * mirror_;
        stage[0] = issueEnd_;
        stage[1] = rangeCount_;
        CR_CUDA(cudaMemcpyAsync(ctl_, stage, 2 * sizeof(unsigned long long), cudaMemcpyHostToDevice, s_));
        // Kernel variant: without the alpha test when no active job's scene has alpha-masked
        // triangles, lean shading when none has textures, punctual lights or alpha masks (a job's
        // paths leave the pool before it ends, so only active jobs' paths are traced or shaded).
        bool noAlpha = true, lean = true;
        for (const Active& a : active_) {
            const DevScene& S = a.job->scene->dev;
            noAlpha = noAlpha && !S.any_alpha_mask;
            lean = lean && !S.any_alpha_mask && S.texture_count == 0 && S.punctual_count == 0;
        }
        const int variant = (noAlpha ? 1 : 0) | (lean ? 2 : 0);
        if (cfg_.graphs) {
            if (!graph_[variant]) {
                cudaGraph_t g = nullptr;
                CR_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
                launchIterations(variant);
                CR_CUDA(cudaStreamEndCapture(s_, &g));
                CR_CUDA(cudaGraphInstantiate(&graph_[variant], g, 0));
                cudaGraphDestroy(g);
            }
            CR_CUDA(cudaGraphLaunch(graph_[variant], s_));
            std::lock_guard<std::mutex> lock(mutex_);
            ++stats_host_.graph_steps;
        } else {
            launchIterations(variant);
        }
        std::lock_guard<std::mutex> lock(mutex_);
        stats_host_.iterations += cfg_.iters;
        stats_host_.launches += 6ull * cfg_.iters;
    }

    template <int BLOCK>
    void setGrids() {
        gridTrace_ = occupancyGrid(reinterpret_cast<const void*>(k_trace<false, true, false, BLOCK>), BLOCK, device_);
        gridShade_ = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeGeneric, true, false, false, BLOCK>), BLOCK, device_);
        gridLight_ = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeNeeNull, true, false, false, BLOCK>), BLOCK, device_);
        gridMiss_ = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeMiss, true, false, false, BLOCK>), BLOCK, device_);
        gridCond_ = occupancyGrid(reinterpret_cast<const void*>(k_shade<kShadeConductor, true, false, false, BLOCK>), BLOCK, device_);
    }

    void launchIterations(int variant) {
        switch (cfg_.block) {
            case 64: launchVariant<64>(variant); break;
            case 256: launchVariant<256>(variant); break;
            default: launchVariant<128>(variant); break;
        }
    }
    template <int BLOCK>
    void launchVariant(int variant) {
        switch (variant) {
            case 0: launchIterationsT<false, false, BLOCK>(); break;
            case 1: launchIterationsT<true, false, BLOCK>(); break;
            default: launchIterationsT<true, true, BLOCK>(); break;  // lean implies no alpha masks
        }
    }

    template <bool NOALPHA, bool LEAN, int BLOCK>
    void launchIterationsT() {
        const DevScene S{};
        const RenderParams P{};
        const Chunk C{};
        const ErrSink E{};
        for (uint32_t i = 0; i < cfg_.iters; ++i) {
            const int cur = static_cast<int>(i & 1);
            const int refill = (i % cfg_.refill) == 0;
            k_regen<true><<<gridRegen_, 128, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_, refill);
            k_trace<false, true, NOALPHA, BLOCK><<<gridTrace_, BLOCK, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_);
            k_shade<kShadeMiss, true, false, LEAN, BLOCK><<<gridMiss_, BLOCK, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_);
            k_shade<kShadeNeeNull, true, false, LEAN, BLOCK><<<gridLight_, BLOCK, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_);
            k_shade<kShadeConductor, true, false, LEAN, BLOCK><<<gridCond_, BLOCK, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_);
            k_shade<kShadeGeneric, true, false, LEAN, BLOCK><<<gridShade_, BLOCK, 0, s_>>>(S, P, st_, q_, cur, C, E, stats_, J_);
        }
        CR_CUDA(cudaGetLastError());
    }

    // Copies the counters the queued graph leaves into mirror m (behind it on the stream).
    void enqueuePoll(int m) {
        Mirror& M = mirrors_[m];
        CR_CUDA(cudaMemcpyAsync(M.counts, q_.counts, kCountWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaMemcpyAsync(&M.ctl[2], ctl_ + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s_));
        M.first = firstOpen_;
        M.count = rangeCount_;
        M.step = stepCount_;
        if (rangeCount_ > firstOpen_)
            CR_CUDA(cudaMemcpyAsync(M.done + firstOpen_, done_ + firstOpen_, (rangeCount_ - firstOpen_) * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaMemcpyAsync(M.err, errKeys_, kMaxJobSlots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaMemcpyAsync(M.stats, stats_, kStatWords * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaEventRecord(M.ready, s_));
    }
    // Waits for mirror m and takes its counters as the engine's view of the pool.
    void processPoll(int m) {
        Mirror& M = mirrors_[m];
        CR_CUDA(cudaEventSynchronize(M.ready));
        CR_CUDA(cudaGetLastError());
        // every step ends at parity 0: the next iteration's live queue and last shadow queue
        live_ = static_cast<uint64_t>(M.counts[kCountExtend0]) + M.counts[kCountShadow1];
        issuedPos_ = M.ctl[2];  // issued[1], written by the step's last k_regen
        hDone_ = M.done;
        hErr_ = M.err;
        polledRanges_ = M.count;  // ranges issued after the copy have no count in this mirror
        polledStep_ = M.step;     // jobs admitted after it have no error key in this mirror
        std::lock_guard<std::mutex> lock(mutex_);
        stats_host_.extend_rays = M.stats[kStatExtendRays];
        stats_host_.shadow_rays = M.stats[kStatShadowRays];
    }
    // Completes the step whose counters are still in flight (the pool is going idle).
    void drainPoll() {
        if (!pollPending_) return;
        processPoll(mirror_ ^ 1);
        complete();
        pollPending_ = false;
    }

    void complete() {
        for (size_t k = 0; k < active_.size();) {
            Active& a = active_[k];
            if (!a.failed && polledStep_ >= a.admitStep && hErr_[a.slot] != kNoKey) {
                a.failed = true;
                a.errKey = hErr_[a.slot];
            }
            while (!a.ranges.empty()) {
                const uint32_t r = a.ranges.front();
                const IssueRange& R = hRanges_[r];
                if (r >= polledRanges_ || hDone_[r] < R.c1 - R.c0) break;
                if (!a.failed) {
                    k_accumulate<<<gridSmall_, 128, 0, s_>>>(st_.out + R.outBase, rangeChunk(R), a.acc);
                    CR_CUDA(cudaGetLastError());
                }
                arena_.give(R.outBase, R.c1 - R.c0);  // reused only by launches after this one
                a.accumulated = R.c1;
                a.ranges.pop_front();
                closed_[r] = true;
                --openRanges_;
                if (!a.failed && a.frameSamples && (a.accumulated % a.frameSamples == 0 || a.accumulated == a.total))
                    emitFrame(a);
            }
            while (firstOpen_ < rangeCount_ && closed_[firstOpen_]) ++firstOpen_;
            bool ended = false;
            if (a.failed && a.ranges.empty()) {
                finishFailed(a);
                ended = true;
            } else if (!a.failed && a.accumulated == a.total) {
                finishOk(a);
                ended = true;
            }
            if (ended) {
                a.buffers.release();
                usedBytes_ -= a.bytes;
                freeSlots_.push_back(a.slot);
                active_.erase(active_.begin() + static_cast<std::ptrdiff_t>(k));
            } else {
                ++k;
            }
        }
    }

    void emitFrame(Active& a) {
        const uint32_t spp = static_cast<uint32_t>(a.accumulated / a.pixels);
        k_film<<<gridSmall_, 128, 0, s_>>>(a.acc, a.film, a.pixels, static_cast<int>(spp));
        CR_CUDA(cudaGetLastError());
        const uint64_t size = crg::encode_film(a.film, a.job->options.width, a.job->options.height, a.job->format,
                                               a.job->exposure, s_, a.frame.data(), a.frame.size());
        if (size > a.frame.size()) throw crh::Error(CR_ERR_CUDA, "progressive frame larger than its bound");
        if (!a.job->first_frame_at) a.job->first_frame_at = now();
        if (a.job->on_frame) a.job->on_frame(spp, a.frame.data(), size, a.job->user);
    }

    void fillStats(Active& a) {
        cr_render_stats& st = a.job->stats;
        std::memset(&st, 0, sizeof(st));
        unsigned long long retries = 0;
        CR_CUDA(cudaMemcpyAsync(&retries, retries_ + a.slot, sizeof(retries), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaStreamSynchronize(s_));
        st.seconds = now() - a.job->started_at;
        st.workers = referenceWorkers(a.job->options);
        st.chunks = a.chunks;
        st.camera_samples = a.total;
        st.boundary_retries = retries;
    }

    void finishOk(Active& a) {
        if (!a.frameSamples) {
            k_film<<<gridSmall_, 128, 0, s_>>>(a.acc, a.film, a.pixels, a.job->options.samples);
            CR_CUDA(cudaGetLastError());
        }
        if (a.job->film_rgb)
            CR_CUDA(cudaMemcpyAsync(a.job->film_rgb, a.film, 3 * a.pixels * sizeof(float), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaStreamSynchronize(s_));
        fillStats(a);
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stats_host_.camera_samples += a.total;
        }
        endJob(a.job, a.ticket, CR_OK, "");
    }

    // The smallest failing key seen, re-run alone for the reference's message (render.cpp:437-438).
    void finishFailed(Active& a) {
        const cr_render_options& o = a.job->options;
        const unsigned long long key = a.errKey;
        const uint32_t sample = static_cast<uint32_t>(key & ((1ull << 21) - 1));
        const uint64_t rank = key >> 21;
        const uint64_t tilesX = (static_cast<uint64_t>(o.width) + 15) / 16;
        const uint64_t tile = rank / 256, within = rank % 256;
        const uint32_t x = static_cast<uint32_t>((tile % tilesX) * 16 + within % 16);
        const uint32_t y = static_cast<uint32_t>((tile / tilesX) * 16 + within / 16);
        DevError host{};
        CR_CUDA(cudaMemsetAsync(oneDetail_, 0, sizeof(DevError), s_));
        CR_CUDA(cudaMemsetAsync(oneStats_, 0, 2 * sizeof(unsigned long long), s_));
        k_trace_one<<<1, 32, 0, s_>>>(a.job->scene->dev, a.P, one_, y * static_cast<uint32_t>(o.width) + x, sample, oneDetail_,
                                      oneStats_, oneStats_ + 1);
        CR_CUDA(cudaMemcpyAsync(&host, oneDetail_, sizeof(DevError), cudaMemcpyDeviceToHost, s_));
        CR_CUDA(cudaStreamSynchronize(s_));
        if (!host.code) {
            host.code = -1;
            host.x = static_cast<int32_t>(x);
            host.y = static_cast<int32_t>(y);
            host.sample = static_cast<int32_t>(sample);
        }
        fillStats(a);
        endJob(a.job, a.ticket, CR_ERR_RENDER, crh::sample_error_message(host));
    }

    int device_;
    EngineConfig cfg_;
    cudaStream_t s_ = nullptr;
    std::chrono::steady_clock::time_point start_;
    Arena arena_;
    DevAlloc pool_, scratchAlloc_;
    PathSoA st_{}, one_{};
    Queues q_{}, oneQ_{};
    uint2* slotOf_ = nullptr;
    unsigned long long* stats_ = nullptr;
    DevScene* scenes_ = nullptr;
    RenderParams* params_ = nullptr;
    unsigned long long *errKeys_ = nullptr, *retries_ = nullptr, *done_ = nullptr, *ctl_ = nullptr;
    IssueRange* ranges_ = nullptr;
    DevError* oneDetail_ = nullptr;
    unsigned long long* oneStats_ = nullptr;
    JobTable J_{};
    // pinned host memory: the issue list, control words, and two mirrors of the counters a
    // step leaves (hDone_ and hErr_ point into the mirror last processed)
    IssueRange* hRanges_ = nullptr;
    unsigned long long* hCtl_ = nullptr;
    struct Mirror {
        unsigned long long *done = nullptr, *ctl = nullptr, *err = nullptr, *stats = nullptr;
        uint32_t* counts = nullptr;
        uint32_t first = 0, count = 0;
        uint64_t step = 0;
        cudaEvent_t ready = nullptr;
    };
    Mirror mirrors_[2];
    int mirror_ = 0;
    bool pollPending_ = false;
    uint32_t polledRanges_ = 0;
    uint64_t stepCount_ = 0, polledStep_ = 0;
    const unsigned long long* hDone_ = nullptr;
    const unsigned long long* hErr_ = nullptr;
    std::vector<DevScene> hScenes_;
    std::vector<RenderParams> hParams_;
    int gridTrace_ = 0, gridShade_ = 0, gridLight_ = 0, gridMiss_ = 0, gridCond_ = 0, gridRegen_ = 0, gridSmall_ = 0;
    cudaGraphExec_t graph_[4] = {};  // one per kernel variant (bit 0: no alpha test, bit 1: lean shading)
    // issue list state
    uint32_t rangeCount_ = 0, uploaded_ = 0, firstOpen_ = 0;
    uint64_t openRanges_ = 0, issueEnd_ = 0, issuedPos_ = 0, live_ = 0;
    std::vector<bool> closed_;
    // jobs
    std::vector<Active> active_;
    std::vector<uint32_t> freeSlots_;
    uint64_t usedBytes_ = 0;
    // shared with submitters and waiters
    std::mutex mutex_;
    std::condition_variable cv_;
    std::deque<std::pair<cr_job*, uint64_t>> pending_;
    std::map<uint64_t, cr_status> ended_;
    uint64_t lastTicket_ = 0;
    cr_engine_stats stats_host_{};
    cr_engine_stats solo_{};  // rays of the jobs rendered alone (the pool's own come from the device)
    double busySeconds_ = 0;
};

}  // namespace

struct cr_server {
    std::unique_ptr<Engine> engine;
    std::thread thread;
    std::atomic<bool> stop{false};
    std::mutex errorMutex;
    std::string error;
};

namespace {

// Jobs of at least 2^22 samples (4 M: a 1024x1024 frame at 4 spp) fill the device on their own
// and render alone; on the 64-scene mix 2^22 measured 1.001x one by one, 2^24 0.985x, 2^20
// 0.985x (the pool's per-sample cost on large jobs against the single render's).
constexpr uint32_t kSoloSamplesLog2 = 22;

// Whether a batch job renders alone: its camera samples between two drains — the whole job, or
// one frame interval (every_samples x pixels) of a progressive job, since a progressive single
// render drains its paths at every frame — reach 2^soloLog2. Progressive jobs of 480x270 at 4
// spp per frame rendered alone ran 39.2 vs 49.0 Msamples/s in the pool (2,000-request stream).
bool rendersAlone(const cr_job& j, uint32_t soloLog2) {
    const cr_render_options& o = j.options;
    if (soloLog2 >= 64 || o.width <= 0 || o.height <= 0 || o.samples <= 0) return false;
    const uint64_t pixels = static_cast<uint64_t>(o.width) * static_cast<uint64_t>(o.height);
    uint64_t unit = pixels * static_cast<uint64_t>(o.samples);
    if (j.every_samples) unit = std::min(unit, pixels * j.every_samples);
    return unit >= (uint64_t{1} << soloLog2);
}

cr_status runBatch(cr_job* jobs, uint32_t count, const cr_engine_tuning* tuning, cr_engine_stats* stats) {
    if (count == 0) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return CR_OK;
    }
    if (!jobs) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "jobs is NULL");
    int device = -1;
    for (uint32_t i = 0; i < count; ++i)
        if (jobs[i].scene) { device = jobs[i].scene->device; break; }
    if (device < 0) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "no job has a scene");
    Engine e(device, tuning, 1);
    // Jobs that fill the device between two drains render alone, in order, on a helper thread
    // beside the pool, which takes the rest.
    const uint32_t soloLog2 = tuning && tuning->solo_samples_log2 ? tuning->solo_samples_log2 : kSoloSamplesLog2;
    const auto wall0 = std::chrono::steady_clock::now();
    std::vector<std::pair<cr_job*, uint64_t>> solo;
    for (uint32_t i = 0; i < count; ++i) {
        const cr_job& j = jobs[i];
        if (j.scene && j.scene->device == device && rendersAlone(j, soloLog2))
            solo.push_back({&jobs[i], e.registerSolo(&jobs[i])});
        else
            e.submit(&jobs[i]);
    }
    // The solo renders run on a helper thread (on their scenes' streams) while this thread steps
    // the pool (on the engine's stream): the pool's kernels fill the device when a solo render's
    // launches drain.
    std::exception_ptr soloError;
    std::thread soloThread([&] {
        try {
            CR_CUDA(cudaSetDevice(device));
            for (auto& [j, ticket] : solo) e.runSolo(j, ticket);
        } catch (...) {
            soloError = std::current_exception();
        }
    });
    struct Join {
        std::thread& t;
        ~Join() { if (t.joinable()) t.join(); }
    } join{soloThread};
    try {
        while (!e.idle()) e.step();
    } catch (const std::exception& ex) {
        e.failAll(CR_ERR_CUDA, ex.what());
        throw;
    }
    soloThread.join();
    if (soloError) std::rethrow_exception(soloError);
    if (stats) {
        *stats = e.stats();
        if (!solo.empty())  // the pool and the solo renders overlap: the batch's wall time
            stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    }
    for (uint32_t i = 0; i < count; ++i)
        if (jobs[i].status != CR_OK) return crh::set_last_error(jobs[i].status, jobs[i].error);
    return CR_OK;
}

}  // namespace

extern "C" {

cr_status cr_gpu_render_batch(cr_job* jobs, uint32_t count, const cr_engine_tuning* tuning, cr_engine_stats* stats) {
    try {
        return runBatch(jobs, count, tuning, stats);
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_gpu_autotune_batch(const cr_job* jobs, uint32_t count, cr_engine_tuning* tuning) {
    uint32_t n = 0;
    return cr_gpu_autotune_batch_trials(jobs, count, tuning, nullptr, 0, &n);
}

cr_status cr_gpu_autotune_batch_trials(const cr_job* jobs, uint32_t count, cr_engine_tuning* tuning,
                                       cr_autotune_trial* trials, uint32_t capacity, uint32_t* trialCount) {
    try {
        if (!jobs || !tuning || count == 0 || !trialCount || (capacity && !trials))
            return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        *trialCount = 0;
        // the jobs that will share the pool (larger ones render alone, see runBatch) at 1 spp
        const uint32_t soloLog2 = tuning->solo_samples_log2 ? tuning->solo_samples_log2 : kSoloSamplesLog2;
        std::vector<cr_job> trial;
        for (uint32_t i = 0; i < count; ++i)
            if (!(jobs[i].scene && rendersAlone(jobs[i], soloLog2))) trial.push_back(jobs[i]);
        if (trial.empty()) return CR_OK;
        for (auto& j : trial) {
            j.options.samples = 1;
            j.film_rgb = nullptr;
            j.every_samples = 0;
            j.on_frame = nullptr;
        }
        // one timed trial batch of the pool's jobs under t
        auto run = [&](cr_engine_tuning t) -> double {
            t.solo_samples_log2 = 64;  // the trial jobs are the pool's
            const auto t0 = std::chrono::steady_clock::now();
            const cr_status st = runBatch(trial.data(), static_cast<uint32_t>(trial.size()), &t, nullptr);
            const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (st != CR_OK) throw crh::Error(st, std::string("autotune trial: ") + crh::last_error_text());
            if (*trialCount < capacity)
                trials[*trialCount] = cr_autotune_trial{t.pool_paths, t.iterations_per_step, t.refill_free_percent,
                                                        t.block_size, sec};
            ++*trialCount;
            return sec;
        };
        cr_engine_tuning best = *tuning;
        if (!best.pool_paths) best.pool_paths = 1u << 24;
        if (!best.iterations_per_step) best.iterations_per_step = 8;
        if (!best.block_size) best.block_size = 128;
        best.refill_interval = 1;
        run(best);  // warm-up: scenes and device blocks touched once
        double bestSeconds = run(best);
        // one dimension after another, each keeping its fastest value
        auto sweep = [&](uint32_t cr_engine_tuning::*field, std::initializer_list<uint32_t> values) {
            for (uint32_t v : values) {
                if (best.*field == v) continue;
                cr_engine_tuning t = best;
                t.*field = v;
                const double sec = run(t);
                if (sec < bestSeconds) { bestSeconds = sec; best = t; }
            }
        };
        sweep(&cr_engine_tuning::pool_paths, {1u << 22, 1u << 23, 1u << 24, 1u << 25});
        sweep(&cr_engine_tuning::iterations_per_step, {8, 16, 32});
        sweep(&cr_engine_tuning::refill_free_percent, {0, 50, 90});
        sweep(&cr_engine_tuning::block_size, {64, 128, 256});
        best.solo_samples_log2 = tuning->solo_samples_log2;  // the trials ran the pool's jobs only
        *tuning = best;
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_server_create(int device, const cr_engine_tuning* tuning, cr_server** out) {
    try {
        if (!out) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        auto srv = std::make_unique<cr_server>();
        srv->engine = std::make_unique<Engine>(device, tuning, 2);
        cr_server* s = srv.get();
        s->thread = std::thread([s] {
            try {
                CR_CUDA(cudaSetDevice(s->engine->device()));
                for (;;) {
                    const bool busy = s->engine->step();
                    if (!busy) {
                        if (s->stop.load() && s->engine->idle()) break;
                        s->engine->waitForWork(s->stop);
                        if (s->stop.load() && s->engine->idle()) break;
                    }
                }
            } catch (const std::exception& e) {
                {
                    std::lock_guard<std::mutex> lock(s->errorMutex);
                    s->error = e.what();
                }
                s->engine->failAll(CR_ERR_CUDA, e.what());
            }
        });
        *out = srv.release();
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_server_submit(cr_server* s, cr_job* job, uint64_t* ticket) {
    try {
        if (!s || !job || !ticket) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        {
            std::lock_guard<std::mutex> lock(s->errorMutex);
            if (!s->error.empty()) return crh::set_last_error(CR_ERR_CUDA, "server stopped: " + s->error);
        }
        *ticket = s->engine->submit(job);
        return CR_OK;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_server_wait(cr_server* s, uint64_t ticket, double timeout_seconds) {
    try {
        if (!s) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
        const cr_status st = s->engine->wait(ticket, timeout_seconds);
        if (st == CR_ERR_DEVICE_TIMEOUT) return crh::set_last_error(st, "job still running");
        return st;
    } catch (const std::exception& e) { return fail(e); }
}

cr_status cr_server_stats(cr_server* s, cr_engine_stats* stats) {
    if (!s || !stats) return crh::set_last_error(CR_ERR_INVALID_ARGUMENT, "NULL argument");
    *stats = s->engine->stats();
    return CR_OK;
}

double cr_server_clock(cr_server* s) { return s ? s->engine->now() : 0.0; }

cr_status cr_server_destroy(cr_server* s) {
    if (!s) return CR_OK;
    s->stop.store(true);
    s->engine->wake();
    if (s->thread.joinable()) s->thread.join();
    delete s;
    return CR_OK;
}

}  // extern "C"
