// Job server (gpt_server_* in include/gpt_b200.h): continuous batching of render jobs over
// device-resident scenes.
//
// The reference renders one job at a time: Renderer::StartSimulation runs RenderFrame for each
// camera state on a worker thread (Renderer.cpp:401-466), and each frame is a host-driven loop over
// that one job's samples (Renderer.cpp:468-647). Here a scheduler thread owns one pool of path
// slots, a table of admitted jobs and the packed arrays of all resident scenes, and runs the
// wavefront in slices. A slice is one launch of a CUDA graph whose WHILE node repeats the
// job-engine iteration (trace, shade, shadow, plan, regenerate, fold, advance) until a job
// completes, a new job is waiting (the doorbell), nothing is left to do, or the slice's iteration
// cap is reached. Between slices the host retires finished jobs and admits waiting ones; the paths
// in flight stay on the device from one slice to the next, so admitted jobs overlap on the GPU.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <memory>
#include <cstddef>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "kernels.h"
#include "runtime.hpp"

namespace pt
{
    namespace
    {
        constexpr uint32_t kDefaultServerPool = 4u << 20;
        constexpr uint32_t kDefaultMaxJobs = 256;
        constexpr uint64_t kDefaultBudget = 16ull << 30;
        constexpr uint32_t kDefaultSliceIterations = 4096;
        constexpr uint64_t kPathStateBytes = 64;  // admission accounting per path a job may have in flight
        constexpr size_t kArenaAlign = 256;
        constexpr size_t kStagingBytes = 16u << 20;  // pinned staging for copying finished images out

        size_t align_up(size_t v) { return (v + kArenaAlign - 1) / kArenaAlign * kArenaAlign; }

        // First-fit allocator over one device allocation: admitting and retiring jobs makes no CUDA
        // allocator call (cudaFree would wait for the running slice).
        class Arena
        {
        public:
            Status init(size_t bytes)
            {
                PT_TRY(buffer_.allocate(bytes));
                free_.clear();
                free_[0] = bytes;
                return Status::Ok();
            }
            bool allocate(size_t bytes, size_t& offset)
            {
                bytes = align_up(bytes);
                for (auto it = free_.begin(); it != free_.end(); ++it)
                {
                    if (it->second < bytes) continue;
                    offset = it->first;
                    const size_t rest = it->second - bytes;
                    free_.erase(it);
                    if (rest) free_[offset + bytes] = rest;
                    return true;
                }
                return false;
            }
            void release(size_t offset, size_t bytes)
            {
                bytes = align_up(bytes);
                auto next = free_.lower_bound(offset);
                if (next != free_.end() && offset + bytes == next->first)
                {
                    bytes += next->second;
                    next = free_.erase(next);
                }
                if (next != free_.begin())
                {
                    auto prev = std::prev(next);
                    if (prev->first + prev->second == offset)
                    {
                        prev->second += bytes;
                        return;
                    }
                }
                free_[offset] = bytes;
            }
            char* base() const { return buffer_.get<char>(); }

        private:
            DeviceBuffer buffer_;
            std::map<size_t, size_t> free_;
        };

        // All resident scenes in one set of arrays. Node child references, triangle input indices,
        // material indices of triangles and lights, and alias entries of every appended scene are
        // rebased to the packed arrays, so traversal and shading index them without per-scene base
        // pointers; a ray only needs its scene's root node (SceneEntry).
        struct ScenePack
        {
            DeviceBuffer nodes, tris, shading, materials, textures, lights, bins, binsPower, entries;
            std::vector<SceneEntry> entry;
            std::vector<std::unique_ptr<TextureObject>> textureObjects;
            uint32_t nodeCount = 0, triangleCount = 0, materialCount = 0, lightCount = 0, depth = 0;
            bool modelPresent[kModelCount] = {};
            bool anyTextures = false;

            SceneView view() const
            {
                SceneView v{};
                v.nodes = nodes.get<Node8>();
                v.tris = tris.get<float4>();
                v.shading = shading.get<float4>();
                v.materials = materials.get<MaterialDev>();
                v.textures = anyTextures ? textures.get<MaterialTextures>() : nullptr;
                v.lights = lights.get<float4>();
                v.bins = bins.get<uint4>();
                v.binsPower = binsPower.get<uint4>();
                v.lightCount = lightCount;
                v.nodeCount = nodeCount;
                v.triangleCount = triangleCount;
                v.depth = depth;
                return v;
            }
        };

        Status Grow(DeviceBuffer& dst, const DeviceBuffer& old, size_t oldBytes, const DeviceBuffer& add, size_t addBytes, cudaStream_t st)
        {
            PT_TRY(dst.allocate(std::max<size_t>(oldBytes + addBytes, 16)));
            if (oldBytes) PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(dst.get<char>(), old.get<char>(), oldBytes, cudaMemcpyDeviceToDevice, st));
            if (addBytes)
                PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(dst.get<char>() + oldBytes, add.get<char>(), addBytes, cudaMemcpyDeviceToDevice, st));
            return Status::Ok();
        }

        Status AppendScene(ScenePack& p, SceneGpu& s, cudaStream_t st)
        {
            if (p.entry.size() >= kMaxScenes) return Status::Err(GPT_ERR_CAPACITY, "At most 256 resident scenes");
            if (static_cast<uint64_t>(p.nodeCount) + s.nodeCount >= (1ull << 24))
                return Status::Err(GPT_ERR_CAPACITY, "Resident scenes exceed 2^24 BVH8 nodes");
            if (static_cast<uint64_t>(p.triangleCount) + s.triangleCount > kMaxTriangles)
                return Status::Err(GPT_ERR_CAPACITY, "Resident scenes exceed 2^24 triangles");
            DeviceBuffer nn, nt, ns, nm, nl, nb, nbp, ntex, ne;
            PT_TRY(Grow(nn, p.nodes, size_t(p.nodeCount) * sizeof(Node8), s.nodes, size_t(s.nodeCount) * sizeof(Node8), st));
            PT_TRY(Grow(nt, p.tris, size_t(p.triangleCount) * kTriangleVec4 * 16, s.tris, size_t(s.triangleCount) * kTriangleVec4 * 16, st));
            PT_TRY(Grow(ns, p.shading, size_t(p.triangleCount) * 144, s.shading, size_t(s.triangleCount) * 144, st));
            PT_TRY(Grow(nm, p.materials, size_t(p.materialCount) * sizeof(MaterialDev), s.materials, size_t(s.materialCount) * sizeof(MaterialDev), st));
            PT_TRY(Grow(nl, p.lights, size_t(p.lightCount) * 112, s.lights, size_t(s.lightCount) * 112, st));
            PT_TRY(Grow(nb, p.bins, size_t(p.lightCount) * 16, s.bins, size_t(s.lightCount) * 16, st));
            PT_TRY(Grow(nbp, p.binsPower, size_t(p.lightCount) * 16, s.binsPower, size_t(s.lightCount) * 16, st));
            PT_CUDA("rebase nodes", launch_rebase_nodes(nn.get<Node8>() + p.nodeCount, s.nodeCount, p.nodeCount, p.triangleCount, st));
            uint32_t* triWords = reinterpret_cast<uint32_t*>(nt.get<float4>() + size_t(p.triangleCount) * kTriangleVec4);
            PT_CUDA("rebase triangles", launch_rebase_field(triWords + 3, s.triangleCount, kTriangleVec4 * 4, p.triangleCount, false, st));
            uint32_t* shadeWords = reinterpret_cast<uint32_t*>(ns.get<float4>() + size_t(p.triangleCount) * 9);
            PT_CUDA("rebase shading", launch_rebase_field(shadeWords + 27, s.triangleCount, 36, p.materialCount, false, st));
            uint32_t* lightWords = reinterpret_cast<uint32_t*>(nl.get<float4>() + size_t(p.lightCount) * 7);
            PT_CUDA("rebase lights", launch_rebase_field(lightWords + 3, s.lightCount, 28, p.triangleCount, false, st));
            PT_CUDA("rebase lights", launch_rebase_field(lightWords + 26, s.lightCount, 28, p.materialCount, false, st));
            uint32_t* binWords = reinterpret_cast<uint32_t*>(nb.get<uint4>() + p.lightCount);
            PT_CUDA("rebase alias table", launch_rebase_field(binWords + 2, s.lightCount, 4, p.lightCount, true, st));
            uint32_t* powerWords = reinterpret_cast<uint32_t*>(nbp.get<uint4>() + p.lightCount);
            PT_CUDA("rebase alias table", launch_rebase_field(powerWords + 2, s.lightCount, 4, p.lightCount, true, st));
            const bool sceneTextures = !s.textures.empty();
            const bool anyTextures = p.anyTextures || sceneTextures;
            if (anyTextures)
            {
                const size_t oldBytes = size_t(p.materialCount) * sizeof(MaterialTextures);
                const size_t addBytes = size_t(s.materialCount) * sizeof(MaterialTextures);
                PT_TRY(ntex.allocate(oldBytes + addBytes));
                if (p.anyTextures && oldBytes)
                    PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(ntex.get<char>(), p.textures.get<char>(), oldBytes, cudaMemcpyDeviceToDevice, st));
                else if (oldBytes)
                    PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(ntex.get<char>(), 0, oldBytes, st));
                if (sceneTextures)
                    PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(ntex.get<char>() + oldBytes, s.materialTextures.get<char>(), addBytes, cudaMemcpyDeviceToDevice, st));
                else
                    PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(ntex.get<char>() + oldBytes, 0, addBytes, st));
            }
            std::vector<SceneEntry> entries = p.entry;
            entries.push_back(SceneEntry{p.nodeCount, p.lightCount, s.lightCount, p.triangleCount});
            PT_TRY(ne.allocate(entries.size() * sizeof(SceneEntry)));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(ne.get<void>(), entries.data(), entries.size() * sizeof(SceneEntry), cudaMemcpyHostToDevice, st));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(st));
            p.nodes.swap(nn);
            p.tris.swap(nt);
            p.shading.swap(ns);
            p.materials.swap(nm);
            p.lights.swap(nl);
            p.bins.swap(nb);
            p.binsPower.swap(nbp);
            if (anyTextures) p.textures.swap(ntex);
            p.entries.swap(ne);
            p.entry = std::move(entries);
            p.nodeCount += s.nodeCount;
            p.triangleCount += s.triangleCount;
            p.materialCount += s.materialCount;
            p.lightCount += s.lightCount;
            p.depth = std::max(p.depth, s.depth);
            for (uint32_t m = 0; m < kModelCount; m++) p.modelPresent[m] = p.modelPresent[m] || s.modelPresent[m];
            p.anyTextures = anyTextures;
            for (auto& t : s.textures) p.textureObjects.push_back(std::move(t));
            s.textures.clear();
            return Status::Ok();
        }

        double seconds_since(std::chrono::steady_clock::time_point t0)
        {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
    }

    struct JobRecord
    {
        uint64_t id = 0;
        gpt_job_desc desc{};
        uint32_t state = GPT_JOB_QUEUED;
        uint32_t tableIndex = kInvalid;
        JobView view{};
        uint32_t pixels = 0, spp = 1, spa = 1, ring = 1, passesDone = 0;
        size_t ringBytes = 0, accumBytes = 0, fbBytes = 0, doneBytes = 0, arenaBytes = 0, arenaOffset = 0;
        uint64_t admittedBytes = 0;
        double tSubmit = -1.0, tAdmit = -1.0, tDone = -1.0;
        bool cancelRequested = false, cancelApplied = false;
        // Shared so that a read copies the image outside the server's lock while a release may drop the record.
        std::shared_ptr<std::vector<uint32_t>> rgba;
        std::shared_ptr<std::vector<float>> accumulation;
    };

    class Server
    {
    public:
        Server(int device, const gpt_server_config& c) : device_(device), cfg_(c)
        {
            if (!cfg_.pool_size) cfg_.pool_size = kDefaultServerPool;
            cfg_.pool_size = std::min(cfg_.pool_size, kMaxPool);
            if (!cfg_.max_jobs) cfg_.max_jobs = kDefaultMaxJobs;
            cfg_.max_jobs = std::min(cfg_.max_jobs, kMaxJobs);
            if (!cfg_.hbm_budget_bytes) cfg_.hbm_budget_bytes = kDefaultBudget;
            if (!cfg_.max_slice_iterations) cfg_.max_slice_iterations = kDefaultSliceIterations;
            cfg_.ring_passes = std::min(cfg_.ring_passes, kMaxRing);
            threads_ = cfg_.trace_block == 64 ? 64 : 128;
            refill_ = (cfg_.trace_refill & 0xFFu) ? std::min(32u, std::max(1u, cfg_.trace_refill & 0xFFu)) : 16u;
            refillShadow_ = ((cfg_.trace_refill >> 8) & 0xFFu) ? std::min(32u, std::max(1u, (cfg_.trace_refill >> 8) & 0xFFu))
                                                                : std::max(1u, refill_ / 2u);
            occupancy_ = cfg_.trace_occupancy == 0 ? 10 : (cfg_.trace_occupancy >= 12 ? 12 : (cfg_.trace_occupancy >= 10 ? 10 : 1));
            schedule_ = cfg_.schedule == 0 ? GPT_SCHEDULE_TWO_CLASS : cfg_.schedule;
            if (!(cfg_.deadline_slowdown > 0.0f)) cfg_.deadline_slowdown = 4.0f;
            if (!(cfg_.short_job_seconds > 0.0f)) cfg_.short_job_seconds = 0.05f;
            t0_ = std::chrono::steady_clock::now();
        }

        ~Server()
        {
            {
                std::scoped_lock lock(mu_);
                stop_ = true;
                if (hostMapped_) *static_cast<volatile uint32_t*>(hostMapped_) = 1u;
            }
            cv_.notify_all();
            if (worker_.joinable()) worker_.join();
            if (graphExec_) cudaGraphExecDestroy(graphExec_);
            if (graph_) cudaGraphDestroy(graph_);
            if (startEvent_) cudaEventDestroy(startEvent_);
            if (stopEvent_) cudaEventDestroy(stopEvent_);
            if (pinned_) cudaFreeHost(pinned_);
            if (staging_) cudaFreeHost(staging_);
            if (hostMapped_) cudaFreeHost(hostMapped_);
            if (copyStream_) cudaStreamDestroy(copyStream_);
            if (shadeFork_) cudaEventDestroy(shadeFork_);
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                if (shadeJoin_[m]) cudaEventDestroy(shadeJoin_[m]);
                if (shadeStreams_[m]) cudaStreamDestroy(shadeStreams_[m]);
            }
            if (stream_) cudaStreamDestroy(stream_);
        }

        Status Init()
        {
            if (cfg_.schedule > GPT_SCHEDULE_TWO_CLASS) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown schedule");
            if (cfg_.bvh_build > GPT_BVH_BUILD_DEVICE) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown BVH build");
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            PT_CUDA("cudaStreamCreateWithFlags", cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
            PT_CUDA("cudaStreamCreateWithFlags", cudaStreamCreateWithFlags(&copyStream_, cudaStreamNonBlocking));
            PT_CUDA("cudaEventCreateWithFlags", cudaEventCreateWithFlags(&shadeFork_, cudaEventDisableTiming));
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                PT_CUDA("cudaStreamCreateWithFlags", cudaStreamCreateWithFlags(&shadeStreams_[m], cudaStreamNonBlocking));
                PT_CUDA("cudaEventCreateWithFlags", cudaEventCreateWithFlags(&shadeJoin_[m], cudaEventDisableTiming));
            }
            PT_CUDA("cudaHostAlloc", cudaHostAlloc(&staging_, kStagingBytes, cudaHostAllocDefault));
            PT_CUDA("cudaEventCreate", cudaEventCreate(&startEvent_));
            PT_CUDA("cudaEventCreate", cudaEventCreate(&stopEvent_));
            PT_CUDA("cudaHostAlloc", cudaHostAlloc(&hostMapped_, 64, cudaHostAllocMapped));
            std::memset(hostMapped_, 0, 64);
            PT_CUDA("cudaHostGetDevicePointer", cudaHostGetDevicePointer(&hostMappedDev_, hostMapped_, 0));
            const size_t P = cfg_.pool_size;
            for (int q = 0; q < 2; q++)
            {
                PT_TRY(rayO_[q].allocate(P * 16));
                PT_TRY(rayD_[q].allocate(P * 16));
            }
            PT_TRY(matQ_.allocate(P * 48 * kModelCount));
            PT_TRY(shO_.allocate(P * 16));
            PT_TRY(shD_.allocate(P * 16));
            PT_TRY(shL_.allocate(P * 16));
            PT_TRY(regenBits_.allocate((P + 31) / 32 * 4));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(regenBits_.get<void>(), 0, (P + 31) / 32 * 4, stream_));
            PT_TRY(slotT_.allocate(P * 16));
            PT_TRY(slotL_.allocate(P * 16));
            PT_TRY(slotSample_.allocate(P * 4));
            PT_TRY(freeList_.allocate(P * 4));
            PT_TRY(counters_.allocate(sizeof(Counters)));
            PT_TRY(ctl_.allocate(sizeof(EngineCtl)));
            PT_TRY(jobs_.allocate(size_t(cfg_.max_jobs) * sizeof(JobView)));
            PT_TRY(order_.allocate(size_t(cfg_.max_jobs) * 4));
            PT_TRY(segments_.allocate(size_t(cfg_.max_jobs) * sizeof(LaunchSegment)));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(jobs_.get<void>(), 0, size_t(cfg_.max_jobs) * sizeof(JobView), stream_));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(ctl_.get<void>(), 0, sizeof(EngineCtl), stream_));
            // pinned staging: counters, engine control, job table mirror, order list, slice words
            pinnedBytes_ = sizeof(Counters) + sizeof(EngineCtl) + size_t(cfg_.max_jobs) * (sizeof(JobView) + 4) + 16;
            PT_CUDA("cudaHostAlloc", cudaHostAlloc(&pinned_, pinnedBytes_, cudaHostAllocDefault));
            std::memset(pinned_, 0, pinnedBytes_);
            hostCounters_ = static_cast<Counters*>(pinned_);
            hostCtl_ = reinterpret_cast<EngineCtl*>(hostCounters_ + 1);
            mirror_ = reinterpret_cast<JobView*>(hostCtl_ + 1);
            orderHost_ = reinterpret_cast<uint32_t*>(mirror_ + cfg_.max_jobs);
            sliceWords_ = orderHost_ + cfg_.max_jobs;
            PT_TRY(arena_.init(cfg_.hbm_budget_bytes));
            PT_CUDA("engine init", launch_engine_init(wavefront(), engineView(), cfg_.pool_size, stream_));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
            for (uint32_t i = cfg_.max_jobs; i-- > 0;) freeTable_.push_back(i);
            worker_ = std::thread([this] { Run(); });
            return Status::Ok();
        }

        // ---------------------------------------------------------------- scenes
        Status AddScene(const gpt_scene_desc& d, uint32_t& id)
        {
            std::scoped_lock lock(mu_);
            if (!pending_.empty() || !active_.empty()) return Status::Err(GPT_ERR_STATE, "Scenes are added while no job is queued or running");
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            std::unique_ptr<SceneGpu> scene;
            PT_TRY(BuildScene(d, stream_, scene, false, cfg_.bvh_build == GPT_BVH_BUILD_DEVICE));
            PT_TRY(AppendScene(pack_, *scene, stream_));
            releaseGraph();
            id = static_cast<uint32_t>(pack_.entry.size() - 1);
            return Status::Ok();
        }

        // ---------------------------------------------------------------- jobs
        Status Submit(const gpt_job_desc& d, uint64_t& id)
        {
            std::scoped_lock lock(mu_);
            if (d.scene >= pack_.entry.size()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown scene id");
            if (d.rng_policy != GPT_RNG_PHILOX && d.rng_policy != GPT_RNG_PCG32) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown rng_policy");
            if (d.light_sampling != GPT_LIGHTS_AREA && d.light_sampling != GPT_LIGHTS_POWER)
                return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown light_sampling");
            JobRecord J;
            J.desc = d;
            // clamps of StartSimulation (Renderer.cpp:340-344, 366-367)
            const uint32_t w = std::min(std::max(d.width, 1u), 7680u);
            const uint32_t h = std::min(std::max(d.height, 1u), 4320u);
            J.desc.width = w;
            J.desc.height = h;
            J.pixels = w * h;
            const uint32_t spp = std::min(std::max(d.samples_per_pixel, 1u), 10'000'000u);
            J.spa = static_cast<uint32_t>(std::sqrt(static_cast<double>(spp)));
            J.spp = J.spa * J.spa;
            const uint64_t total = uint64_t(J.spp) * J.pixels;
            if (total >= 0xFFFFFFFFull) return Status::Err(GPT_ERR_CAPACITY, "A job is limited to 2^32-1 samples");
            uint32_t ring = cfg_.ring_passes;
            if (ring == 0)
            {
                // four pool-fulls of passes: a window this deep rarely waits on the oldest pass's longest paths
                const uint64_t fill = (4ull * cfg_.pool_size + J.pixels - 1) / J.pixels;
                ring = static_cast<uint32_t>(std::min<uint64_t>(std::max<uint64_t>(fill, 2), kMaxRing));
            }
            J.ring = std::min(ring, J.spp);
            J.ringBytes = align_up(size_t(J.ring) * J.pixels * 12);
            J.accumBytes = align_up(size_t(J.pixels) * 32);
            J.fbBytes = align_up(size_t(J.pixels) * 4);
            J.doneBytes = align_up(size_t(J.ring) * 4);
            J.arenaBytes = J.ringBytes + J.accumBytes + J.fbBytes + J.doneBytes;
            const uint64_t inflight = std::min<uint64_t>(uint64_t(J.ring) * J.pixels, cfg_.pool_size);
            J.admittedBytes = kPathStateBytes * inflight + J.arenaBytes;
            if (J.admittedBytes > cfg_.hbm_budget_bytes)
                return Status::Err(GPT_ERR_CAPACITY, "Job needs " + std::to_string(J.admittedBytes) + " bytes, above the HBM budget");
            J.id = nextId_++;
            J.tSubmit = seconds_since(t0_);
            id = J.id;
            // End the running slice only when the new job can be admitted now: jobs are admitted in
            // submission order (per class under the two-class order), so behind a waiting job of its
            // class, or with the budget, the job table or the active-job limit full, a new slice could not
            // start it (a completing job ends the slice and admits waiting jobs anyway). Under overload
            // this keeps arrivals from cutting slices short.
            bool waitingAhead = false;  // a waiting job that would be admitted first
            for (uint64_t pid : pending_)
                if (admission_class(records_[pid]) == admission_class(J))
                {
                    waitingAhead = true;
                    break;
                }
            const bool admittable = !waitingAhead && fits_budget(J) && !freeTable_.empty() &&
                                    (cfg_.max_active_jobs == 0 || active_.size() + toCopy_.size() < cfg_.max_active_jobs);
            records_.emplace(J.id, std::move(J));
            pending_.push_back(id);
            if (admittable) *static_cast<volatile uint32_t*>(hostMapped_) = 1u;
            cv_.notify_all();
            return Status::Ok();
        }

        Status Poll(uint64_t id, gpt_job_status& st)
        {
            std::scoped_lock lock(mu_);
            auto it = records_.find(id);
            if (it == records_.end()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown job id");
            const JobRecord& J = it->second;
            st = gpt_job_status{};
            st.state = J.state;
            st.passes_done = J.passesDone;
            st.passes_total = J.spp;
            st.samples_total = uint64_t(J.spp) * J.pixels;
            st.admitted_bytes = J.admittedBytes;
            st.submit_s = J.tSubmit;
            st.admit_s = J.tAdmit;
            st.done_s = J.tDone;
            return Status::Ok();
        }

        Status Wait(uint64_t id, double timeout)
        {
            std::unique_lock<std::mutex> lock(mu_);
            auto finished = [&]
            {
                auto it = records_.find(id);
                return it == records_.end() || it->second.state >= GPT_JOB_DONE;
            };
            if (records_.find(id) == records_.end()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown job id");
            if (!doneCv_.wait_for(lock, std::chrono::duration<double>(std::max(timeout, 0.0)), finished))
                return Status::Err(GPT_ERR_TIMEOUT, "Job not finished within the timeout");
            return Status::Ok();
        }

        // The copy runs outside the lock: the worker thread, which takes the lock between slices, is
        // not held up by a large image on its way to the caller.
        Status Read(uint64_t id, uint32_t* rgba, float* accumulation)
        {
            std::shared_ptr<std::vector<uint32_t>> image;
            std::shared_ptr<std::vector<float>> accum;
            {
                std::scoped_lock lock(mu_);
                auto it = records_.find(id);
                if (it == records_.end()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown job id");
                const JobRecord& J = it->second;
                if (J.state != GPT_JOB_DONE) return Status::Err(GPT_ERR_STATE, "Job has no result (not done, cancelled or failed)");
                if (accumulation && (!J.accumulation || J.accumulation->empty()))
                    return Status::Err(GPT_ERR_STATE, "Job was submitted without keep_accumulation");
                image = J.rgba;
                accum = J.accumulation;
            }
            if (rgba && image) std::memcpy(rgba, image->data(), image->size() * 4);
            if (accumulation) std::memcpy(accumulation, accum->data(), accum->size() * 4);
            return Status::Ok();
        }

        Status Release(uint64_t id)
        {
            std::scoped_lock lock(mu_);
            auto it = records_.find(id);
            if (it == records_.end()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown job id");
            if (it->second.state < GPT_JOB_DONE) return Status::Err(GPT_ERR_STATE, "Job is still queued or running");
            records_.erase(it);
            return Status::Ok();
        }

        // GPT_LOOP_GRAPH or GPT_LOOP_HOST for the slices launched from now on.
        void SetLoopMode(uint32_t mode) { loopMode_.store(mode); }

        Status Cancel(uint64_t id)
        {
            std::scoped_lock lock(mu_);
            auto it = records_.find(id);
            if (it == records_.end()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown job id");
            JobRecord& J = it->second;
            if (J.state == GPT_JOB_QUEUED)
            {
                pending_.erase(std::find(pending_.begin(), pending_.end(), id));
                J.state = GPT_JOB_CANCELLED;
                J.tDone = seconds_since(t0_);
                doneCv_.notify_all();
            }
            else if (J.state == GPT_JOB_RUNNING)
            {
                J.cancelRequested = true;
                *static_cast<volatile uint32_t*>(hostMapped_) = 1u;
                cv_.notify_all();
            }
            return Status::Ok();
        }

        void Stats(gpt_server_stats& s)
        {
            std::scoped_lock lock(mu_);
            s = gpt_server_stats{};
            s.slices = slices_;
            s.iterations = hostCounters_->iteration;
            s.samples = hostCounters_->launched;
            s.rays = hostCounters_->raysTraced;
            s.shadow_rays = hostCounters_->shadowRaysTraced;
            s.admitted_bytes = admitted_;
            s.admitted_high_water = highWater_;
            s.budget_bytes = cfg_.hbm_budget_bytes;
            s.active_jobs = static_cast<uint32_t>(active_.size());
            s.queued_jobs = static_cast<uint32_t>(pending_.size());
            s.completed_jobs = completed_;
            s.scenes = static_cast<uint32_t>(pack_.entry.size());
            s.device_ms = deviceMs_;
            for (int p = 0; p < 4; p++) s.phase_ms[p] = static_cast<float>(static_cast<double>(hostCounters_->tAccum[p]) * 1e-6);
        }

        std::string LastError()
        {
            std::scoped_lock lock(mu_);
            return lastError_;
        }

    private:
        Wavefront wavefront() const
        {
            Wavefront w{};
            for (int q = 0; q < 2; q++)
            {
                w.rayO[q] = rayO_[q].get<float4>();
                w.rayD[q] = rayD_[q].get<float4>();
            }
            for (uint32_t m = 0; m < kModelCount; m++) w.matQ[m] = matQ_.get<float4>() + size_t(m) * cfg_.pool_size * 3;
            w.shO = shO_.get<float4>();
            w.shD = shD_.get<float4>();
            w.shL = shL_.get<float4>();
            w.regenBits = regenBits_.get<uint32_t>();  // the engine always regenerates from the bitmap
            w.slotT = slotT_.get<float4>();
            w.slotL = slotL_.get<float4>();
            w.slotSample = slotSample_.get<uint32_t>();
            w.capacity = cfg_.pool_size;
            w.logCapacity = 0;
            w.queueLog = nullptr;
            w.ctr = counters_.get<Counters>();
            w.cancel = nullptr;
            w.progress = reinterpret_cast<volatile unsigned long long*>(static_cast<char*>(hostMappedDev_) + 16);
            return w;
        }

        EngineView engineView() const
        {
            EngineView v{};
            v.jobs = jobs_.get<JobView>();
            v.order = order_.get<uint32_t>();
            v.segments = segments_.get<LaunchSegment>();
            v.freeList = freeList_.get<uint32_t>();
            v.ctl = ctl_.get<EngineCtl>();
            v.scenes = pack_.entries.get<SceneEntry>();
            v.doorbell = static_cast<const volatile uint32_t*>(hostMappedDev_);
            return v;
        }

        void releaseGraph()
        {
            if (graphExec_) cudaGraphExecDestroy(graphExec_);
            if (graph_) cudaGraphDestroy(graph_);
            graphExec_ = nullptr;
            graph_ = nullptr;
        }

        // The launch parameters of one engine iteration: inside the slice graph's WHILE node
        // (graphLoop, with its conditional handle) or launched from the host (GPT_LOOP_HOST).
        EngineLaunch iterationLaunch(int sms, bool graphLoop, cudaGraphConditionalHandle handle)
        {
            EngineLaunch L{};
            L.scene = pack_.view();
            L.wf = wavefront();
            L.ev = engineView();
            L.handle = handle;
            for (uint32_t m = 0; m < kModelCount; m++) L.modelPresent[m] = pack_.modelPresent[m];
            L.anyLights = pack_.lightCount > 0;
            L.traceThreads = threads_;
            L.occupancy = occupancy_;
            L.traceBlocks = trace_grid_blocks(device_, threads_, pack_.depth, occupancy_);
            L.refill = refill_;
            L.refillShadow = refillShadow_;
            L.shadeBlocks = sms * 8;
            L.sms = sms;
            L.graphLoop = graphLoop;
            L.shadeFork = shadeFork_;
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                L.shadeJoin[m] = shadeJoin_[m];
                L.shadeStreams[m] = shadeStreams_[m];
            }
            return L;
        }

        Status buildGraph()
        {
            releaseGraph();
            int sms = 0;
            PT_CUDA("cudaDeviceGetAttribute", cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
            PT_CUDA("cudaGraphCreate", cudaGraphCreate(&graph_, 0));
            cudaGraphConditionalHandle handle;
            PT_CUDA("cudaGraphConditionalHandleCreate", cudaGraphConditionalHandleCreate(&handle, graph_, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t whileNode;
            PT_CUDA("cudaGraphAddNode", cudaGraphAddNode(&whileNode, graph_, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            const EngineLaunch L = iterationLaunch(sms, true, handle);
            PT_CUDA("cudaStreamBeginCaptureToGraph", cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            const cudaError_t le = launch_engine_iteration(L, stream_);
            const cudaError_t ce = cudaStreamEndCapture(stream_, &body);
            PT_CUDA("engine iteration launch", le);
            PT_CUDA("cudaStreamEndCapture", ce);
            PT_CUDA("cudaGraphInstantiate", cudaGraphInstantiate(&graphExec_, graph_, 0));
            return Status::Ok();
        }

        // A short job of the two-class order: its render time alone, at the server's measured rate, is
        // below short_job_seconds.
        bool is_short(const JobRecord& J) const
        {
            const double samples = static_cast<double>(uint64_t(J.spp) * J.pixels);
            return samples / rateEstimate_.load(std::memory_order_relaxed) < cfg_.short_job_seconds;
        }
        // Admission queue of a job: short jobs (0) and the others (1) under the two-class order, one queue otherwise.
        int admission_class(const JobRecord& J) const { return schedule_ == GPT_SCHEDULE_TWO_CLASS && is_short(J) ? 0 : 1; }
        // Whether the job's bytes fit the budget now. Under the two-class order a long job may fill only
        // seven eighths of it, so that short arrivals find memory while long jobs hold the rest; a long
        // job larger than that is admitted only onto an empty device.
        bool fits_budget(const JobRecord& J) const
        {
            uint64_t limit = cfg_.hbm_budget_bytes;
            if (admission_class(J) == 1 && schedule_ == GPT_SCHEDULE_TWO_CLASS)
            {
                const uint64_t longLimit = limit - limit / 8;
                if (J.admittedBytes <= longLimit || admitted_ > 0) limit = longLimit;
            }
            return admitted_ + J.admittedBytes <= limit;
        }

        // Under mu_: starts a waiting job in its arena block at `offset` (job table entry, device view,
        // cleared accumulator); the caller removes it from the waiting list.
        Status admit(JobRecord& J, size_t offset)
        {
            NvtxRange range("gpt server admit");
            J.arenaOffset = offset;
            J.tableIndex = freeTable_.back();
            freeTable_.pop_back();
            char* base = arena_.base() + offset;
            JobView v{};
            std::memcpy(v.camera, &J.desc.camera, sizeof(v.camera));
            v.width = J.desc.width;
            v.height = J.desc.height;
            v.spp = J.spp;
            v.spa = J.spa;
            v.depthLimit = std::min(std::max(J.desc.path_depth, 1u), 100u);
            v.nee = J.desc.use_nee ? 1u : 0u;
            v.maxIterations = 0;
            v.scene = J.desc.scene;
            v.totalSamples = uint64_t(J.spp) * J.pixels;
            v.sampleRadiance = reinterpret_cast<float*>(base);
            v.rngOffset = J.desc.rng_offset;
            v.rngPolicy = J.desc.rng_policy;
            v.lightMode = J.desc.light_sampling;
            v.pixels = J.pixels;
            v.ring = J.ring;
            v.state = kJobActive;
            v.folded = 0;
            v.launched = 0;
            v.accum = reinterpret_cast<float4*>(base + J.ringBytes);
            v.framebuffer = reinterpret_cast<uint32_t*>(base + J.ringBytes + J.accumBytes);
            v.passDone = reinterpret_cast<uint32_t*>(base + J.ringBytes + J.accumBytes + J.fbBytes);
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(v.accum, 0, J.accumBytes, stream_));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(v.passDone, 0, J.doneBytes, stream_));
            mirror_[J.tableIndex] = v;
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(jobs_.get<JobView>() + J.tableIndex, &mirror_[J.tableIndex], sizeof(JobView),
                                                       cudaMemcpyHostToDevice, stream_));
            J.view = v;
            J.state = GPT_JOB_RUNNING;
            J.tAdmit = seconds_since(t0_);
            admitted_ += J.admittedBytes;
            highWater_ = std::max(highWater_, admitted_);
            active_.push_back(J.id);
            return Status::Ok();
        }

        // Under mu_: apply cancellations, admit waiting jobs in submission order (per admission class)
        // while a table entry, the budget and the arena allow, and stage the slice's order list and
        // control words.
        Status prepareSlice()
        {
            for (uint64_t id : active_)
            {
                JobRecord& J = records_[id];
                if (!J.cancelRequested || J.cancelApplied) continue;
                // no more launches: the job ends with the samples it has handed out
                const uint64_t launched = mirror_[J.tableIndex].launched;
                PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(reinterpret_cast<char*>(jobs_.get<JobView>() + J.tableIndex) + offsetof(JobView, totalSamples),
                                                           &launched, sizeof(uint64_t), cudaMemcpyHostToDevice, stream_));
                PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
                J.cancelApplied = true;
            }
            // Waiting jobs are admitted in submission order. Under the two-class order the classes queue
            // separately, short jobs first, and long jobs leave an eighth of the budget to short jobs
            // (fits_budget): a long job that does not fit blocks the long jobs behind it (they keep their
            // order) but not the short ones. With one queue and the whole budget open to every job, a
            // backlog of long jobs held the budget and every short arrival waited for memory (200 arrivals
            // at 50 jobs/s: median latency 2.1 s against 0.11 s at 20 jobs/s).
            const bool twoClass = schedule_ == GPT_SCHEDULE_TWO_CLASS;
            for (int pass = twoClass ? 0 : 1; pass < 2; pass++)
            {
                for (auto it = pending_.begin(); it != pending_.end();)
                {
                    // jobs whose images are still being copied out count as active (one at a time means no overlap at all)
                    if (cfg_.max_active_jobs && active_.size() + toCopy_.size() >= cfg_.max_active_jobs) break;
                    if (freeTable_.empty()) break;
                    JobRecord& J = records_[*it];
                    if (twoClass && admission_class(J) != pass)
                    {
                        ++it;
                        continue;
                    }
                    size_t offset = 0;
                    if (!fits_budget(J) || !arena_.allocate(J.arenaBytes, offset)) break;
                    PT_TRY(admit(J, offset));
                    it = pending_.erase(it);
                }
            }
            // Slot priority of the next slice: the device plan hands idle slots to the jobs in this order
            // (by class, then key; the stable sort keeps submission order among equal keys).
            struct Rank
            {
                int cls;
                double key;
                uint32_t table;
            };
            std::vector<Rank> ranked;
            ranked.reserve(active_.size());
            for (uint64_t id : active_)
            {
                const JobRecord& J = records_[id];
                const uint32_t t = J.tableIndex;
                const JobView& v = mirror_[t];
                const uint64_t left = v.totalSamples > v.launched ? v.totalSamples - v.launched : 0;
                int cls = 0;
                double key = 0.0;  // oldest first: all equal
                if (schedule_ == GPT_SCHEDULE_SHORTEST_FIRST) key = static_cast<double>(left);
                else if (schedule_ == GPT_SCHEDULE_DEADLINE)
                    key = J.tSubmit + cfg_.deadline_slowdown * static_cast<double>(v.totalSamples) / rateEstimate_.load(std::memory_order_relaxed);
                else if (schedule_ == GPT_SCHEDULE_TWO_CLASS)
                {
                    // short jobs (estimated render time alone below short_job_seconds) first, fewest samples
                    // left first; long jobs after them in submission order
                    const bool isShort = is_short(J);
                    cls = isShort ? 0 : 1;
                    key = isShort ? static_cast<double>(left) : 0.0;
                }
                ranked.push_back(Rank{cls, key, t});
            }
            std::stable_sort(ranked.begin(), ranked.end(),
                             [](const Rank& a, const Rank& b) { return a.cls != b.cls ? a.cls < b.cls : a.key < b.key; });
            uint32_t n = 0;
            // two classes: long jobs take their turns in submission order; a later one gets slots only once
            // the ones ahead have launched everything (not merely while their pass windows are full)
            for (const auto& r : ranked) orderHost_[n++] = r.table | (schedule_ == GPT_SCHEDULE_TWO_CLASS && r.cls == 1 ? kOrderInTurn : 0u);
            sliceWords_[0] = n;
            sliceWords_[1] = 0;
            sliceWords_[2] = cfg_.max_slice_iterations;
            sliceWords_[3] = 0;
            if (n) PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(order_.get<uint32_t>(), orderHost_, size_t(n) * 4, cudaMemcpyHostToDevice, stream_));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(reinterpret_cast<char*>(ctl_.get<EngineCtl>()) + offsetof(EngineCtl, orderCount), sliceWords_, 16,
                                                       cudaMemcpyHostToDevice, stream_));
            return Status::Ok();
        }

        // Under mu_: one graph launch, then the counters and the job table come back (queued on the
        // render stream; waitSlice collects them). With GPT_LOOP_HOST the slice's iterations are
        // launched one by one by waitSlice instead.
        Status launchSlice()
        {
            hostSlice_ = loopMode_.load() == GPT_LOOP_HOST;
            if (hostSlice_)
            {
                PT_CUDA("cudaEventRecord", cudaEventRecord(startEvent_, stream_));
                return Status::Ok();
            }
            if (!graphExec_) PT_TRY(buildGraph());
            PT_CUDA("cudaEventRecord", cudaEventRecord(startEvent_, stream_));
            PT_CUDA("cudaGraphLaunch", cudaGraphLaunch(graphExec_, stream_));
            return readBack();
        }

        Status readBack()
        {
            PT_CUDA("cudaEventRecord", cudaEventRecord(stopEvent_, stream_));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(hostCounters_, counters_.get<void>(), sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(hostCtl_, ctl_.get<void>(), sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(mirror_, jobs_.get<void>(), size_t(cfg_.max_jobs) * sizeof(JobView), cudaMemcpyDeviceToHost, stream_));
            return Status::Ok();
        }

        // Without mu_, GPT_LOOP_HOST: the slice's iterations as ordinary launches, the loop condition
        // read after each (the graph's WHILE node reads it on the device). ncu profiles these kernels;
        // it does not profile kernel nodes of graphs with conditional nodes.
        Status hostLoopSlice()
        {
            int sms = 0;
            PT_CUDA("cudaDeviceGetAttribute", cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
            const EngineLaunch L = iterationLaunch(sms, false, 0);
            const uint64_t cap = uint64_t(cfg_.max_slice_iterations) + 1;
            for (uint64_t it = 0; it < cap; it++)
            {
                PT_CUDA("engine iteration", launch_engine_iteration(L, stream_));
                PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&hostCounters_->done, &counters_.get<Counters>()->done, 4, cudaMemcpyDeviceToHost, stream_));
                PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
                if (hostCounters_->done) break;
            }
            return readBack();
        }

        // Without mu_: waits for the slice launched by launchSlice.
        Status waitSlice()
        {
            NvtxRange range("gpt server slice");
            if (hostSlice_) PT_TRY(hostLoopSlice());
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
            float ms = 0.0f;
            PT_CUDA("cudaEventElapsedTime", cudaEventElapsedTime(&ms, startEvent_, stopEvent_));
            deviceMs_ += ms;
            slices_++;
            // paths per second of the server (device time), the clock of the two-class and deadline
            // orders. Samples are counted when launched, and a slice can refill the whole pool in its
            // first iteration, so one short slice overstates the rate many times over: the estimate is
            // taken over windows of at least 100 ms of device time (a pool-full then moves it by a few
            // per cent) and smoothed across windows.
            const uint64_t samples = hostCounters_->launched;
            if (samples > lastSliceSamples_) rateSamples_ += samples - lastSliceSamples_;
            rateMs_ += ms;
            if (rateMs_ >= 100.0)
            {
                const double rate = static_cast<double>(rateSamples_) / (rateMs_ / 1000.0);
                rateEstimate_.store(0.5 * rateEstimate_.load(std::memory_order_relaxed) + 0.5 * rate, std::memory_order_relaxed);
                rateSamples_ = 0;
                rateMs_ = 0.0;
            }
            lastSliceSamples_ = samples;
            if (hostCounters_->errorFlags)
                return Status::Err(GPT_ERR_DEVICE_FAULT, "Traversal reported error flags " + std::to_string(hostCounters_->errorFlags));
            if (hostCtl_->stalled) return Status::Err(GPT_ERR_DEVICE_FAULT, "Job engine stalled with unfinished jobs");
            return Status::Ok();
        }

        // Under mu_: progress of running jobs. Finished jobs leave the active list and wait in toCopy_
        // for their images to reach host memory; their table entry and arena range stay theirs until
        // then (the device no longer touches a finished job's buffers).
        Status retire()
        {
            for (size_t i = 0; i < active_.size();)
            {
                JobRecord& J = records_[active_[i]];
                const JobView& m = mirror_[J.tableIndex];
                J.passesDone = m.folded;
                if (m.state != kJobDone)
                {
                    i++;
                    continue;
                }
                if (J.cancelApplied)
                    finish(J, GPT_JOB_CANCELLED);
                else
                {
                    toCopy_.push_back(J.id);
                }
                active_.erase(active_.begin() + static_cast<std::ptrdiff_t>(i));
            }
            return Status::Ok();
        }

        // Without mu_: images (and accumulations) of finished jobs to host memory through pinned
        // staging on the copy stream, while the next slice runs on the render stream. Their host
        // buffers are allocated here too, not under the lock between slices (no other thread reads a
        // record's image before finish() marks it done).
        Status copyImages(const std::vector<JobRecord*>& jobs)
        {
            char* st = static_cast<char*>(staging_);
            for (JobRecord* J : jobs)
            {
                J->rgba = std::make_shared<std::vector<uint32_t>>(J->pixels);
                if (J->desc.keep_accumulation) J->accumulation = std::make_shared<std::vector<float>>(size_t(J->pixels) * 4);
                // RGBA8 image in chunks of the fixed staging buffer
                const char* src = reinterpret_cast<const char*>(J->view.framebuffer);
                char* dst = reinterpret_cast<char*>(J->rgba->data());
                for (size_t done = 0, total = size_t(J->pixels) * 4; done < total;)
                {
                    const size_t n = std::min(kStagingBytes, total - done);
                    PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(st, src + done, n, cudaMemcpyDeviceToHost, copyStream_));
                    PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(copyStream_));
                    std::memcpy(dst + done, st, n);
                    done += n;
                }
                if (!J->desc.keep_accumulation) continue;
                // the accumulator holds (sum, compensation) pairs per pixel; the sums are the accumulation
                const size_t rows = kStagingBytes / 16;
                for (size_t px = 0; px < J->pixels;)
                {
                    const size_t n = std::min(rows, size_t(J->pixels) - px);
                    PT_CUDA("cudaMemcpy2DAsync", cudaMemcpy2DAsync(st, 16, J->view.accum + 2 * px, 32, 16, n, cudaMemcpyDeviceToHost, copyStream_));
                    PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(copyStream_));
                    std::memcpy(J->accumulation->data() + 4 * px, st, n * 16);
                    px += n;
                }
            }
            return Status::Ok();
        }

        void finish(JobRecord& J, uint32_t state)
        {
            if (J.tableIndex != kInvalid)
            {
                arena_.release(J.arenaOffset, J.arenaBytes);
                freeTable_.push_back(J.tableIndex);
                mirror_[J.tableIndex].state = kJobFree;
                J.tableIndex = kInvalid;
                admitted_ -= J.admittedBytes;
            }
            J.state = state;
            J.tDone = seconds_since(t0_);
            doneCv_.notify_all();
        }

        // A failed slice fails every running job and restarts the engine with an empty pool.
        void failActive(const Status& st)
        {
            lastError_ = st.message;
            for (uint64_t id : active_) finish(records_[id], GPT_JOB_FAILED);
            active_.clear();
            cudaGetLastError();
            cudaMemsetAsync(jobs_.get<void>(), 0, size_t(cfg_.max_jobs) * sizeof(JobView), stream_);
            launch_engine_init(wavefront(), engineView(), cfg_.pool_size, stream_);
            cudaStreamSynchronize(stream_);
        }

        // Scheduler thread. Per round: admit waiting jobs and launch a slice; while it runs, copy out
        // the images of the jobs the previous slice finished and hand them to their waiters; then
        // collect the slice's results.
        void Run()
        {
            cudaSetDevice(device_);
            std::unique_lock<std::mutex> lock(mu_);
            for (;;)
            {
                cv_.wait(lock, [&] { return stop_ || !pending_.empty() || !active_.empty() || !toCopy_.empty(); });
                if (stop_) break;
                // cleared before the queue is read: a job submitted from now on rings again
                *static_cast<volatile uint32_t*>(hostMapped_) = 0u;
                Status st = prepareSlice();
                if (!st.ok())
                {
                    failActive(st);
                    continue;
                }
                const bool run = !active_.empty();
                if (run && !(st = launchSlice()).ok())
                {
                    failActive(st);
                    continue;
                }
                std::vector<JobRecord*> batch;
                for (uint64_t id : toCopy_) batch.push_back(&records_[id]);
                toCopy_.clear();
                if (!batch.empty())
                {
                    lock.unlock();
                    const Status cs = copyImages(batch);
                    lock.lock();
                    if (!cs.ok()) lastError_ = cs.message;
                    for (JobRecord* J : batch)
                    {
                        finish(*J, cs.ok() ? GPT_JOB_DONE : GPT_JOB_FAILED);
                        if (cs.ok()) completed_++;
                    }
                }
                if (!run) continue;
                lock.unlock();
                st = waitSlice();
                lock.lock();
                if (!st.ok())
                {
                    failActive(st);
                    continue;
                }
                st = retire();
                if (!st.ok()) failActive(st);
            }
        }

        int device_;
        gpt_server_config cfg_;
        int threads_ = 128, occupancy_ = 10;
        uint32_t schedule_ = GPT_SCHEDULE_TWO_CLASS;
        std::atomic<uint32_t> loopMode_{GPT_LOOP_GRAPH};  // slices as one graph launch, or iterations launched by the host
        bool hostSlice_ = false;                          // the slice in flight runs its iterations from the host
        std::atomic<double> rateEstimate_{1e9};  // paths per second, smoothed (initial guess: one B200 on a mid-size scene); read by Submit
        uint64_t lastSliceSamples_ = 0;
        uint64_t rateSamples_ = 0;         // samples launched in the current rate window
        double rateMs_ = 0.0;              // device milliseconds of the current rate window
        uint32_t refill_ = 16, refillShadow_ = 8;
        std::chrono::steady_clock::time_point t0_;
        cudaStream_t stream_ = nullptr;
        cudaStream_t copyStream_ = nullptr;  // images of finished jobs to host memory, beside the running slice
        cudaEvent_t shadeFork_ = nullptr;     // the shading kernels run as parallel branches of the slice graph
        cudaEvent_t shadeJoin_[kModelCount] = {};
        cudaStream_t shadeStreams_[kModelCount] = {};
        void* staging_ = nullptr;            // pinned staging of those copies, kStagingBytes
        std::vector<uint64_t> toCopy_;       // finished jobs whose images are not on the host yet
        cudaEvent_t startEvent_ = nullptr, stopEvent_ = nullptr;
        void* hostMapped_ = nullptr;     // [0] doorbell, [16..31] progress
        void* hostMappedDev_ = nullptr;
        void* pinned_ = nullptr;
        size_t pinnedBytes_ = 0;
        Counters* hostCounters_ = nullptr;
        EngineCtl* hostCtl_ = nullptr;
        JobView* mirror_ = nullptr;
        uint32_t* orderHost_ = nullptr;
        uint32_t* sliceWords_ = nullptr;
        DeviceBuffer rayO_[2], rayD_[2], matQ_, shO_, shD_, shL_, regenBits_, slotT_, slotL_, slotSample_, freeList_;
        DeviceBuffer counters_, ctl_, jobs_, order_, segments_;
        ScenePack pack_;
        Arena arena_;
        cudaGraph_t graph_ = nullptr;
        cudaGraphExec_t graphExec_ = nullptr;

        std::mutex mu_;
        std::condition_variable cv_, doneCv_;
        std::map<uint64_t, JobRecord> records_;
        std::deque<uint64_t> pending_;
        std::vector<uint64_t> active_;
        std::vector<uint32_t> freeTable_;
        uint64_t nextId_ = 1;
        uint64_t admitted_ = 0, highWater_ = 0, slices_ = 0;
        uint32_t completed_ = 0;
        double deviceMs_ = 0.0;
        bool stop_ = false;
        std::string lastError_;
        std::thread worker_;
    };
}

struct gpt_server
{
    std::unique_ptr<pt::Server> impl;
    std::mutex errorMutex;
    std::string lastError;
};

namespace
{
    int ServerReport(gpt_server* s, const pt::Status& st)
    {
        if (!st.ok())
        {
            std::scoped_lock lock(s->errorMutex);
            s->lastError = st.message;
        }
        return st.code;
    }
}

extern "C"
{
    int gpt_server_create(gpt_server** out, int device, const gpt_server_config* config)
    {
        if (!out) return GPT_ERR_INVALID_ARGUMENT;
        *out = nullptr;
        gpt_server_config c{};
        if (config) c = *config;
        auto s = std::make_unique<gpt_server>();
        s->impl = std::make_unique<pt::Server>(device, c);
        const pt::Status st = s->impl->Init();
        if (!st.ok()) return st.code;
        *out = s.release();
        return GPT_OK;
    }

    int gpt_server_destroy(gpt_server* s)
    {
        delete s;
        return GPT_OK;
    }

    int gpt_server_add_scene(gpt_server* s, const gpt_scene_desc* d, uint32_t* id)
    {
        if (!s || !d || !id) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->AddScene(*d, *id));
    }

    int gpt_server_submit(gpt_server* s, const gpt_job_desc* j, uint64_t* id)
    {
        if (!s || !j || !id) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Submit(*j, *id));
    }

    int gpt_server_poll(gpt_server* s, uint64_t id, gpt_job_status* st)
    {
        if (!s || !st) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Poll(id, *st));
    }

    int gpt_server_wait(gpt_server* s, uint64_t id, double timeout_s)
    {
        if (!s) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Wait(id, timeout_s));
    }

    int gpt_server_read(gpt_server* s, uint64_t id, uint32_t* rgba, float* accumulation)
    {
        if (!s) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Read(id, rgba, accumulation));
    }

    int gpt_server_release(gpt_server* s, uint64_t id)
    {
        if (!s) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Release(id));
    }

    int gpt_server_cancel(gpt_server* s, uint64_t id)
    {
        if (!s) return GPT_ERR_INVALID_ARGUMENT;
        return ServerReport(s, s->impl->Cancel(id));
    }

    int gpt_server_set_loop_mode(gpt_server* s, uint32_t mode)
    {
        if (!s) return GPT_ERR_INVALID_ARGUMENT;
        if (mode > GPT_LOOP_HOST) return ServerReport(s, pt::Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown loop mode"));
        s->impl->SetLoopMode(mode);
        return GPT_OK;
    }

    int gpt_server_get_stats(gpt_server* s, gpt_server_stats* out)
    {
        if (!s || !out) return GPT_ERR_INVALID_ARGUMENT;
        s->impl->Stats(*out);
        return GPT_OK;
    }

    int gpt_server_peek_last_error(gpt_server* s, char* buffer, size_t length)
    {
        if (!s) return 0;
        std::string msg;
        {
            std::scoped_lock lock(s->errorMutex);
            msg = s->lastError;
        }
        const std::string engine = s->impl->LastError();
        if (msg.empty()) msg = engine;
        if (msg.empty()) return 0;
        if (buffer && length)
        {
            const size_t n = std::min(length - 1, msg.size());
            std::memcpy(buffer, msg.data(), n);
            buffer[n] = 0;
        }
        return 1;
    }
}
