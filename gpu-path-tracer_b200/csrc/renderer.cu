// Host runtime of the B200 wavefront path tracer and its C ABI (include/gpt_b200.h).
//
// Mirrors Core::Graphics::Cuda::Renderer (Core/Include/Core/Graphics/Cuda/PathTracing/Renderer.hpp:42-189,
// Core/Source/Graphics/Cuda/PathTracing/Renderer.cpp): buffer initialisation, scene upload, a worker-thread
// simulation over camera motion states with stop/resume, a locked host frame, last-error reporting.
// The frame itself differs by design: the reference drives every wavefront iteration from the host with
// two blocking synchronisations (Renderer.cpp:532,590); here one CUDA graph holds the whole frame and a
// conditional WHILE node repeats the iteration body until the device-side counters say the frame is done.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gpt_b200.h"
#include "bvh8.hpp"
#include "bvh_device.hpp"
#include "kernels.h"
#include "runtime.hpp"

namespace pt
{
    // gpt_inject_allocation_failure: allocations left until the injected failure (0 = none armed).
    std::atomic<uint32_t> g_allocationCountdown{0};

    bool InjectedAllocationFailure()
    {
        uint32_t c = g_allocationCountdown.load();
        while (c != 0)
            if (g_allocationCountdown.compare_exchange_weak(c, c - 1)) return c == 1;
        return false;
    }

    static Status CreateTexture(const gpt_texture_desc& d, TextureObject& t)
    {
        if (d.width == 0 || d.height == 0 || !d.data || (d.channels != 1 && d.channels != 3 && d.channels != 4) || d.format > GPT_TEXEL_F32)
            return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unsupported texture description");
        const bool u8 = d.format != GPT_TEXEL_F32;
        const size_t texels = static_cast<size_t>(d.width) * d.height;
        const uint32_t outChannels = d.channels == 1 ? 1 : 4;
        const size_t elem = (u8 ? 1 : 4) * outChannels;
        std::vector<unsigned char> expanded;
        const void* src = d.data;
        if (d.channels == 3)  // Import::ConvertRgbToRgba: alpha 255 (u8) or 1.0 (float)
        {
            expanded.resize(texels * elem);
            for (size_t i = 0; i < texels; i++)
            {
                if (u8)
                {
                    const unsigned char* in = static_cast<const unsigned char*>(d.data) + i * 3;
                    unsigned char* o = expanded.data() + i * 4;
                    o[0] = in[0];
                    o[1] = in[1];
                    o[2] = in[2];
                    o[3] = 255;
                }
                else
                {
                    const float* in = static_cast<const float*>(d.data) + i * 3;
                    float* o = reinterpret_cast<float*>(expanded.data()) + i * 4;
                    o[0] = in[0];
                    o[1] = in[1];
                    o[2] = in[2];
                    o[3] = 1.0f;
                }
            }
            src = expanded.data();
        }
        cudaChannelFormatDesc cd = u8 ? (outChannels == 1 ? cudaCreateChannelDesc<uchar1>() : cudaCreateChannelDesc<uchar4>())
                                      : (outChannels == 1 ? cudaCreateChannelDesc<float1>() : cudaCreateChannelDesc<float4>());
        PT_CUDA("cudaMallocArray", cudaMallocArray(&t.array, &cd, d.width, d.height));
        const size_t pitch = static_cast<size_t>(d.width) * elem;
        PT_CUDA("cudaMemcpy2DToArray", cudaMemcpy2DToArray(t.array, 0, 0, src, pitch, pitch, d.height, cudaMemcpyHostToDevice));
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = t.array;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.normalizedCoords = 1;
        td.sRGB = d.format == GPT_TEXEL_U8_SRGB ? 1 : 0;
        td.readMode = u8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        PT_CUDA("cudaCreateTextureObject", cudaCreateTextureObject(&t.object, &res, &td, nullptr));
        return Status::Ok();
    }

    static bool WritePng(const std::string& path, const uint32_t* rgba, uint32_t w, uint32_t h)
    {
        std::vector<unsigned char> raw(static_cast<size_t>(h) * (1 + 4 * static_cast<size_t>(w)));
        for (uint32_t y = 0; y < h; y++)
        {
            unsigned char* row = raw.data() + static_cast<size_t>(y) * (1 + 4 * static_cast<size_t>(w));
            row[0] = 0;
            std::memcpy(row + 1, rgba + static_cast<size_t>(h - 1 - y) * w, 4 * static_cast<size_t>(w));
        }
        uLongf zlen = compressBound(static_cast<uLong>(raw.size()));
        std::vector<unsigned char> z(zlen);
        if (compress2(z.data(), &zlen, raw.data(), static_cast<uLong>(raw.size()), 6) != Z_OK) return false;
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return false;
        auto be32 = [](uint32_t v, unsigned char* o) { o[0] = v >> 24; o[1] = v >> 16; o[2] = v >> 8; o[3] = v; };
        auto chunk = [&](const char* type, const unsigned char* data, uint32_t len)
        {
            unsigned char hdr[8];
            be32(len, hdr);
            std::memcpy(hdr + 4, type, 4);
            std::fwrite(hdr, 1, 8, f);
            if (len) std::fwrite(data, 1, len, f);
            uLong crc = crc32(0L, reinterpret_cast<const Bytef*>(type), 4);
            if (len) crc = crc32(crc, data, len);
            unsigned char c[4];
            be32(static_cast<uint32_t>(crc), c);
            std::fwrite(c, 1, 4, f);
        };
        const unsigned char sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
        std::fwrite(sig, 1, 8, f);
        unsigned char ihdr[13];
        be32(w, ihdr);
        be32(h, ihdr + 4);
        ihdr[8] = 8;
        ihdr[9] = 6;
        ihdr[10] = ihdr[11] = ihdr[12] = 0;
        chunk("IHDR", ihdr, 13);
        chunk("IDAT", z.data(), static_cast<uint32_t>(zlen));
        chunk("IEND", nullptr, 0);
        return std::fclose(f) == 0;
    }

    // Scene upload of Renderer::InitializeSceneBuffers (Renderer.cpp:292-306): validation, image textures,
    // BVH8 (host or device), shading records, light list and alias table (device).
    Status BuildScene(const gpt_scene_desc& d, cudaStream_t stream, std::unique_ptr<SceneGpu>& out, bool withBinary, bool deviceBvh)
    {
        if (d.triangle_count == 0 || !d.positions || !d.normals || !d.tangents || !d.uvs || !d.material_ids || !d.materials ||
            d.material_count == 0)
            return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Scene description is incomplete");
        NvtxRange rangeUpload("gpt scene upload");
        const auto tUpload = std::chrono::steady_clock::now();
        const uint32_t n = d.triangle_count;
        std::vector<uint32_t> models(n);
        bool present[kModelCount] = {};
        for (uint32_t m = 0; m < d.material_count; m++)
            if (d.materials[m].model >= kModelCount)
                return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Material has an unknown shading model");
        for (uint32_t t = 0; t < n; t++)
        {
            const uint32_t mat = d.material_ids[t];
            if (mat >= d.material_count) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Triangle material index out of range");
            models[t] = d.materials[mat].model;
            present[models[t]] = true;
        }
        auto scene = std::make_unique<SceneGpu>();
        std::copy(present, present + kModelCount, scene->modelPresent);
        // image textures of the material slots
        if (d.texture_count > 0 && d.material_textures)
        {
            if (!d.textures) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Texture table is missing");
            std::vector<MaterialTextures> slots(d.material_count);
            for (uint32_t i = 0; i < d.texture_count; i++)
            {
                scene->textures.push_back(std::make_unique<TextureObject>());
                PT_TRY(CreateTexture(d.textures[i], *scene->textures.back()));
            }
            for (uint32_t m = 0; m < d.material_count; m++)
            {
                slots[m] = MaterialTextures{};
                for (int k = 0; k < GPT_TEX_SLOTS; k++)
                {
                    const int32_t ti = d.material_textures[static_cast<size_t>(m) * GPT_TEX_SLOTS + k];
                    if (ti < 0) continue;
                    if (static_cast<uint32_t>(ti) >= d.texture_count)
                        return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Material texture index out of range");
                    const bool scalar = k == GPT_TEX_SHININESS;
                    if ((d.textures[ti].channels == 1) != scalar)
                        return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Shininess maps have one channel, other maps three or four");
                    slots[m].tex[k] = scene->textures[ti]->object;
                }
            }
            PT_TRY(scene->materialTextures.allocate(slots.size() * sizeof(MaterialTextures)));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->materialTextures.get<void>(), slots.data(), slots.size() * sizeof(MaterialTextures),
                                                       cudaMemcpyHostToDevice, stream));
        }
        // Vertex positions go up first: the device BVH build and the shading records read them.
        DeviceBuffer pos, nrm, tan, uv, mid;
        PT_TRY(pos.allocate(static_cast<size_t>(n) * 9 * 4));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(pos.get<void>(), d.positions, static_cast<size_t>(n) * 36, cudaMemcpyHostToDevice, stream));
        scene->triangleCount = n;
        scene->materialCount = d.material_count;
        scene->deviceBvh = deviceBvh;
        const auto tBvh = std::chrono::steady_clock::now();
        NvtxRange rangeBvh(deviceBvh ? "gpt bvh8 build (device)" : "gpt bvh8 build (host)");
        Bvh8 bvh;
        if (deviceBvh)
        {
            // BVH8 on the device (Morton order, clustering, collapse, quantisation); no binary BVH
            DeviceBuffer modelsDev;
            PT_TRY(modelsDev.allocate(static_cast<size_t>(n) * 4));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(modelsDev.get<void>(), models.data(), static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, stream));
            DeviceBvh dev;
            PT_TRY(BuildBvh8Device(pos.get<float>(), modelsDev.get<uint32_t>(), n, stream, dev));
            scene->nodes.swap(dev.nodes);
            scene->tris.swap(dev.tris);
            scene->nodeCount = dev.nodeCount;
            scene->depth = dev.depth;
            withBinary = false;
        }
        else
        {
            // BVH8 on the host (binned SAH, collapse, quantisation).
            try
            {
                bvh = BuildBvh8(d.positions, models.data(), n, static_cast<int>(std::max(1u, std::thread::hardware_concurrency())), withBinary);
            }
            catch (const std::exception& e)
            {
                return Status::Err(GPT_ERR_INVALID_ARGUMENT, std::string("BVH build failed: ") + e.what());
            }
            if (bvh.depth > kMaxStack) return Status::Err(GPT_ERR_CAPACITY, "BVH8 deeper than the traversal stack");
            if (bvh.nodes.size() >= (1u << 24)) return Status::Err(GPT_ERR_CAPACITY, "BVH8 has more than 2^24 nodes");
            scene->nodeCount = static_cast<uint32_t>(bvh.nodes.size());
            scene->depth = bvh.depth;
            PT_TRY(scene->nodes.allocate(bvh.nodes.size() * sizeof(Node8)));
            PT_TRY(scene->tris.allocate(bvh.tris.size() * sizeof(float4)));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->nodes.get<void>(), bvh.nodes.data(), bvh.nodes.size() * sizeof(Node8), cudaMemcpyHostToDevice, stream));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->tris.get<void>(), bvh.tris.data(), bvh.tris.size() * sizeof(float4), cudaMemcpyHostToDevice, stream));
        }
        scene->bvhSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tBvh).count();
        rangeBvh.end();
        PT_TRY(scene->shading.allocate(static_cast<size_t>(n) * 9 * sizeof(float4)));
        PT_TRY(scene->materials.allocate(static_cast<size_t>(d.material_count) * sizeof(MaterialDev)));
        if (withBinary)
        {
            if (bvh.depth2 > kMaxStack) return Status::Err(GPT_ERR_CAPACITY, "Binary BVH deeper than the traversal stack");
            scene->nodeCount2 = static_cast<uint32_t>(bvh.nodes2.size());
            scene->depth2 = bvh.depth2;
            PT_TRY(scene->nodes2.allocate(bvh.nodes2.size() * sizeof(Node2)));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->nodes2.get<void>(), bvh.nodes2.data(), bvh.nodes2.size() * sizeof(Node2),
                                                       cudaMemcpyHostToDevice, stream));
        }
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->materials.get<void>(), d.materials, static_cast<size_t>(d.material_count) * sizeof(MaterialDev), cudaMemcpyHostToDevice, stream));
        // Vertex attributes go up once; shading records, lights and the alias table are built on the device.
        PT_TRY(nrm.allocate(static_cast<size_t>(n) * 9 * 4));
        PT_TRY(tan.allocate(static_cast<size_t>(n) * 12 * 4));
        PT_TRY(uv.allocate(static_cast<size_t>(n) * 6 * 4));
        PT_TRY(mid.allocate(static_cast<size_t>(n) * 4));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(nrm.get<void>(), d.normals, static_cast<size_t>(n) * 36, cudaMemcpyHostToDevice, stream));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(tan.get<void>(), d.tangents, static_cast<size_t>(n) * 48, cudaMemcpyHostToDevice, stream));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(uv.get<void>(), d.uvs, static_cast<size_t>(n) * 24, cudaMemcpyHostToDevice, stream));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(mid.get<void>(), d.material_ids, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, stream));
        PT_CUDA("shading records", launch_shading_records(pos.get<float>(), nrm.get<float>(), tan.get<float>(), uv.get<float>(), mid.get<uint32_t>(), n,
                                                          scene->shading.get<float4>(), stream));
        DeviceBuffer flags, index, scanScratch, lightCountDev;
        PT_TRY(flags.allocate(static_cast<size_t>(n) * 4));
        PT_TRY(index.allocate(static_cast<size_t>(n) * 4));
        PT_TRY(scanScratch.allocate(scan_scratch_elements(n) * 8));
        PT_TRY(lightCountDev.allocate(16));
        PT_CUDA("light build", launch_light_build(scene->shading.get<float4>(), scene->materials.get<MaterialDev>(), n,
                                                  flags.get<uint32_t>(), index.get<uint32_t>(), scanScratch.get<uint32_t>(), lightCountDev.get<uint32_t>(), stream));
        uint32_t lightCount = 0;
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&lightCount, lightCountDev.get<void>(), 4, cudaMemcpyDeviceToHost, stream));
        PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream));
        scene->lightCount = lightCount;
        if (lightCount > 0)
        {
            DeviceBuffer weights, powerWeights, powerScratch, prefix, stackIndex, stackValue;
            PT_TRY(scene->lights.allocate(static_cast<size_t>(lightCount) * 7 * sizeof(float4)));
            PT_TRY(scene->bins.allocate(static_cast<size_t>(lightCount) * sizeof(uint4)));
            PT_TRY(scene->binsPower.allocate(static_cast<size_t>(lightCount) * sizeof(uint4)));
            PT_TRY(weights.allocate(static_cast<size_t>(lightCount) * 8));
            PT_TRY(powerWeights.allocate(static_cast<size_t>(lightCount) * 8));
            PT_TRY(powerScratch.allocate(alias_power_scratch_bytes(lightCount)));
            PT_TRY(prefix.allocate(static_cast<size_t>(lightCount) * 8));
            PT_TRY(stackIndex.allocate(static_cast<size_t>(lightCount) * 8));
            PT_TRY(stackValue.allocate(static_cast<size_t>(lightCount) * 8));
            const MaterialTextures* tex = scene->textures.empty() ? nullptr : scene->materialTextures.get<MaterialTextures>();
            PT_CUDA("light records", launch_light_records(pos.get<float>(), scene->shading.get<float4>(), scene->materials.get<MaterialDev>(), tex,
                                                          n, flags.get<uint32_t>(), index.get<uint32_t>(), scene->lights.get<float4>(),
                                                          weights.get<double>(), powerWeights.get<double>(), stream));
            PT_CUDA("alias table", launch_alias_build(weights.get<double>(), lightCount, prefix.get<double>(), scanScratch.get<double>(),
                                                      scene->bins.get<uint4>(), stackIndex.get<uint32_t>(), stackValue.get<float>(), stream));
            PT_CUDA("power alias table", launch_alias_build_power(powerWeights.get<double>(), weights.get<double>(), lightCount,
                                                                  powerScratch.get<void>(), scene->binsPower.get<uint4>(), stream));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream));
        }
        const SceneEntry entry{0u, 0u, lightCount, 0u};
        PT_TRY(scene->entry.allocate(sizeof(SceneEntry)));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(scene->entry.get<void>(), &entry, sizeof(entry), cudaMemcpyHostToDevice, stream));
        PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream));
        scene->uploadSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tUpload).count();
        out = std::move(scene);
        return Status::Ok();
    }

    class Renderer
    {
    public:
        explicit Renderer(int device) : device_(device) {}
        ~Renderer()
        {
            StopRendering();
            releaseGraph();
            if (startEvent_) cudaEventDestroy(startEvent_);
            if (traceStart_) cudaEventDestroy(traceStart_);
            if (traceStop_) cudaEventDestroy(traceStop_);
            if (stopEvent_) cudaEventDestroy(stopEvent_);
            if (hostMapped_) cudaFreeHost(hostMapped_);
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
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            PT_CUDA("cudaStreamCreateWithFlags", cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
            PT_CUDA("cudaEventCreateWithFlags", cudaEventCreateWithFlags(&shadeFork_, cudaEventDisableTiming));
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                PT_CUDA("cudaStreamCreateWithFlags", cudaStreamCreateWithFlags(&shadeStreams_[m], cudaStreamNonBlocking));
                PT_CUDA("cudaEventCreateWithFlags", cudaEventCreateWithFlags(&shadeJoin_[m], cudaEventDisableTiming));
            }
            PT_CUDA("cudaEventCreate", cudaEventCreate(&startEvent_));
            PT_CUDA("cudaEventCreate", cudaEventCreate(&stopEvent_));
            PT_CUDA("cudaHostAlloc", cudaHostAlloc(&hostMapped_, 64, cudaHostAllocMapped));
            std::memset(hostMapped_, 0, 64);
            PT_CUDA("cudaHostGetDevicePointer", cudaHostGetDevicePointer(&hostMappedDev_, hostMapped_, 0));
            PT_TRY(job_.allocate(sizeof(JobView)));
            PT_TRY(counters_.allocate(sizeof(Counters)));
            PT_TRY(cursor_.allocate(64));
            return Status::Ok();
        }

        // ---------------------------------------------------------------- buffers
        Status InitializeRenderingBuffers(uint32_t width, uint32_t height)  // Renderer.cpp:265-290
        {
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            PT_TRY(ensurePool(kDefaultPool));
            PT_TRY(ensureFrame(width, height));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(framebuffer_.get<uint32_t>(), 0, static_cast<size_t>(width) * height * 4, stream_));
            PT_TRY(copyFrameToHost());
            return Status::Ok();
        }

        Status ensureFrame(uint32_t width, uint32_t height)
        {
            if (width == 0 || height == 0) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Frame size must be positive");
            const size_t pixels = static_cast<size_t>(width) * height;
            PT_TRY(accumulation_.allocate(pixels * sizeof(float4)));
            PT_TRY(framebuffer_.allocate(pixels * sizeof(uint32_t)));
            {
                std::scoped_lock lock(frameMutex_);
                hostFrame_.resize(pixels);
            }
            width_ = width;
            height_ = height;
            return Status::Ok();
        }

        Status ensurePool(uint32_t pool)
        {
            if (pool == pool_ && slotT_.get<float4>()) return Status::Ok();
            releaseGraph();
            const size_t P = pool;
            for (int q = 0; q < 2; q++)
            {
                PT_TRY(rayO_[q].allocate(P * 16));
                PT_TRY(rayD_[q].allocate(P * 16));
            }
            PT_TRY(matQ_.allocate(P * 48 * kModelCount));
            PT_TRY(shO_.allocate(P * 16));
            PT_TRY(shD_.allocate(P * 16));
            PT_TRY(shL_.allocate(P * 16));
            PT_TRY(regen_.allocate(P * 4));
            PT_TRY(regenBits_.allocate((P + 31) / 32 * 4));
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(regenBits_.get<void>(), 0, (P + 31) / 32 * 4, stream_));
            PT_TRY(slotT_.allocate(P * 16));
            PT_TRY(slotL_.allocate(P * 16));
            PT_TRY(slotSample_.allocate(P * 4));
            PT_TRY(queueLog_.allocate(static_cast<size_t>(kLogCapacity) * kQueueLogColumns * 4));
            pool_ = pool;
            return Status::Ok();
        }

        Wavefront wavefront(bool queues = false) const
        {
            Wavefront w{};
            for (int q = 0; q < 2; q++)
            {
                w.rayO[q] = rayO_[q].get<float4>();
                w.rayD[q] = rayD_[q].get<float4>();
            }
            for (uint32_t m = 0; m < kModelCount; m++) w.matQ[m] = matQ_.get<float4>() + static_cast<size_t>(m) * pool_ * 3;
            w.shO = shO_.get<float4>();
            w.shD = shD_.get<float4>();
            w.shL = shL_.get<float4>();
            w.regen = regen_.get<uint32_t>();
            w.regenBits = queues ? nullptr : regenBits_.get<uint32_t>();
            w.slotT = slotT_.get<float4>();
            w.slotL = slotL_.get<float4>();
            w.slotSample = slotSample_.get<uint32_t>();
            w.capacity = pool_;
            w.logCapacity = kLogCapacity;
            w.queueLog = queueLog_.get<uint32_t>();
            w.ctr = counters_.get<Counters>();
            w.cancel = static_cast<const volatile uint32_t*>(hostMappedDev_);
            w.progress = reinterpret_cast<volatile unsigned long long*>(static_cast<char*>(hostMappedDev_) + 16);
            return w;
        }

        // ---------------------------------------------------------------- scene
        Status InitializeSceneBuffers(const gpt_scene_desc& d)  // Renderer.cpp:292-306
        {
            if (rendering_.load()) return Status::Err(GPT_ERR_STATE, "Cannot upload a scene while rendering");
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            std::unique_ptr<SceneGpu> scene;
            PT_TRY(BuildScene(d, stream_, scene, true, bvhBuild_ == GPT_BVH_BUILD_DEVICE));
            releaseGraph();
            scene->version = ++sceneVersion_;
            scene_ = std::move(scene);
            return Status::Ok();
        }

        // ---------------------------------------------------------------- frame
        struct FrameConfig
        {
            uint32_t width, height, spp, spa, depth, nee, pool;
            uint64_t totalSamples;
            int traceThreads;
            uint32_t refill, refillShadow;
            int occupancy;
            uint32_t bvh;
            bool queues;   // the reference's wavefront structure (regeneration queue, shading in sequence)
            uint32_t maxIterations;  // 0 = automatic
            uint32_t stack;          // traversal stack entries chosen by the caller, 0 = the tree's depth
        };

        Status resolveConfig(const gpt_render_settings& s, FrameConfig& c) const
        {
            // clamps of StartSimulation (Renderer.cpp:340-344, 366-367)
            c.width = std::min(std::max(s.width, 1u), 7680u);
            c.height = std::min(std::max(s.height, 1u), 4320u);
            const uint32_t spp = std::min(std::max(s.samples_per_pixel, 1u), 10'000'000u);
            c.spa = static_cast<uint32_t>(std::sqrt(static_cast<double>(spp)));
            c.spp = c.spa * c.spa;
            c.depth = std::min(std::max(s.path_depth, 1u), 100u);
            c.nee = s.use_nee ? 1u : 0u;
            c.pool = s.pool_size ? std::min(s.pool_size, kMaxPool) : kDefaultPool;
            c.totalSamples = static_cast<uint64_t>(c.spp) * c.width * c.height;
            if (s.max_samples && s.max_samples < c.totalSamples) c.totalSamples = s.max_samples;
            if (c.totalSamples >= 0xFFFFFFFFull)
                return Status::Err(GPT_ERR_CAPACITY, "A frame is limited to 2^32-1 samples (per-sample radiance capture)");
            if (s.rng_policy != GPT_RNG_PHILOX && s.rng_policy != GPT_RNG_PCG32)
                return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown rng_policy");
            if (s.light_sampling != GPT_LIGHTS_AREA && s.light_sampling != GPT_LIGHTS_POWER)
                return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown light_sampling");
            c.traceThreads = s.trace_block ? static_cast<int>(s.trace_block) : 128;
            if (c.traceThreads != 64 && c.traceThreads != 128) c.traceThreads = 128;
            // bits 0-7: closest-hit traversal (0 = 16); bits 8-15: shadow rays (0 = half the closest-hit value)
            c.refill = (s.trace_refill & 0xFFu) ? std::min(32u, std::max(1u, s.trace_refill & 0xFFu)) : 16u;
            c.refillShadow = ((s.trace_refill >> 8) & 0xFFu) ? std::min(32u, std::max(1u, (s.trace_refill >> 8) & 0xFFu))
                                                              : std::max(1u, c.refill / 2u);
            c.occupancy = s.trace_occupancy == 0 ? 10 : (s.trace_occupancy >= 12 ? 12 : (s.trace_occupancy >= 10 ? 10 : 1));
            if (s.bvh_format > GPT_BVH2_FP32) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown BVH format");
            c.bvh = s.bvh_format == GPT_BVH2_FP32 ? kBvh2Fp32 : kBvh8Quantised;
            if (c.bvh == kBvh2Fp32 && !scene_->nodeCount2)
                return Status::Err(GPT_ERR_STATE, "The scene has no binary BVH");
            if (s.wavefront_layout > GPT_WAVEFRONT_QUEUES) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown wavefront layout");
            c.queues = s.wavefront_layout == GPT_WAVEFRONT_QUEUES;
            c.maxIterations = s.max_iterations;
            if (s.trace_stack > kMaxStack) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "trace_stack above 64 entries");
            c.stack = s.trace_stack;
            return Status::Ok();
        }

        // The scene as the frame's kernels see it.
        SceneView frameView(const FrameConfig&) const { return scene_->view(); }

        void releaseGraph()
        {
            if (graphExec_) cudaGraphExecDestroy(graphExec_);
            if (graph_) cudaGraphDestroy(graph_);
            graphExec_ = nullptr;
            graph_ = nullptr;
        }

        Status buildGraph(const FrameConfig& c)
        {
            releaseGraph();
            int sms = 0;
            PT_CUDA("cudaDeviceGetAttribute", cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
            const SceneView sv = frameView(c);
            const Wavefront wf = wavefront(c.queues);
            const JobView* jobDev = job_.get<JobView>();
            // prologue and resolve as captured child graphs
            cudaGraph_t pro = nullptr, res = nullptr;
            PT_CUDA("cudaStreamBeginCapture", cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            cudaError_t le = launch_frame_prologue(wf, jobDev, c.pool, sms * 8, stream_);
            cudaError_t ce = cudaStreamEndCapture(stream_, &pro);
            PT_CUDA("prologue launch", le);
            PT_CUDA("cudaStreamEndCapture", ce);
            PT_CUDA("cudaStreamBeginCapture", cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            le = launch_resolve(jobDev, accumulation_.get<float4>(), framebuffer_.get<uint32_t>(), sms * 8, stream_);
            ce = cudaStreamEndCapture(stream_, &res);
            PT_CUDA("resolve launch", le);
            PT_CUDA("cudaStreamEndCapture", ce);

            PT_CUDA("cudaGraphCreate", cudaGraphCreate(&graph_, 0));
            cudaGraphNode_t proNode, whileNode, resNode;
            PT_CUDA("cudaGraphAddChildGraphNode", cudaGraphAddChildGraphNode(&proNode, graph_, nullptr, 0, pro));
            cudaGraphConditionalHandle handle;
            PT_CUDA("cudaGraphConditionalHandleCreate", cudaGraphConditionalHandleCreate(&handle, graph_, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            PT_CUDA("cudaGraphAddNode", cudaGraphAddNode(&whileNode, graph_, &proNode, 1, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            IterationLaunch L{};
            L.scene = sv;
            L.wf = wf;
            L.job = jobDev;
            L.scenes = scene_->entry.get<SceneEntry>();
            L.handle = handle;
            for (uint32_t m = 0; m < kModelCount; m++) L.modelPresent[m] = scene_->modelPresent[m];
            L.nee = c.nee != 0;
            L.traceThreads = c.traceThreads;
            L.occupancy = c.occupancy;
            L.traceBlocks = trace_grid_blocks(device_, c.traceThreads, sv.depth, c.occupancy, c.bvh);
            L.refill = c.refill;
            L.refillShadow = c.refillShadow;
            L.bvhFormat = c.bvh;
            L.stackCap = static_cast<int>(c.stack);
            L.shadeFork = c.queues ? nullptr : shadeFork_;
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                L.shadeJoin[m] = shadeJoin_[m];
                L.shadeStreams[m] = shadeStreams_[m];
            }
            L.shadeBlocks = sms * 8;
            L.sms = sms;
            L.graphLoop = true;
            PT_CUDA("cudaStreamBeginCaptureToGraph", cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            le = launch_iteration(L, stream_);
            ce = cudaStreamEndCapture(stream_, &body);
            PT_CUDA("iteration launch", le);
            PT_CUDA("cudaStreamEndCapture", ce);
            PT_CUDA("cudaGraphAddChildGraphNode", cudaGraphAddChildGraphNode(&resNode, graph_, &whileNode, 1, res));
            cudaGraphDestroy(pro);
            cudaGraphDestroy(res);
            PT_CUDA("cudaGraphInstantiate", cudaGraphInstantiate(&graphExec_, graph_, 0));
            graphKey_ = key(c);
            return Status::Ok();
        }

        // The reference's host-driven structure (Renderer.cpp:517-623): every kernel is an ordinary
        // launch and the host reads the loop condition after each iteration. Used for per-kernel
        // profiling (ncu cannot profile nodes of graphs with conditional nodes), for CUDA-event
        // timing of the traversal kernel, and as the host-driven baseline of the graph loop.
        Status hostLoop(const FrameConfig& c, uint32_t maxIterations, float& traceEventMs)
        {
            int sms = 0;
            PT_CUDA("cudaDeviceGetAttribute", cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
            const SceneView sv = frameView(c);
            const Wavefront wf = wavefront(c.queues);
            const JobView* jobDev = job_.get<JobView>();
            if (!traceStart_) PT_CUDA("cudaEventCreate", cudaEventCreate(&traceStart_));
            if (!traceStop_) PT_CUDA("cudaEventCreate", cudaEventCreate(&traceStop_));
            IterationLaunch L{};
            L.scene = sv;
            L.wf = wf;
            L.job = jobDev;
            L.scenes = scene_->entry.get<SceneEntry>();
            L.handle = 0;
            for (uint32_t m = 0; m < kModelCount; m++) L.modelPresent[m] = scene_->modelPresent[m];
            L.nee = c.nee != 0;
            L.traceThreads = c.traceThreads;
            L.occupancy = c.occupancy;
            L.traceBlocks = trace_grid_blocks(device_, c.traceThreads, sv.depth, c.occupancy, c.bvh);
            L.refill = c.refill;
            L.refillShadow = c.refillShadow;
            L.bvhFormat = c.bvh;
            L.stackCap = static_cast<int>(c.stack);
            L.shadeFork = c.queues ? nullptr : shadeFork_;
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                L.shadeJoin[m] = shadeJoin_[m];
                L.shadeStreams[m] = shadeStreams_[m];
            }
            L.shadeBlocks = sms * 8;
            L.sms = sms;
            L.graphLoop = false;
            L.traceStart = traceStart_;
            L.traceStop = traceStop_;
            volatile uint32_t* doneHost = reinterpret_cast<volatile uint32_t*>(static_cast<char*>(hostMapped_) + 32);
            traceEventMs = 0.0f;
            PT_CUDA("cudaEventRecord", cudaEventRecord(startEvent_, stream_));
            PT_CUDA("prologue", launch_frame_prologue(wf, jobDev, c.pool, sms * 8, stream_));
            for (uint32_t it = 0; it <= maxIterations; it++)
            {
                PT_CUDA("iteration", launch_iteration(L, stream_));
                PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(const_cast<uint32_t*>(doneHost), &counters_.get<Counters>()->done, 4, cudaMemcpyDeviceToHost, stream_));
                PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
                float ms = 0.0f;
                PT_CUDA("cudaEventElapsedTime", cudaEventElapsedTime(&ms, traceStart_, traceStop_));
                traceEventMs += ms;
                if (*doneHost) break;
            }
            PT_CUDA("resolve", launch_resolve(jobDev, accumulation_.get<float4>(), framebuffer_.get<uint32_t>(), sms * 8, stream_));
            PT_CUDA("cudaEventRecord", cudaEventRecord(stopEvent_, stream_));
            return Status::Ok();
        }

        std::string key(const FrameConfig& c) const
        {
            char buf[256];
            std::snprintf(buf, sizeof(buf), "%llu/%u/%u/%d/%u/%d/%u/%d/%u/%u/%u/%p/%p", static_cast<unsigned long long>(scene_->version), c.pool,
                          c.nee, c.traceThreads, c.refill | (c.refillShadow << 8), c.occupancy, c.bvh, c.queues ? 1 : 0, c.stack, width_, height_,
                          static_cast<void*>(accumulation_.get<void>()),
                          static_cast<void*>(framebuffer_.get<void>()));
            return buf;
        }

        Status RenderFrame(const gpt_device_camera& cam, const gpt_render_settings& s, gpt_frame_stats* stats, bool copyToHost = true)
        {
            if (!scene_) return Status::Err(GPT_ERR_NO_SCENE, "No scene has been uploaded");
            NvtxRange range("gpt render frame");
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            FrameConfig c;
            PT_TRY(resolveConfig(s, c));
            PT_TRY(ensurePool(c.pool));
            if (c.width != width_ || c.height != height_ || !framebuffer_.get<void>() || !accumulation_.get<void>())
            {
                releaseGraph();
                PT_TRY(ensureFrame(c.width, c.height));
            }
            const size_t radianceBytes = static_cast<size_t>(c.totalSamples) * 12;
            if (radianceBytes > sampleRadiance_.bytes())
            {
                releaseGraph();
                PT_TRY(sampleRadiance_.allocate(radianceBytes));
            }
            JobView jv{};
            std::memcpy(jv.camera, &cam, sizeof(jv.camera));
            jv.width = c.width;
            jv.height = c.height;
            jv.spp = c.spp;
            jv.spa = c.spa;
            jv.depthLimit = c.depth;
            jv.nee = c.nee;
            jv.totalSamples = c.totalSamples;
            jv.sampleRadiance = sampleRadiance_.get<float>();
            jv.rngOffset = s.rng_offset;
            jv.rngPolicy = s.rng_policy;
            jv.lightMode = s.light_sampling;
            const uint64_t rounds = (c.totalSamples + c.pool - 1) / c.pool;
            jv.maxIterations = static_cast<uint32_t>(std::min<uint64_t>(0xFFFFFFF0ull, static_cast<uint64_t>(c.depth) * (rounds + 2) + 64));
            if (c.maxIterations) jv.maxIterations = std::min(jv.maxIterations, c.maxIterations);
            hostJob_ = jv;
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(job_.get<void>(), &hostJob_, sizeof(JobView), cudaMemcpyHostToDevice, stream_));
            lastTotalSamples_ = c.totalSamples;
            lastPixels_ = static_cast<size_t>(c.width) * c.height;
            float traceEventMs = 0.0f;
            if (s.loop_mode == GPT_LOOP_HOST)
                PT_TRY(hostLoop(c, jv.maxIterations, traceEventMs));
            else
            {
                if (!graphExec_ || graphKey_ != key(c)) PT_TRY(buildGraph(c));
                PT_CUDA("cudaEventRecord", cudaEventRecord(startEvent_, stream_));
                PT_CUDA("cudaGraphLaunch", cudaGraphLaunch(graphExec_, stream_));
                PT_CUDA("cudaEventRecord", cudaEventRecord(stopEvent_, stream_));
            }
            Counters ctr{};
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&hostCounters_, counters_.get<void>(), sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
            if (copyToHost) PT_TRY(copyFrameToHost());
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
            ctr = hostCounters_;
            float ms = 0.0f;
            PT_CUDA("cudaEventElapsedTime", cudaEventElapsedTime(&ms, startEvent_, stopEvent_));
            if (ctr.errorFlags) return Status::Err(GPT_ERR_DEVICE_FAULT, "Traversal reported error flags " + std::to_string(ctr.errorFlags));
            lastIterations_ = ctr.iteration;
            if (stats)
            {
                *stats = gpt_frame_stats{};
                stats->iterations = ctr.iteration;
                uint32_t models = 0;
                for (uint32_t m = 0; m < kModelCount; m++) models += scene_->modelPresent[m] ? 1u : 0u;
                const uint32_t perIteration = 1u + models + (c.nee && scene_->lightCount ? 1u : 0u) + 2u;
                stats->kernel_launches = 2u + ctr.iteration * perIteration + 1u;
                stats->samples = ctr.launched;
                stats->rays = ctr.raysTraced;
                stats->shadow_rays = ctr.shadowRaysTraced;
                for (int k = 0; k < 2; k++)
                {
                    stats->node_visits[k] = ctr.nodeVisits[k];
                    stats->triangle_tests[k] = ctr.triTests[k];
                }
                stats->device_ms = ms;
                stats->trace_event_ms = traceEventMs;
                for (int p = 0; p < 4; p++) stats->phase_ms[p] = static_cast<float>(static_cast<double>(ctr.tAccum[p]) * 1e-6);
            }
            return Status::Ok();
        }

        // Measured choice of the frame's tuning knobs for a workload: every candidate renders a reduced
        // frame (the whole image, so all of the scene is represented) twice, and the lowest device time
        // per sample wins. A pool candidate's trial frame has the smallest square sample count per pixel
        // (at least 4, at most the frame's own) that gives two pool-fulls of samples, so the pool stays
        // full for most of the trial as it does in the real frame. Results do not depend on the knobs;
        // only speed does.
        Status Autotune(const gpt_device_camera& cam, const gpt_render_settings& base, gpt_render_settings& best, float& bestMs,
                        uint32_t& tried)
        {
            if (!scene_) return Status::Err(GPT_ERR_NO_SCENE, "No scene has been uploaded");
            NvtxRange range("gpt autotune");
            gpt_render_settings trial = base;
            trial.max_samples = 0;
            trial.loop_mode = GPT_LOOP_GRAPH;
            const uint64_t pixels = static_cast<uint64_t>(std::max(base.width, 1u)) * std::max(base.height, 1u);
            const uint32_t spp = std::max(base.samples_per_pixel, 1u);
            const uint32_t pools[] = {1u << 20, 2u << 20, 4u << 20, 8u << 20, 16u << 20};
            const uint32_t occupancies[] = {1u, 10u, 12u};
            const uint32_t refills[] = {8u, 16u};
            const uint32_t blocks[] = {64u, 128u};
            const auto trialSpp = [&](uint32_t pool)
            {
                uint32_t side = 2;
                while (side * side < spp && static_cast<uint64_t>(side) * side * pixels < 2ull * pool) side++;
                return std::min(side * side, spp);
            };
            const auto perSample = [&](const gpt_render_settings& t, float& score) -> Status
            {
                score = 1e30f;
                for (int rep = 0; rep < 2; rep++)
                {
                    gpt_frame_stats st{};
                    PT_TRY(RenderFrame(cam, t, &st, false));
                    if (rep && st.samples) score = static_cast<float>(static_cast<double>(st.device_ms) / static_cast<double>(st.samples));
                }
                return Status::Ok();
            };
            best = base;
            bestMs = 1e30f;  // device ms per sample of the best trial until the end, then per frame of the base settings
            tried = 0;
            // the frame's own sample count bounds the useful pool size
            const uint64_t frameSamples = pixels * spp;
            for (uint32_t pool : pools)
            {
                if (pool > 2 * frameSamples && pool != pools[0]) continue;
                trial.samples_per_pixel = trialSpp(pool);
                for (uint32_t occ : occupancies)
                    for (uint32_t refill : refills)
                        for (uint32_t tb : blocks)
                        {
                            trial.pool_size = pool;
                            trial.trace_occupancy = occ;
                            trial.trace_refill = refill;
                            trial.trace_block = tb;
                            float score = 1e30f;
                            PT_TRY(perSample(trial, score));
                            tried++;
                            if (score < bestMs)
                            {
                                bestMs = score;
                                best = base;
                                best.pool_size = pool;
                                best.trace_occupancy = occ;
                                best.trace_refill = refill;
                                best.trace_block = tb;
                            }
                        }
            }
            // shadow rays tune their own refill threshold with the other knobs fixed
            const uint32_t closestRefill = best.trace_refill & 0xFFu;
            for (uint32_t shadowRefill : {2u, 4u, 8u, 16u})
            {
                trial = best;
                trial.samples_per_pixel = trialSpp(best.pool_size);
                trial.max_samples = 0;
                trial.loop_mode = GPT_LOOP_GRAPH;
                trial.trace_refill = closestRefill | (shadowRefill << 8);
                float score = 1e30f;
                PT_TRY(perSample(trial, score));
                tried++;
                if (score < bestMs)
                {
                    bestMs = score;
                    best.trace_refill = trial.trace_refill;
                }
            }
            bestMs = static_cast<float>(static_cast<double>(bestMs) * static_cast<double>(frameSamples));
            return Status::Ok();
        }

        Status copyFrameToHost()
        {
            std::scoped_lock lock(frameMutex_);
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(hostFrame_.data(), framebuffer_.get<void>(), hostFrame_.size() * 4, cudaMemcpyDeviceToHost, stream_));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(stream_));
            return Status::Ok();
        }

        Status Clear(uint8_t r, uint8_t g, uint8_t b, uint8_t a)  // Renderer.cpp:322-328, 677-687
        {
            if (rendering_.load()) return Status::Err(GPT_ERR_STATE, "Cannot clear renderer while rendering");
            if (!framebuffer_.get<void>()) return Status::Err(GPT_ERR_STATE, "Rendering buffers are not initialized");
            const uint32_t v = static_cast<uint32_t>(r) | (static_cast<uint32_t>(g) << 8) | (static_cast<uint32_t>(b) << 16) | (static_cast<uint32_t>(a) << 24);
            PT_CUDA("Clear", launch_clear(framebuffer_.get<uint32_t>(), width_ * height_, v, stream_));
            return copyFrameToHost();
        }

        // ---------------------------------------------------------------- batch traversal
        Status Intersect(const float* rays, uint32_t n, uint32_t* tri, float* uvt, uint8_t* occ, cudaStream_t s, uint32_t bvh = kBvh8Quantised)
        {
            if (!scene_) return Status::Err(GPT_ERR_NO_SCENE, "No scene has been uploaded");
            if (n == 0) return Status::Ok();
            if (!rays || (!occ && (!tri || !uvt))) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Null ray or output pointer");
            PT_CUDA("cudaSetDevice", cudaSetDevice(device_));
            cudaStream_t st = s ? s : stream_;
            uint32_t* cursor = cursor_.get<uint32_t>();
            PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(cursor, 0, 8, st));
            const SceneView sv = scene_->view();
            if (bvh == kBvh2Fp32 && !sv.nodes2) return Status::Err(GPT_ERR_STATE, "The scene has no binary BVH");
            const int blocks = trace_grid_blocks(device_, 128, sv.depth, 1, bvh);
            PT_CUDA("intersect", launch_batch_trace(sv, 0u, rays, n, cursor, tri, uvt, occ, blocks, 128, cursor + 1, st, bvh));
            uint32_t err = 0;
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&err, cursor + 1, 4, cudaMemcpyDeviceToHost, st));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(st));
            if (err) return Status::Err(GPT_ERR_DEVICE_FAULT, "Traversal reported error flags " + std::to_string(err));
            return Status::Ok();
        }

        // ---------------------------------------------------------------- simulation thread
        Status StartSimulation(uint32_t width, uint32_t height, float fovY, const gpt_motion_state* states, uint32_t count, uint32_t spp,
                               uint32_t depth, const char* outputFolder, bool nee)
        {
            width = std::min(std::max(width, 1u), 7680u);
            height = std::min(std::max(height, 1u), 4320u);
            spp = std::min(std::max(spp, 1u), 10'000'000u);
            depth = std::min(std::max(depth, 1u), 100u);
            if (rendering_.load()) return Status::Err(GPT_ERR_STATE, "Renderer is already rendering");
            if (!scene_) return Status::Err(GPT_ERR_NO_SCENE, "No scene has been uploaded");
            if (worker_.joinable()) worker_.join();
            {
                std::scoped_lock lock(errorMutex_);
                lastError_.clear();
                hasError_ = false;
            }
            if (width != width_ || height != height_) PT_TRY(ensureFrame(width, height));
            motion_.assign(states, states + count);
            fovY_ = fovY;
            outputFolder_ = outputFolder ? outputFolder : "";
            simSettings_ = gpt_render_settings{};
            simSettings_.width = width;
            simSettings_.height = height;
            simSettings_.samples_per_pixel = spp;
            simSettings_.path_depth = depth;
            simSettings_.use_nee = nee ? 1 : 0;
            const uint32_t spa = static_cast<uint32_t>(std::sqrt(static_cast<double>(spp)));
            totalSamples_ = static_cast<uint64_t>(spa) * spa * width * height;
            totalFrames_ = count;
            doneFrames_.store(0);
            return launchWorker(0);
        }

        Status ResumeSimulation(uint32_t startFrame)  // Renderer.cpp:401-427
        {
            if (rendering_.load()) return Status::Err(GPT_ERR_STATE, "Renderer is already rendering");
            if (startFrame >= motion_.size()) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "Start frame is out of range - nothing to render");
            if (worker_.joinable()) worker_.join();
            doneFrames_.store(startFrame);
            return launchWorker(startFrame);
        }

        Status launchWorker(uint32_t startFrame)
        {
            *static_cast<volatile uint32_t*>(hostMapped_) = 0u;
            stopRequested_.store(false);
            rendering_.store(true);
            try
            {
                worker_ = std::thread([this, startFrame]() { SimulationLoop(startFrame); });
            }
            catch (...)
            {
                rendering_.store(false);
                return Status::Err(GPT_ERR_STATE, "Failed to start render thread");
            }
            return Status::Ok();
        }

        void SimulationLoop(uint32_t startFrame)  // Renderer.cpp:442-466
        {
            cudaSetDevice(device_);
            const float aspect = static_cast<float>(simSettings_.width) / static_cast<float>(simSettings_.height);
            const int digits = static_cast<int>(std::max<size_t>(4, std::to_string(totalFrames_ ? totalFrames_ - 1 : 0).size()));
            for (uint32_t frame = startFrame; frame < totalFrames_; frame++)
            {
                gpt_device_camera cam;
                gpt_make_device_camera(fovY_, aspect, &motion_[frame], &cam);
                Status st = RenderFrame(cam, simSettings_, nullptr, true);
                if (st.ok() && !stopRequested_.load() && !outputFolder_.empty())
                {
                    char name[64];
                    std::snprintf(name, sizeof(name), "frame_%0*u.png", digits, doneFrames_.load());
                    std::error_code ec;
                    std::filesystem::create_directories(outputFolder_, ec);
                    std::vector<uint32_t> copy;
                    {
                        std::scoped_lock lock(frameMutex_);
                        copy = hostFrame_;
                    }
                    if (!WritePng((std::filesystem::path(outputFolder_) / name).string(), copy.data(), simSettings_.width, simSettings_.height))
                        st = Status::Err(GPT_ERR_STATE, "Failed to save rendered frame");
                }
                if (!st.ok())
                {
                    cudaDeviceSynchronize();
                    std::scoped_lock lock(errorMutex_);
                    lastError_ = st.message;
                    hasError_ = true;
                    break;
                }
                if (stopRequested_.load()) break;
                doneFrames_.fetch_add(1);
            }
            rendering_.store(false);
        }

        Status StopRendering()  // Renderer.cpp:429-440
        {
            if (worker_.joinable())
            {
                stopRequested_.store(true);
                if (hostMapped_) *static_cast<volatile uint32_t*>(hostMapped_) = 1u;
                worker_.join();
            }
            if (stream_) cudaStreamSynchronize(stream_);
            // the cancellation request applies to the stopped simulation only
            if (hostMapped_) *static_cast<volatile uint32_t*>(hostMapped_) = 0u;
            rendering_.store(false);
            return Status::Ok();
        }

        uint64_t DoneSamples() const
        {
            if (!hostMapped_) return 0;
            if (rendering_.load())
                return *reinterpret_cast<const volatile unsigned long long*>(static_cast<const char*>(hostMapped_) + 16);
            return doneFrames_.load() >= totalFrames_ && totalFrames_ ? totalSamples_ : 0;
        }

        void SetError(const Status& s)
        {
            std::scoped_lock lock(errorMutex_);
            lastError_ = s.message;
            hasError_ = true;
        }

        int device_;
        cudaStream_t stream_ = nullptr;
        cudaEvent_t startEvent_ = nullptr, stopEvent_ = nullptr;
        cudaEvent_t traceStart_ = nullptr, traceStop_ = nullptr;
        cudaEvent_t shadeFork_ = nullptr;
        cudaEvent_t shadeJoin_[kModelCount] = {};
        cudaStream_t shadeStreams_[kModelCount] = {};
        void* hostMapped_ = nullptr;
        void* hostMappedDev_ = nullptr;
        static constexpr uint32_t kDefaultPool = 1u << 20;
        static constexpr uint32_t kLogCapacity = 1u << 16;
        uint32_t pool_ = 0;
        DeviceBuffer rayO_[2], rayD_[2], matQ_, shO_, shD_, shL_, regen_, regenBits_, slotT_, slotL_, slotSample_, queueLog_;
        DeviceBuffer counters_, job_, cursor_, accumulation_, framebuffer_, sampleRadiance_;
        JobView hostJob_{};
        Counters hostCounters_{};
        std::unique_ptr<SceneGpu> scene_;
        uint64_t sceneVersion_ = 0;
        uint32_t width_ = 0, height_ = 0;
        std::vector<uint32_t> hostFrame_;
        std::mutex frameMutex_;
        cudaGraph_t graph_ = nullptr;
        cudaGraphExec_t graphExec_ = nullptr;
        std::string graphKey_;
        uint64_t lastTotalSamples_ = 0;
        size_t lastPixels_ = 0;
        uint32_t lastIterations_ = 0;
        // simulation
        std::thread worker_;
        std::atomic<bool> rendering_{false}, stopRequested_{false};
        std::atomic<uint32_t> doneFrames_{0};
        uint32_t totalFrames_ = 0;
        uint64_t totalSamples_ = 0;
        std::vector<gpt_motion_state> motion_;
        float fovY_ = 0.0f;
        std::string outputFolder_;
        gpt_render_settings simSettings_{};
        mutable std::mutex errorMutex_;
        std::string lastError_;
        bool hasError_ = false;
        uint32_t bvhBuild_ = GPT_BVH_BUILD_HOST;  // where the next scene upload builds its BVH8
    };
}

struct gpt_renderer
{
    std::unique_ptr<pt::Renderer> impl;
};

namespace
{
    int Report(gpt_renderer* r, const pt::Status& s)
    {
        if (!s.ok() && r && r->impl) r->impl->SetError(s);
        return s.code;
    }

    int CopyMessage(const std::string& m, char* buffer, size_t length)
    {
        if (buffer && length)
        {
            const size_t n = std::min(length - 1, m.size());
            std::memcpy(buffer, m.data(), n);
            buffer[n] = '\0';
        }
        return 1;
    }
}

extern "C"
{
    const char* gpt_status_string(int status)
    {
        switch (status)
        {
            case GPT_OK: return "ok";
            case GPT_ERR_INVALID_ARGUMENT: return "invalid argument";
            case GPT_ERR_CUDA: return "CUDA error";
            case GPT_ERR_OUT_OF_MEMORY: return "out of device memory";
            case GPT_ERR_STATE: return "invalid renderer state";
            case GPT_ERR_NO_SCENE: return "no scene uploaded";
            case GPT_ERR_CAPACITY: return "size above a documented limit";
            case GPT_ERR_TIMEOUT: return "bounded wait timed out";
            case GPT_ERR_DEVICE_FAULT: return "kernel reported an error flag";
            default: return "unknown status";
        }
    }

    int gpt_create(gpt_renderer** out, int device)
    {
        if (!out) return GPT_ERR_INVALID_ARGUMENT;
        *out = nullptr;
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return GPT_ERR_CUDA;
        auto r = std::make_unique<gpt_renderer>();
        r->impl = std::make_unique<pt::Renderer>(device);
        pt::Status s = r->impl->Init();
        if (!s.ok()) return s.code;
        *out = r.release();
        return GPT_OK;
    }

    void gpt_destroy(gpt_renderer* renderer) { delete renderer; }

    int gpt_init_rendering_buffers(gpt_renderer* r, uint32_t width, uint32_t height)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->InitializeRenderingBuffers(width, height));
    }

    int gpt_init_scene_buffers(gpt_renderer* r, const gpt_scene_desc* scene)
    {
        if (!r || !scene) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->InitializeSceneBuffers(*scene));
    }

    int gpt_clear(gpt_renderer* r, uint8_t red, uint8_t green, uint8_t blue, uint8_t alpha)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->Clear(red, green, blue, alpha));
    }

    int gpt_start_simulation(gpt_renderer* r, uint32_t width, uint32_t height, float fov_y, const gpt_motion_state* states, uint32_t count,
                             uint32_t spp, uint32_t depth, const char* output_folder, int use_nee)
    {
        if (!r || (!states && count)) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->StartSimulation(width, height, fov_y, states, count, spp, depth, output_folder, use_nee != 0));
    }

    int gpt_resume_simulation(gpt_renderer* r, uint32_t start_frame)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->ResumeSimulation(start_frame));
    }

    int gpt_stop_rendering(gpt_renderer* r)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->StopRendering());
    }

    int gpt_is_rendering(const gpt_renderer* r) { return r && r->impl->rendering_.load() ? 1 : 0; }
    uint32_t gpt_get_done_frames(const gpt_renderer* r) { return r ? r->impl->doneFrames_.load() : 0; }
    uint32_t gpt_get_total_frames(const gpt_renderer* r) { return r ? r->impl->totalFrames_ : 0; }
    uint64_t gpt_get_done_samples(const gpt_renderer* r) { return r ? r->impl->DoneSamples() : 0; }
    uint64_t gpt_get_total_samples(const gpt_renderer* r) { return r ? r->impl->totalSamples_ : 0; }
    uint32_t gpt_get_width(const gpt_renderer* r) { return r ? r->impl->width_ : 0; }
    uint32_t gpt_get_height(const gpt_renderer* r) { return r ? r->impl->height_ : 0; }

    int gpt_lock_frame(gpt_renderer* r, const uint32_t** data, size_t* size, size_t* element_size)
    {
        if (!r || !data || !size || !element_size) return GPT_ERR_INVALID_ARGUMENT;
        r->impl->frameMutex_.lock();
        *data = r->impl->hostFrame_.data();
        *size = r->impl->hostFrame_.size();
        *element_size = sizeof(uint32_t);
        return GPT_OK;
    }

    int gpt_unlock_frame(gpt_renderer* r)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        r->impl->frameMutex_.unlock();
        return GPT_OK;
    }

    int gpt_peek_last_error(const gpt_renderer* r, char* buffer, size_t length)
    {
        if (!r) return 0;
        std::scoped_lock lock(r->impl->errorMutex_);
        if (!r->impl->hasError_) return 0;
        return CopyMessage(r->impl->lastError_, buffer, length);
    }

    int gpt_consume_last_error(gpt_renderer* r, char* buffer, size_t length)
    {
        if (!r) return 0;
        std::scoped_lock lock(r->impl->errorMutex_);
        if (!r->impl->hasError_) return 0;
        CopyMessage(r->impl->lastError_, buffer, length);
        r->impl->hasError_ = false;
        r->impl->lastError_.clear();
        return 1;
    }

    int gpt_render_frame(gpt_renderer* r, const gpt_device_camera* camera, const gpt_render_settings* settings, gpt_frame_stats* stats)
    {
        if (!r || !camera || !settings) return GPT_ERR_INVALID_ARGUMENT;
        if (r->impl->rendering_.load()) return Report(r, pt::Status::Err(GPT_ERR_STATE, "Renderer is already rendering"));
        *static_cast<volatile uint32_t*>(r->impl->hostMapped_) = 0u;  // a synchronous frame is never cancelled
        return Report(r, r->impl->RenderFrame(*camera, *settings, stats, true));
    }

    int gpt_read_framebuffer(gpt_renderer* r, uint32_t* rgba, size_t pixel_count)
    {
        if (!r || !rgba) return GPT_ERR_INVALID_ARGUMENT;
        std::scoped_lock lock(r->impl->frameMutex_);
        if (pixel_count > r->impl->hostFrame_.size()) return GPT_ERR_CAPACITY;
        std::memcpy(rgba, r->impl->hostFrame_.data(), pixel_count * 4);
        return GPT_OK;
    }

    int gpt_read_accumulation(gpt_renderer* r, float* out, size_t pixel_count)
    {
        if (!r || !out) return GPT_ERR_INVALID_ARGUMENT;
        if (pixel_count > r->impl->lastPixels_) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        cudaError_t e = cudaMemcpy(out, r->impl->accumulation_.get<void>(), pixel_count * 16, cudaMemcpyDeviceToHost);
        return Report(r, pt::CudaStatus("cudaMemcpy", e));
    }

    int gpt_read_accumulation_fp64(gpt_renderer* r, double* out, size_t pixel_count)
    {
        if (!r || !out) return GPT_ERR_INVALID_ARGUMENT;
        if (pixel_count > r->impl->lastPixels_ || !r->impl->lastTotalSamples_) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        pt::DeviceBuffer sums;
        pt::Status st = sums.allocate(pixel_count * 3 * sizeof(double));
        if (!st.ok()) return Report(r, st);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->impl->device_);
        cudaError_t e = pt::launch_resolve_fp64(r->impl->job_.get<pt::JobView>(), sums.get<double>(), sms * 8, r->impl->stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out, sums.get<void>(), pixel_count * 3 * sizeof(double), cudaMemcpyDeviceToHost, r->impl->stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(r->impl->stream_);
        return Report(r, pt::CudaStatus("resolve fp64", e));
    }

    int gpt_copy_accumulation_device(gpt_renderer* r, float* dst, size_t pixel_count, void* stream)
    {
        if (!r || !dst) return GPT_ERR_INVALID_ARGUMENT;
        if (pixel_count > r->impl->lastPixels_) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : r->impl->stream_;
        cudaError_t e = cudaMemcpyAsync(dst, r->impl->accumulation_.get<void>(), pixel_count * 16, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(s);
        return Report(r, pt::CudaStatus("cudaMemcpyAsync", e));
    }

    int gpt_read_sample_radiance(gpt_renderer* r, float* out, uint64_t count)
    {
        if (!r || !out) return GPT_ERR_INVALID_ARGUMENT;
        if (count > r->impl->lastTotalSamples_) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        cudaError_t e = cudaMemcpy(out, r->impl->sampleRadiance_.get<void>(), static_cast<size_t>(count) * 12, cudaMemcpyDeviceToHost);
        return Report(r, pt::CudaStatus("cudaMemcpy", e));
    }

    int gpt_read_queue_log(gpt_renderer* r, uint32_t* rows, uint32_t max_rows, uint32_t* row_count)
    {
        if (!r || !rows || !row_count) return GPT_ERR_INVALID_ARGUMENT;
        const uint32_t n = std::min({max_rows, r->impl->lastIterations_, pt::Renderer::kLogCapacity});
        cudaSetDevice(r->impl->device_);
        cudaError_t e = cudaMemcpy(rows, r->impl->queueLog_.get<void>(), static_cast<size_t>(n) * pt::kQueueLogColumns * 4, cudaMemcpyDeviceToHost);
        *row_count = n;
        return Report(r, pt::CudaStatus("cudaMemcpy", e));
    }

    int gpt_intersect_closest(gpt_renderer* r, const float* rays, uint32_t n, uint32_t* tri_out, float* uvt_out, void* stream)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->Intersect(rays, n, tri_out, uvt_out, nullptr, static_cast<cudaStream_t>(stream)));
    }

    int gpt_intersect_any(gpt_renderer* r, const float* rays, uint32_t n, uint8_t* occluded_out, void* stream)
    {
        if (!r || !occluded_out) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->Intersect(rays, n, nullptr, nullptr, occluded_out, static_cast<cudaStream_t>(stream)));
    }

    int gpt_intersect_closest_binary(gpt_renderer* r, const float* rays, uint32_t n, uint32_t* tri_out, float* uvt_out, void* stream)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->Intersect(rays, n, tri_out, uvt_out, nullptr, static_cast<cudaStream_t>(stream), pt::kBvh2Fp32));
    }

    int gpt_intersect_any_binary(gpt_renderer* r, const float* rays, uint32_t n, uint8_t* occluded_out, void* stream)
    {
        if (!r || !occluded_out) return GPT_ERR_INVALID_ARGUMENT;
        return Report(r, r->impl->Intersect(rays, n, nullptr, nullptr, occluded_out, static_cast<cudaStream_t>(stream), pt::kBvh2Fp32));
    }

    int gpt_scene_info_binary(const gpt_renderer* r, uint32_t* node_count, uint32_t* depth)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        if (!r->impl->scene_) return GPT_ERR_NO_SCENE;
        if (node_count) *node_count = r->impl->scene_->nodeCount2;
        if (depth) *depth = r->impl->scene_->depth2;
        return GPT_OK;
    }

    int gpt_scene_upload_times(const gpt_renderer* r, double* bvh_build_seconds, double* upload_seconds)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        if (!r->impl->scene_) return GPT_ERR_NO_SCENE;
        if (bvh_build_seconds) *bvh_build_seconds = r->impl->scene_->bvhSeconds;
        if (upload_seconds) *upload_seconds = r->impl->scene_->uploadSeconds;
        return GPT_OK;
    }

    int gpt_set_bvh_build(gpt_renderer* r, uint32_t build)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        if (build > GPT_BVH_BUILD_DEVICE) return Report(r, pt::Status::Err(GPT_ERR_INVALID_ARGUMENT, "Unknown BVH build"));
        r->impl->bvhBuild_ = build;
        return GPT_OK;
    }

    int gpt_check_bvh(gpt_renderer* r, const float* positions, uint32_t triangle_count, uint64_t* containment_violations,
                      uint64_t* triangles_not_exactly_once, uint64_t* leaf_triangles)
    {
        if (!r || !positions) return GPT_ERR_INVALID_ARGUMENT;
        const pt::SceneGpu* sc = r->impl->scene_.get();
        if (!sc) return GPT_ERR_NO_SCENE;
        if (triangle_count != sc->triangleCount)
            return Report(r, pt::Status::Err(GPT_ERR_INVALID_ARGUMENT, "Triangle count differs from the uploaded scene"));
        pt::Bvh8 b;
        b.nodes.resize(sc->nodeCount);
        b.tris.resize(static_cast<size_t>(sc->triangleCount) * pt::kTriangleVec4);
        b.depth = sc->depth;
        cudaError_t e = cudaSetDevice(r->impl->device_);
        if (e == cudaSuccess) e = cudaMemcpy(b.nodes.data(), sc->nodes.get<void>(), b.nodes.size() * sizeof(pt::Node8), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(b.tris.data(), sc->tris.get<void>(), b.tris.size() * sizeof(float4), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return Report(r, pt::CudaStatus("cudaMemcpy", e));
        b.order.resize(sc->triangleCount);
        for (uint32_t k = 0; k < sc->triangleCount; k++)
        {
            const float w = b.tris[static_cast<size_t>(k) * pt::kTriangleVec4].w;  // input index of leaf position k
            std::memcpy(&b.order[k], &w, 4);
        }
        const pt::Bvh8Check c = pt::CheckBvh8(b, positions, triangle_count);
        if (containment_violations) *containment_violations = c.containmentViolations;
        if (triangles_not_exactly_once) *triangles_not_exactly_once = c.trianglesNotExactlyOnce;
        if (leaf_triangles) *leaf_triangles = c.leafTriangles;
        return GPT_OK;
    }

    int gpt_scene_info(const gpt_renderer* r, uint32_t* node_count, uint32_t* depth, uint32_t* light_count, uint32_t* triangle_count)
    {
        if (!r) return GPT_ERR_INVALID_ARGUMENT;
        if (!r->impl->scene_) return GPT_ERR_NO_SCENE;
        const pt::SceneGpu& s = *r->impl->scene_;
        if (node_count) *node_count = s.nodeCount;
        if (depth) *depth = s.depth;
        if (light_count) *light_count = s.lightCount;
        if (triangle_count) *triangle_count = s.triangleCount;
        return GPT_OK;
    }

    int gpt_read_alias_table(gpt_renderer* r, uint32_t* bins, uint32_t count)
    {
        if (!r || !bins) return GPT_ERR_INVALID_ARGUMENT;
        if (!r->impl->scene_) return GPT_ERR_NO_SCENE;
        if (count > r->impl->scene_->lightCount) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        cudaError_t e = cudaMemcpy(bins, r->impl->scene_->bins.get<void>(), static_cast<size_t>(count) * 16, cudaMemcpyDeviceToHost);
        return Report(r, pt::CudaStatus("cudaMemcpy", e));
    }

    int gpt_inject_allocation_failure(uint32_t after)
    {
        pt::g_allocationCountdown.store(after);
        return GPT_OK;
    }

    int gpt_read_alias_table_power(gpt_renderer* r, uint32_t* bins, uint32_t count)
    {
        if (!r || !bins) return GPT_ERR_INVALID_ARGUMENT;
        if (!r->impl->scene_) return GPT_ERR_NO_SCENE;
        if (count > r->impl->scene_->lightCount) return GPT_ERR_CAPACITY;
        cudaSetDevice(r->impl->device_);
        cudaError_t e = cudaMemcpy(bins, r->impl->scene_->binsPower.get<void>(), static_cast<size_t>(count) * 16, cudaMemcpyDeviceToHost);
        return Report(r, pt::CudaStatus("cudaMemcpy", e));
    }

    int gpt_bvh8_check(const gpt_scene_desc* d, uint32_t* node_count, uint32_t* depth, uint64_t* violations, uint64_t* misplaced)
    {
        if (!d || d->triangle_count == 0 || !d->positions || !d->material_ids || !d->materials) return GPT_ERR_INVALID_ARGUMENT;
        std::vector<uint32_t> models(d->triangle_count);
        for (uint32_t t = 0; t < d->triangle_count; t++)
        {
            if (d->material_ids[t] >= d->material_count) return GPT_ERR_INVALID_ARGUMENT;
            models[t] = d->materials[d->material_ids[t]].model;
        }
        try
        {
            pt::Bvh8 b = pt::BuildBvh8(d->positions, models.data(), d->triangle_count,
                                       static_cast<int>(std::max(1u, std::thread::hardware_concurrency())), true);
            pt::Bvh8Check c = pt::CheckBvh8(b, d->positions, d->triangle_count);
            if (node_count) *node_count = static_cast<uint32_t>(b.nodes.size());
            if (depth) *depth = b.depth;
            if (violations) *violations = c.containmentViolations;
            if (misplaced) *misplaced = c.trianglesNotExactlyOnce;
        }
        catch (const std::exception&)
        {
            return GPT_ERR_INVALID_ARGUMENT;
        }
        return GPT_OK;
    }

    int gpt_autotune(gpt_renderer* r, const gpt_device_camera* camera, const gpt_render_settings* base, gpt_render_settings* best,
                     float* best_ms, uint32_t* candidates)
    {
        if (!r || !camera || !base || !best) return GPT_ERR_INVALID_ARGUMENT;
        if (r->impl->rendering_.load()) return Report(r, pt::Status::Err(GPT_ERR_STATE, "Renderer is already rendering"));
        float ms = 0.0f;
        uint32_t tried = 0;
        const int rc = Report(r, r->impl->Autotune(*camera, *base, *best, ms, tried));
        if (best_ms) *best_ms = ms;
        if (candidates) *candidates = tried;
        return rc;
    }

    int gpt_abi_struct_sizes(uint32_t* sizes, uint32_t count)
    {
        if (!sizes) return GPT_ERR_INVALID_ARGUMENT;
        const uint32_t all[12] = {sizeof(gpt_material), sizeof(gpt_scene_desc), sizeof(gpt_device_camera), sizeof(gpt_motion_state),
                                  sizeof(gpt_render_settings), sizeof(gpt_frame_stats), sizeof(gpt_texture_desc), sizeof(gpt_server_config),
                                  sizeof(gpt_job_desc), sizeof(gpt_job_status), sizeof(gpt_server_stats), sizeof(gpt_motion_sample)};
        for (uint32_t i = 0; i < count && i < 12; i++) sizes[i] = all[i];
        return GPT_OK;
    }

    // MakeDeviceCamera (Renderer.cpp:237-257) with glm's quaternion rotation v + 2w(q x v) + 2 q x (q x v),
    // Forward = -Z, Right = +X, Up = +Y (Utils/Math/CoordinateSystem.hpp:8-10).
    int gpt_make_device_camera(float fov_y, float aspect, const gpt_motion_state* s, gpt_device_camera* out)
    {
        if (!s || !out) return GPT_ERR_INVALID_ARGUMENT;
        const float w = s->rotation[0], x = s->rotation[1], y = s->rotation[2], z = s->rotation[3];
        auto rotate = [&](float vx, float vy, float vz, float* o)
        {
            const float uvx = y * vz - z * vy, uvy = z * vx - x * vz, uvz = x * vy - y * vx;
            const float uuvx = y * uvz - z * uvy, uuvy = z * uvx - x * uvz, uuvz = x * uvy - y * uvx;
            o[0] = vx + ((uvx * w) + uuvx) * 2.0f;
            o[1] = vy + ((uvy * w) + uuvy) * 2.0f;
            o[2] = vz + ((uvz * w) + uuvz) * 2.0f;
        };
        float fwd[3], right[3], up[3];
        rotate(0.0f, 0.0f, -1.0f, fwd);
        rotate(1.0f, 0.0f, 0.0f, right);
        rotate(0.0f, 1.0f, 0.0f, up);
        const float halfH = std::tan(fov_y * 0.5f);
        const float halfW = halfH * aspect;
        for (int k = 0; k < 3; k++)
        {
            out->origin[k] = s->position[k];
            out->horizontal[k] = 2.0f * halfW * right[k];
            out->vertical[k] = 2.0f * halfH * up[k];
            out->lower_left[k] = s->position[k] + fwd[k] - halfW * right[k] - halfH * up[k];
        }
        return GPT_OK;
    }
}
