// Host runtime pieces shared by the frame renderer (renderer.cu) and the job engine (engine.cu):
// status values, RAII device buffers, texture objects and device-resident scenes.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gpt_b200.h"
#include "pt_internal.h"

namespace pt
{
    struct Status
    {
        int code = GPT_OK;
        std::string message;
        static Status Ok() { return {}; }
        static Status Err(int c, std::string m) { return Status{c, std::move(m)}; }
        bool ok() const { return code == GPT_OK; }
    };

    inline Status CudaStatus(const char* op, cudaError_t e)
    {
        if (e == cudaSuccess) return Status::Ok();
        // Error text format of the reference (Cuda/Utils/Error.cpp:22-25).
        std::string msg = std::string(op) + " failed: " + cudaGetErrorName(e) + ": " + cudaGetErrorString(e);
        return Status::Err(e == cudaErrorMemoryAllocation ? GPT_ERR_OUT_OF_MEMORY : GPT_ERR_CUDA, msg);
    }

#define PT_TRY(expr)                      \
    do                                    \
    {                                     \
        Status _s = (expr);               \
        if (!_s.ok()) return _s;          \
    } while (0)
#define PT_CUDA(op, expr) PT_TRY(CudaStatus(op, (expr)))

    // A named host range on the calling thread's NVTX stack (scene upload and its stages, frames,
    // the autotuner, job-server slices), so a profiler's timeline shows which host step issued the
    // kernels under it (ncu: --nvtx --nvtx-include "gpt render frame/"). NVTX is header-only: with
    // no tool attached a push or pop is one predictable branch. end() closes the range early; the
    // destructor closes it on every return path otherwise.
    class NvtxRange
    {
    public:
        explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
        ~NvtxRange() { end(); }
        NvtxRange(const NvtxRange&) = delete;
        NvtxRange& operator=(const NvtxRange&) = delete;
        void end()
        {
            if (open_) nvtxRangePop();
            open_ = false;
        }

    private:
        bool open_ = true;
    };

    // True when this device allocation is the one gpt_inject_allocation_failure chose to fail.
    bool InjectedAllocationFailure();

    // RAII device allocation (the reference's DeviceBuffer1D, Runtime/Memory/DeviceBuffer1D.cpp:33-80).
    class DeviceBuffer
    {
    public:
        DeviceBuffer() = default;
        DeviceBuffer(const DeviceBuffer&) = delete;
        DeviceBuffer& operator=(const DeviceBuffer&) = delete;
        ~DeviceBuffer() { reset(); }
        // Grows the buffer to at least `bytes` (contents are not kept). The new allocation is made before
        // the old one is freed, so a failed call leaves the buffer as it was.
        Status allocate(size_t bytes)
        {
            if (bytes <= bytes_ && ptr_) return Status::Ok();
            if (bytes == 0) return Status::Ok();
            if (InjectedAllocationFailure())
                return Status::Err(GPT_ERR_OUT_OF_MEMORY, "cudaMalloc failed: out of memory (injected by gpt_inject_allocation_failure)");
            void* fresh = nullptr;
            PT_CUDA("cudaMalloc", cudaMalloc(&fresh, bytes));
            reset();
            ptr_ = fresh;
            bytes_ = bytes;
            return Status::Ok();
        }
        void reset()
        {
            if (ptr_) cudaFree(ptr_);
            ptr_ = nullptr;
            bytes_ = 0;
        }
        void swap(DeviceBuffer& other)
        {
            std::swap(ptr_, other.ptr_);
            std::swap(bytes_, other.bytes_);
        }
        template <typename T>
        T* get() const { return static_cast<T*>(ptr_); }
        size_t bytes() const { return bytes_; }

    private:
        void* ptr_ = nullptr;
        size_t bytes_ = 0;
    };

    // An image texture with the reference's descriptors (Texture.cpp:65-189).
    struct TextureObject
    {
        cudaArray_t array = nullptr;
        cudaTextureObject_t object = 0;
        TextureObject() = default;
        TextureObject(const TextureObject&) = delete;
        TextureObject& operator=(const TextureObject&) = delete;
        ~TextureObject()
        {
            if (object) cudaDestroyTextureObject(object);
            if (array) cudaFreeArray(array);
        }
    };

    struct SceneGpu
    {
        DeviceBuffer nodes, tris, shading, materials, lights, bins, binsPower, materialTextures, entry, nodes2;
        std::vector<std::unique_ptr<TextureObject>> textures;
        uint32_t nodeCount = 0, triangleCount = 0, depth = 0, lightCount = 0, materialCount = 0;
        uint32_t nodeCount2 = 0, depth2 = 0;  // binary FP32 BVH, built when the scene is uploaded with it
        bool modelPresent[kModelCount] = {};
        uint64_t version = 0;
        double bvhSeconds = 0.0, uploadSeconds = 0.0;  // BVH build (host or device); whole upload (wall clock)
        bool deviceBvh = false;                         // the BVH8 was built on the device
        SceneView view() const
        {
            SceneView v{};
            v.nodes = nodes.get<Node8>();
            v.tris = tris.get<float4>();
            v.shading = shading.get<float4>();
            v.materials = materials.get<MaterialDev>();
            v.textures = textures.empty() ? nullptr : materialTextures.get<MaterialTextures>();
            v.lights = lights.get<float4>();
            v.bins = bins.get<uint4>();
            v.binsPower = binsPower.get<uint4>();
            v.lightCount = lightCount;
            v.nodeCount = nodeCount;
            v.triangleCount = triangleCount;
            v.depth = depth;
            v.nodes2 = nodeCount2 ? nodes2.get<Node2>() : nullptr;
            v.depth2 = depth2;
            return v;
        }
    };

    // Minimal PNG writer (zlib deflate) for SaveRenderedFrame (Renderer.cpp:649-675): RGBA8, rows
    // flipped vertically like Import::FlipVertically.
    // Validates a scene description and builds its device copy: image textures, BVH8, shading records,
    // light list and alias table. The BVH8 is built on the host (binned SAH), with `withBinary` also the
    // binary FP32 BVH, or with `deviceBvh` on the device (clustering; no binary BVH).
    Status BuildScene(const gpt_scene_desc& d, cudaStream_t stream, std::unique_ptr<SceneGpu>& out, bool withBinary = false,
                      bool deviceBvh = false);
}
