// Allocation-free light alias-table build.
//
// Who needs this: callers that must not allocate device memory at the time they build a
// light sampler. Typical cases are code running inside a real-time frame loop whose memory
// budget is fixed up front, engines that route every device allocation through their own
// pool and forbid the CUDA allocator, and code paths that run while another component holds
// the device in a state where cudaMalloc/cudaFree would stall or serialise the GPU (cudaFree
// synchronises the whole device). For them gpt_build_alias_table_noalloc builds the same table
// as the scene upload, but its working memory is a fixed array compiled into this library.
//
// The working memory is the file-scope device array below: GPT_NOALLOC_MAX_LIGHTS lights at
// 32 bytes each plus the prefix-sum block sums, about 2 MiB. Every GPU that loads the library
// keeps this array until the process exits. Host code never uses the array's name as an
// address: on its first call on a device the entry point asks the runtime for the device
// address (cudaGetSymbolAddress, with that device current) and caches it per device.
//
// All calls share the one array, and the array keeps whatever the previous call left in it.
// Nothing here reads a value before this call has written it, so no clearing is needed. Two
// calls whose work overlaps on the GPU (different streams, or different host threads on the
// same device without ordering) race on the array and corrupt each other's tables: order them.
//
// The cached address belongs to the device's current primary context. A device reset
// (cudaDeviceReset) after the first call tears that context down and is not supported: the
// library would keep using the old address.
//
// The weights must be finite and non-negative with a positive sum, as the scene upload's
// emitter areas are (the reference asserts the sum, AliasTable.hpp:24). Other weights give a
// table of NaN or infinite probabilities; the entry point does not read them back to check.
#include <cstdint>
#include <mutex>

#include "../../include/gpt_b200.h"
#include "kernels.h"

namespace
{
    constexpr uint32_t kMaxLights = GPT_NOALLOC_MAX_LIGHTS;
    constexpr size_t kAlign = 256;

    constexpr size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

    // Layout of the scratch array for kMaxLights lights.
    constexpr size_t kWeightsOff = 0;                                                   // double[n]
    constexpr size_t kPrefixOff = align_up(kWeightsOff + sizeof(double) * kMaxLights);  // double[n]
    constexpr size_t kStackIndexOff = align_up(kPrefixOff + sizeof(double) * kMaxLights);      // uint32[2n]
    constexpr size_t kStackValueOff = align_up(kStackIndexOff + sizeof(uint32_t) * 2 * kMaxLights);  // float[2n]
    constexpr size_t kScanOff = align_up(kStackValueOff + sizeof(float) * 2 * kMaxLights);     // double[scan sums]
    constexpr size_t kScanElements = 512;  // >= scan_scratch_elements(kMaxLights)
    constexpr size_t kScratchBytes = align_up(kScanOff + sizeof(double) * kScanElements);

    static __device__ __align__(256) unsigned char g_aliasScratch[kScratchBytes];

    constexpr int kMaxDevices = 64;
    std::mutex g_mutex;
    void* g_scratchAddress[kMaxDevices] = {};

    __global__ void weights_to_double_kernel(const float* weights, uint32_t n, double* out)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            out[i] = static_cast<double>(weights[i]);
    }

    // Device address of the scratch array on the current device (set up once per device).
    int scratch_address(void** out)
    {
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return GPT_ERR_CUDA;
        std::scoped_lock lock(g_mutex);
        if (!g_scratchAddress[device])
        {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_aliasScratch) != cudaSuccess || ptr == nullptr) return GPT_ERR_CUDA;
            g_scratchAddress[device] = ptr;
        }
        *out = g_scratchAddress[device];
        return GPT_OK;
    }
}

extern "C" int gpt_build_alias_table_noalloc(const float* weights, uint32_t light_count, uint32_t* bins, void* stream)
{
    static_assert(kScanElements >= 3 + (kMaxLights + 1023) / 1024 + 2, "scan scratch too small");
    if (light_count == 0) return GPT_OK;
    if (!weights || !bins) return GPT_ERR_INVALID_ARGUMENT;
    // the kernels read 4-byte weights and store whole 16-byte bins
    if (reinterpret_cast<uintptr_t>(bins) % 16 != 0 || reinterpret_cast<uintptr_t>(weights) % 4 != 0) return GPT_ERR_INVALID_ARGUMENT;
    if (light_count > kMaxLights) return GPT_ERR_CAPACITY;
    if (pt::scan_scratch_elements(light_count) > kScanElements) return GPT_ERR_CAPACITY;
    void* base = nullptr;
    const int rc = scratch_address(&base);
    if (rc != GPT_OK) return rc;
    unsigned char* scratch = static_cast<unsigned char*>(base);
    double* w = reinterpret_cast<double*>(scratch + kWeightsOff);
    double* prefix = reinterpret_cast<double*>(scratch + kPrefixOff);
    uint32_t* stackIndex = reinterpret_cast<uint32_t*>(scratch + kStackIndexOff);
    float* stackValue = reinterpret_cast<float*>(scratch + kStackValueOff);
    double* scan = reinterpret_cast<double*>(scratch + kScanOff);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t blocks = (light_count + 255) / 256;
    weights_to_double_kernel<<<blocks, 256, 0, s>>>(weights, light_count, w);
    if (cudaGetLastError() != cudaSuccess) return GPT_ERR_CUDA;
    if (pt::launch_alias_build(w, light_count, prefix, scan, reinterpret_cast<uint4*>(bins), stackIndex, stackValue, s) != cudaSuccess)
        return GPT_ERR_CUDA;
    return GPT_OK;
}
