// Host-side launchers of the kernels in kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "pt_internal.h"

namespace pt
{
    struct IterationLaunch
    {
        SceneView scene;
        Wavefront wf;
        const JobView* job;       // device pointer
        const SceneEntry* scenes; // device pointer, one entry (lights of the scene)
        cudaGraphConditionalHandle handle;
        bool modelPresent[kModelCount];
        bool nee;
        int traceBlocks;
        int traceThreads;
        uint32_t refill;
        uint32_t refillShadow;     // the same threshold for the shadow-ray (any-hit) traversal
        int occupancy;             // traversal kernel variant: 1, 10 or 12 resident blocks per SM targeted
        int shadeBlocks;           // grid of the 256-thread regeneration-queue kernel (the reference-structure layout)
        int sms;                   // multiprocessors: each shading grid is sms x that kernel's resident blocks per SM
        bool graphLoop;            // true: inside the frame graph's WHILE node; false: host-driven loop
        uint32_t bvhFormat;        // kBvh8Quantised or kBvh2Fp32 (scene.nodes2 must be present)
        int stackCap;              // traversal stack entries a ray may use (0 = the whole stack)
        cudaEvent_t traceStart;    // optional events around the closest-hit traversal launch (host loop)
        cudaEvent_t traceStop;
        // Optional fork/join: the shading kernels of the models present run on their own streams,
        // concurrently (parallel branches when captured into the frame graph). nullptr = in order.
        cudaEvent_t shadeFork;
        cudaEvent_t shadeJoin[kModelCount];
        cudaStream_t shadeStreams[kModelCount];
    };

    // One iteration of the job engine over all resident scenes and active jobs.
    struct EngineLaunch
    {
        SceneView scene;           // packed arrays of all resident scenes
        Wavefront wf;
        EngineView ev;
        cudaGraphConditionalHandle handle;
        bool modelPresent[kModelCount];
        bool anyLights;
        int traceBlocks;
        int traceThreads;
        uint32_t refill;
        uint32_t refillShadow;
        int occupancy;
        int shadeBlocks;           // grid of the 256-thread folding kernel
        int sms;                   // multiprocessors: each shading grid is sms x that kernel's resident blocks per SM
        bool graphLoop;
        // Optional fork/join of the shading kernels, as in IterationLaunch. nullptr = in order.
        cudaEvent_t shadeFork;
        cudaEvent_t shadeJoin[kModelCount];
        cudaStream_t shadeStreams[kModelCount];
    };

    int trace_grid_blocks(int device, int threads, uint32_t depth, int occupancy, uint32_t bvhFormat = kBvh8Quantised);
    cudaError_t launch_engine_init(const Wavefront& wf, const EngineView& ev, uint32_t pool, cudaStream_t stream);
    cudaError_t launch_engine_iteration(const EngineLaunch& launch, cudaStream_t stream);
    cudaError_t launch_rebase_field(uint32_t* base, uint32_t n, uint32_t strideWords, uint32_t offset, bool skipInvalid, cudaStream_t stream);
    cudaError_t launch_rebase_nodes(Node8* nodes, uint32_t n, uint32_t nodeOffset, uint32_t triOffset, cudaStream_t stream);
    cudaError_t launch_iteration(const IterationLaunch& launch, cudaStream_t stream);
    cudaError_t launch_frame_prologue(const Wavefront& wf, const JobView* job, uint32_t pool, int blocks, cudaStream_t stream);
    cudaError_t launch_resolve(const JobView* job, float4* accumulation, uint32_t* framebuffer, int blocks, cudaStream_t stream);
    cudaError_t launch_resolve_fp64(const JobView* job, double* sums, int blocks, cudaStream_t stream);
    cudaError_t launch_clear(uint32_t* framebuffer, uint32_t n, uint32_t value, cudaStream_t stream);
    cudaError_t launch_batch_trace(const SceneView& scene, uint32_t root, const float* rays, uint32_t n, uint32_t* cursor, uint32_t* triOut,
                                   float* uvtOut, uint8_t* occOut, int blocks, int threads, uint32_t* errorFlags, cudaStream_t stream,
                                   uint32_t bvhFormat = kBvh8Quantised);
    cudaError_t launch_shading_records(const float* positions, const float* normals, const float* tangents, const float* uvs,
                                       const uint32_t* materialIds, uint32_t n, float4* shading, cudaStream_t stream);
    cudaError_t launch_light_build(const float4* shading, const MaterialDev* materials, uint32_t n,
                                   uint32_t* flags, uint32_t* index, uint32_t* scanScratch, uint32_t* lightCount, cudaStream_t stream);
    cudaError_t launch_light_records(const float* positions, const float4* shading, const MaterialDev* materials,
                                     const MaterialTextures* textures, uint32_t n, const uint32_t* flags, const uint32_t* index,
                                     float4* lights, double* weights, double* powerWeights, cudaStream_t stream);
    cudaError_t launch_alias_build(const double* weights, uint32_t n, double* prefix, double* scanScratch, uint4* bins,
                                   uint32_t* stackIndex, float* stackValue, cudaStream_t stream);
    size_t scan_scratch_elements(uint32_t n);
    size_t alias_power_scratch_bytes(uint32_t n);
    cudaError_t launch_alias_build_power(const double* weights, const double* areaWeights, uint32_t n, void* scratch, uint4* bins,
                                         cudaStream_t stream);
}
