// Internal layouts shared by the host runtime (renderer.cu, bvh8.cpp) and the kernels.
//
// HBM layout (all structure-of-arrays, 16-byte vector records, one CUDA allocation each):
//   BVH8 node        128 B  (Node8 below)           scene-resident
//   triangle (MT)     48 B  v0|orig, e1|model, e2     leaf order, scene-resident
//   triangle shading 144 B  3 normals, 3 tangents, gN|material, uvs (Triangle.hpp:24-38 layout), input order
//   light           112 B   v0|index, e1|area, e2, gN, emission, uv0|uvE1, uvE2|material
//   alias bin         16 B  q, p, alias, value (AliasTableView.hpp:8-14)
//   path slot         36 B  throughput|depth/flags, radiance|rng position, sample index
//   ray queue entry   32 B  origin|slot, direction|tMax   (x2, ping-pong)
//   hit record        16 B  triangle, u, v, t             (aligned with the current ray queue)
//   material queue     4 B  ray-queue index               (x6, one per shading model)
//   shadow queue      48 B  origin|slot, direction|tMax, radiance
//   regen queue        4 B  slot
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pt
{
    constexpr uint32_t kInvalid = 0xFFFFFFFFu;
    constexpr uint32_t kModelCount = 6;
    constexpr uint32_t kModelEmissive = 5;
    constexpr float kMinT = 1e-4f;
    constexpr float kMaxT = 1e34f;
    constexpr uint64_t kRandomSeed = 1234;
    constexpr uint32_t kRussianRouletteStartDepth = 3;
    constexpr uint32_t kQueueLogColumns = 9;
    constexpr uint32_t kMaxStack = 64;

    // BVH8 node, 128 bytes = 8 x uint4, loaded as one L1 line.
    //  w[0] = px, py, pz (float bits), ex | ey<<8 | ez<<16 | innerMask<<24   (biased float exponents of the scales)
    //  w[1] = qlo.x[0..7] (x,y words), qlo.y[0..7] (z,w words)
    //  w[2] = qlo.z[0..7], qhi.x[0..7]
    //  w[3] = qhi.y[0..7], qhi.z[0..7]
    //  w[4], w[5] = child[0..7]: internal -> node index, leaf -> first triangle (leaf order)
    //  w[6] = count[0..7] (bytes, leaf triangle counts), leafMask, 0
    //  w[7] = reserved
    // Child slots are assigned by octant, so that visiting slot (i ^ rayOctant) for i = 0..7
    // is an approximate front-to-back order.
    struct __align__(16) Node8
    {
        uint4 w[8];
    };
    static_assert(sizeof(Node8) == 128, "BVH8 node is 128 bytes");

    struct __align__(16) MaterialDev  // == gpt_material
    {
        uint32_t model;
        float color[3];
        float specular[3];
        float shininess;
        float rma[3];
        float emission[3];
        float normal[3];
        float ior;
        float transmission;
        float reserved;
    };
    static_assert(sizeof(MaterialDev) == 80, "material record is 80 bytes");

    // Texture objects of a material's slots (0 = use the constant of MaterialDev).
    struct __align__(16) MaterialTextures
    {
        unsigned long long tex[6];  // color, specular, shininess, rma, emission, normal
        unsigned long long pad[2];
    };
    static_assert(sizeof(MaterialTextures) == 64, "material texture record is 64 bytes");

    struct SceneView
    {
        const Node8* nodes;
        const float4* tris;       // 3 per triangle, leaf order
        const float4* shading;    // 9 per triangle, input order
        const MaterialDev* materials;
        const MaterialTextures* textures;  // per material, nullptr when the scene has no image textures
        const float4* lights;     // 7 per light
        const uint4* bins;        // alias table
        uint32_t lightCount;
        uint32_t nodeCount;
        uint32_t triangleCount;
        uint32_t depth;           // BVH8 depth (stack entries needed)
    };

    struct JobView
    {
        float camera[12];         // origin, lowerLeftCorner, horizontal, vertical
        uint32_t width, height, spp, spa;
        uint32_t depthLimit, nee, maxIterations, pad1;   // maxIterations: hard cap of the device loop
        uint64_t totalSamples;
        float* sampleRadiance;    // [totalSamples][3]
        uint64_t rngOffset;       // added to the sample index to form the Philox subsequence
    };

    // Device-resident frame control block. One thread (advance kernel) mutates it
    // between the other kernels of an iteration.
    struct Counters
    {
        uint32_t rayCount[2];
        uint32_t cur;
        uint32_t matCount[kModelCount];
        uint32_t shadowCount;
        uint32_t regenCount;
        uint32_t traceCursor;
        uint32_t shadowCursor;
        uint32_t iteration;
        uint32_t done;
        uint32_t errorFlags;
        unsigned long long launched;
        unsigned long long raysTraced;
        unsigned long long shadowRaysTraced;
        // Device time of each kernel phase: first-block start and last-block end (%globaltimer, ns)
        // of the current launch, summed over iterations by the advance kernel.
        // Phases: 0 closest-hit traversal, 1 shading (all models), 2 shadow traversal, 3 regeneration.
        unsigned long long tStart[4];
        unsigned long long tEnd[4];
        unsigned long long tAccum[4];
        // Traversal work: BVH8 node visits and triangle tests; [0] closest hit, [1] shadow rays.
        unsigned long long nodeVisits[2];
        unsigned long long triTests[2];
    };

    struct Wavefront
    {
        float4* rayO[2];
        float4* rayD[2];
        float4* hit;
        uint32_t* matQ[kModelCount];
        float4* shO;
        float4* shD;
        float4* shL;
        uint32_t* regen;
        float4* slotT;            // throughput xyz, w = bits(depth | delta << 8)
        float4* slotL;            // radiance xyz, w = bits(rng stream position)
        uint32_t* slotSample;
        uint32_t capacity;
        uint32_t logCapacity;
        uint32_t* queueLog;
        Counters* ctr;
        const volatile uint32_t* cancel;            // host-mapped: nonzero ends the frame after the current iteration
        volatile unsigned long long* progress;      // host-mapped: [0] samples launched, [1] iterations
    };

    enum ErrorFlags : uint32_t
    {
        kErrStackOverflow = 1u,
        kErrQueueOverflow = 2u,
        kErrIterationCap = 4u,
    };
}
