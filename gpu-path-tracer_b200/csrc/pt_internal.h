// Internal layouts shared by the host runtime (renderer.cu, bvh8.cpp) and the kernels.
//
// HBM layout (all structure-of-arrays, 16-byte vector records, one CUDA allocation each):
//   BVH8 node        128 B  (Node8 below)           scene-resident
//   triangle (MT)     64 B  v0|orig, e1|model, e2, 0  leaf order, scene-resident (32-byte aligned:
//                           v0 and e1 in one 256-bit load, e2 in a 128-bit one)
//   triangle shading 144 B  3 normals, 3 tangents, gN|material, uvs (Triangle.hpp:24-38 layout), input order
//   light           112 B   v0|index, e1|area, e2, gN, emission, uv0|uvE1, uvE2|material
//   alias bin         16 B  q, p, alias, value (AliasTableView.hpp:8-14); two tables, area and power weights
//   path slot         36 B  throughput|depth/flags/job, radiance|rng position, sample index
//   ray queue entry   32 B  origin|tag, direction|tMax   (x2, ping-pong; tag = slot | scene << 24)
//   material queue    48 B  origin|tag, direction|tMax, triangle|u|v|t   (x6, one per shading model: the
//                           closest-hit kernel writes the ray and its hit, so shading reads one entry)
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
    // Ray and shadow-ray entries carry a tag: the path slot in the low 24 bits and the resident
    // scene in the high 8. Path metadata: depth (8 bits) | delta flag (bit 8) | job << 16.
    constexpr uint32_t kSlotBits = 24;
    constexpr uint32_t kSlotMask = (1u << kSlotBits) - 1u;
    constexpr uint32_t kMaxPool = 1u << kSlotBits;
    constexpr uint32_t kMaxScenes = 256;
    constexpr uint32_t kMaxTriangles = 1u << 24;  // leaf references hold 24-bit triangle positions
    constexpr uint32_t kTriangleVec4 = 4;         // 16-byte words per traversal triangle record (64 B)
    constexpr uint32_t kMaxJobs = 65536;
    constexpr uint32_t kMaxRing = 256;

    // Random-number policy of a job. Philox: cuRAND Philox4_32_10, seed 1234, subsequence = sample
    // index (the reference's streams, PathData.hpp:37-73). PCG32: a per-sample PCG32 stream seeded by
    // a hash of (seed, pixel, sample), O'Neill's PCG-XSH-RR 64/32.
    enum RngPolicy : uint32_t
    {
        kRngPhilox = 0,
        kRngPcg32 = 1,
    };

    // Light selection of NEE. Area: probability proportional to the emitter's area, the reference's
    // LightSampler (LightSampler.cpp:16-19). Power: proportional to area x luminance of the emission.
    enum LightMode : uint32_t
    {
        kLightsArea = 0,
        kLightsPower = 1,
    };

    // BVH8 node, 128 bytes = 8 x uint4, loaded as one L1 line.
    //  w[0] = px, py, pz (float bits), ex | ey<<8 | ez<<16 | innerMask<<24   (biased float exponents of the scales)
    //  w[1] = qlo.x[0..7] (x,y words), qlo.y[0..7] (z,w words)
    //  w[2] = qlo.z[0..7], qhi.x[0..7]
    //  w[3] = qhi.y[0..7], qhi.z[0..7]
    //  w[4], w[5] = child[0..7]: internal -> node index, leaf -> first triangle (leaf order, bits 0-23)
    //               | triangle count << 24
    //  w[6] = count[0..7] (bytes, leaf triangle counts), leafMask, 0   (builder and checker only)
    //  w[7] = reserved
    // Empty slots hold inverted boxes (lo 255, hi 0) and child reference 0. A node visit reads w[0..3]
    // (64 bytes); a leaf or a pop reads one child reference.
    // Child slots are assigned by octant, so that visiting slot (i ^ rayOctant) for i = 0..7
    // is an approximate front-to-back order.
    struct __align__(16) Node8
    {
        uint4 w[8];
    };
    static_assert(sizeof(Node8) == 128, "BVH8 node is 128 bytes");

    // Binary BVH node with FP32 child boxes, 64 bytes = 4 x uint4 (the plain format, compared with the
    // quantised BVH8 on the same binned-SAH binary tree the BVH8 is collapsed from).
    //  w[0] = lo0.x, lo0.y, lo0.z, hi0.x      (float bits; child boxes padded and rounded outward)
    //  w[1] = hi0.y, hi0.z, lo1.x, lo1.y
    //  w[2] = lo1.z, hi1.x, hi1.y, hi1.z
    //  w[3] = ref0, ref1, count0 | count1 << 8 | leafMask << 16 | validMask << 24, 0
    // ref: internal child -> node index, leaf child -> first triangle (leaf order, shared with BVH8).
    struct __align__(16) Node2
    {
        uint4 w[4];
    };
    static_assert(sizeof(Node2) == 64, "binary BVH node is 64 bytes");

    enum BvhFormat : uint32_t
    {
        kBvh8Quantised = 0,
        kBvh2Fp32 = 1,
    };

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
        const float4* tris;       // kTriangleVec4 per triangle, leaf order
        const float4* shading;    // 9 per triangle, input order
        const MaterialDev* materials;
        const MaterialTextures* textures;  // per material, nullptr when the scene has no image textures
        const float4* lights;     // 7 per light
        const uint4* bins;        // alias table, area weights (the reference's light sampler)
        const uint4* binsPower;   // alias table, power weights (area x emission luminance)
        uint32_t lightCount;
        uint32_t nodeCount;
        uint32_t triangleCount;
        uint32_t depth;           // BVH8 depth (stack entries needed)
        const Node2* nodes2;      // binary FP32 BVH of the same scene (frame renderer only), nullptr if absent
        uint32_t depth2;          // binary BVH depth
    };

    // Per resident scene: where its BVH8 starts in the packed node array and its slice of the
    // packed light list / alias table (alias entries are stored rebased to the packed list).
    struct __align__(16) SceneEntry
    {
        uint32_t root;
        uint32_t lightOffset;
        uint32_t lightCount;
        uint32_t triangleOffset;
    };

    // One render job. The single-frame renderer uses one of these (job 0, sample-major output);
    // the job engine keeps a table of them (pass-major launch order, pass ring + Kahan accumulator).
    struct JobView
    {
        float camera[12];         // origin, lowerLeftCorner, horizontal, vertical
        uint32_t width, height, spp, spa;
        uint32_t depthLimit, nee, maxIterations, scene;   // maxIterations: hard cap of the device loop
        uint64_t totalSamples;    // launch indices [0, totalSamples)
        float* sampleRadiance;    // frame renderer: [totalSamples][3]; engine: ring [ring][pixels][3]
        uint64_t rngOffset;       // added to the sample index to form the Philox subsequence
        // job engine only
        uint32_t pixels, ring, state, folded;             // ring: pass buffers; folded: passes summed into accum
        uint64_t launched;        // launch indices handed out so far
        float4* accum;            // [pixels][2]: Kahan sum (xyz), compensation (xyz)
        uint32_t* framebuffer;    // RGBA8, written when the last pass is folded
        uint32_t* passDone;       // [ring] finished samples of the pass held by each ring buffer
        uint32_t rngPolicy;       // RngPolicy
        uint32_t lightMode;       // LightMode
    };

    // Bit of a job-server order entry (the rest is the job-table index): the job takes path slots only
    // once every marked job ahead of it has launched all its samples.
    constexpr uint32_t kOrderInTurn = 0x80000000u;

    enum JobState : uint32_t
    {
        kJobFree = 0,
        kJobActive = 1,
        kJobDone = 2,
    };

    // Launches of one planned iteration for one job: new samples [start, start + count) of the
    // iteration take launch indices first, first + 1, ... of job `job`.
    struct LaunchSegment
    {
        uint32_t job;
        uint32_t start;
        uint64_t first;
    };

    // Device-resident state of the job engine beyond the wavefront counters. The first four
    // words belong to the device; the host writes the last four before every slice.
    struct EngineCtl
    {
        uint32_t freeCount;       // idle path slots on the free list
        uint32_t launchCount;     // new samples planned for this iteration
        uint32_t segmentCount;
        uint32_t stalled;         // set if an unfinished job can make no progress (logic error)
        uint32_t orderCount;      // active jobs, oldest first
        uint32_t sliceIterations;
        uint32_t maxSliceIterations;
        uint32_t completed;       // jobs finished during the current slice
    };

    struct EngineView
    {
        JobView* jobs;
        const uint32_t* order;    // [orderCount] job-table indices, oldest first
        LaunchSegment* segments;  // [capacity of the job table]
        uint32_t* freeList;       // [pool]
        EngineCtl* ctl;
        const SceneEntry* scenes;
        const volatile uint32_t* doorbell;  // host-mapped: nonzero ends the slice after the current iteration
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
        uint32_t regenCursor;     // new samples handed out by the bitmap regeneration of the iteration
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
        float4* matQ[kModelCount];   // per model: entries of 3 float4 = origin|tag, direction|tMax, triangle|u|v|t
        float4* shO;
        float4* shD;
        float4* shL;
        uint32_t* regen;
        uint32_t* regenBits;      // bit per slot set when its path finished (nullptr: the regen queue, frame renderer only)
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
