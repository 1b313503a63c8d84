// sm_100a kernels of the wavefront path tracer.
//
// Per wavefront iteration (one CUDA-graph body, no host round trip):
//   trace_kernel<closest>  BVH8 closest hit for the current ray queue -> per-model queues of (ray, hit) entries
//   shade_kernel<model>    one launch per shading model present (MaterialEval.cu:194-912)
//   trace_kernel<any>      NEE shadow rays, any hit; unoccluded radiance added to the path slot
//   regen_bits_kernel      finished paths -> per-sample radiance; new samples -> next ray queue
//   advance_kernel         one thread: queue bookkeeping, log, loop condition (Renderer.cpp:573-619)
// Every expression that reaches a result is written in the reference's operator order. The
// product library compiles this file as the reference's kernels are compiled (multiply-add
// contraction, CUDA's sinf/cosf/powf/rsqrtf); the deterministic library compiles it with
// -fmad=false and the IEEE definitions of pt_math.cuh (PT_CUDA_MATH).
#include <curand_kernel.h>

#include "kernels.h"
#include "traverse.cuh"

namespace pt
{
    // ------------------------------------------------------------------ warp helpers
    __device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

    // Warp-aggregated queue slot reservation: one atomic per converged group of lanes.
    __device__ __forceinline__ uint32_t agg_push(uint32_t* counter)
    {
        const unsigned mask = __activemask();
        const int leader = __ffs(mask) - 1;
        const uint32_t lane = lane_id();
        uint32_t base = 0;
        if (static_cast<int>(lane) == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
        base = __shfl_sync(mask, base, leader);
        return base + static_cast<uint32_t>(__popc(mask & ((1u << lane) - 1u)));
    }

    // Same, grouping lanes by key (queue id); counters[key] is the queue's size.
    __device__ __forceinline__ uint32_t agg_push_keyed(uint32_t* counters, uint32_t key)
    {
        const unsigned active = __activemask();
        const unsigned peers = __match_any_sync(active, key);
        const int leader = __ffs(peers) - 1;
        const uint32_t lane = lane_id();
        uint32_t base = 0;
        if (static_cast<int>(lane) == leader) base = atomicAdd(&counters[key], static_cast<uint32_t>(__popc(peers)));
        base = __shfl_sync(peers, base, leader);
        return base + static_cast<uint32_t>(__popc(peers & ((1u << lane) - 1u)));
    }

    __device__ __forceinline__ unsigned long long global_ns()
    {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }

    // Phase timing: thread 0 of every block stamps its start (min) and its end (max).
    __device__ __forceinline__ void phase_begin(Counters* c, int phase)
    {
        if (c != nullptr && threadIdx.x == 0) atomicMin(&c->tStart[phase], global_ns());
    }
    __device__ __forceinline__ void phase_end(Counters* c, int phase)
    {
        __syncthreads();
        if (c != nullptr && threadIdx.x == 0) atomicMax(&c->tEnd[phase], global_ns());
    }

    __device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
    __device__ __forceinline__ uint4 ldg4(const uint4* p) { return __ldg(p); }
    // 32 read-only bytes in one 256-bit load (sm_100); p must be 32-byte aligned. Halves the load
    // instructions of a node visit and of a triangle test against 16-byte loads.
    __device__ __forceinline__ void ldg8(const uint4* p, uint4& a, uint4& b)
    {
        asm("ld.global.nc.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
            : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
            : "l"(p));
    }

    // ------------------------------------------------------------------ traversal
    // Registers of a ray in flight. Values a traversal step reads rarely live in the thread's slot
    // of shared memory instead (ColdSlot), which keeps the node test free of register spills.
    struct TraversalState
    {
        RayPre ray;
        float hitT;        // closest hit so far (tMax of the query until a hit)
        uint32_t pending;  // binary BVH: node to visit next, kInvalid when the stack decides
        int sp;
    };

    // Traversal work of a lane: node visits in bits 0-15, triangle tests in bits 16-31 (flushed to
    // the frame counters before either field can overflow).
    constexpr uint32_t kVisit = 1u;
    constexpr uint32_t kTestShift = 16;

    // Shared-memory slot of one thread: [0] = direction xyz, tag; [1] = hit u, v,
    // triangle | model << 24 (kInvalid while there is no hit), queue index.
    struct ColdSlot
    {
        float4* p;
        __device__ float3 direction() const
        {
            const float4 a = p[0];
            return make_float3(a.x, a.y, a.z);
        }
    };

    // Triangles [first, first + count) of a leaf (leaf order). Returns false when an any-hit query
    // found an occluder (traversal over); closest hit keeps the best hit in st.hit.
    // FIXED: the query's tMin is the wavefront's constant kMinT (no register holds it).
    template <bool ANY, bool FIXED>
    __device__ __forceinline__ bool leaf_tests(const SceneView& sc, TraversalState& st, ColdSlot cold, uint32_t first, uint32_t count,
                                               bool& occluded, uint32_t& work)
    {
        const float tmin = FIXED ? kMinT : st.ray.tmin;
        work += count << kTestShift;
        const float3 d = cold.direction();
        for (uint32_t k = 0; k < count; k++)
        {
            const uint4* tp = reinterpret_cast<const uint4*>(sc.tris) + static_cast<size_t>(first + k) * kTriangleVec4;
            uint4 ua, ub;
            ldg8(tp, ua, ub);
            const float4 a = make_float4(__uint_as_float(ua.x), __uint_as_float(ua.y), __uint_as_float(ua.z), __uint_as_float(ua.w));
            const float4 b = make_float4(__uint_as_float(ub.x), __uint_as_float(ub.y), __uint_as_float(ub.z), __uint_as_float(ub.w));
            const float4 c = ldg4(reinterpret_cast<const float4*>(tp + 2));
            float t, u, v;
            if (!intersect_triangle(a, b, c, st.ray.o, d, t, u, v)) continue;
            if (ANY)
            {
                if (t >= tmin && t < st.hitT)
                {
                    occluded = true;
                    return false;
                }
            }
            else
            {
                // better_hit with the best triangle read from shared memory: it matters only at a tie
                if (t >= tmin && t <= st.hitT)
                {
                    const uint32_t orig = __float_as_uint(a.w);
                    bool better = t < st.hitT;
                    if (!better)
                    {
                        const uint32_t best = __float_as_uint(cold.p[1].z);
                        better = best != kInvalid && orig < (best & 0xFFFFFFu);
                    }
                    if (better)
                    {
                        st.hitT = t;
                        cold.p[1].x = u;
                        cold.p[1].y = v;
                        cold.p[1].z = __uint_as_float(orig | (__float_as_uint(b.w) << 24));  // triangle, shading model
                    }
                }
            }
        }
        return true;
    }

    // Slab test of one FP32 box of a binary node against [tmin, tmax]. Each per-axis distance is one
    // subtraction and one multiplication by the rounded reciprocal (at most 3 roundings, relative error
    // below 2^-21); entry distances are lowered and exit distances raised by 2^-20 of their magnitude,
    // so a box the exact arithmetic would hit is never culled. tnear: the widened entry distance.
    __device__ __forceinline__ bool slab_fp32(float lx, float ly, float lz, float hx, float hy, float hz, const RayPre& r, float tmin,
                                              float tmax, float& tnear)
    {
        const float kEps = 9.5367431640625e-07f;  // 2^-20
        const float ax = (lx - r.o.x) * r.invd.x, bx = (hx - r.o.x) * r.invd.x;
        const float ay = (ly - r.o.y) * r.invd.y, by = (hy - r.o.y) * r.invd.y;
        const float az = (lz - r.o.z) * r.invd.z, bz = (hz - r.o.z) * r.invd.z;
        float nx = fminf(ax, bx), fx = fmaxf(ax, bx);
        float ny = fminf(ay, by), fy = fmaxf(ay, by);
        float nz = fminf(az, bz), fz = fmaxf(az, bz);
        nx = nx - fabsf(nx) * kEps;
        ny = ny - fabsf(ny) * kEps;
        nz = nz - fabsf(nz) * kEps;
        fx = fx + fabsf(fx) * kEps;
        fy = fy + fabsf(fy) * kEps;
        fz = fz + fabsf(fz) * kEps;
        const float tn = fmaxf(fmaxf(nx, ny), fmaxf(nz, tmin));
        const float tf = fminf(fminf(fx, fy), fminf(fz, tmax));
        tnear = tn;
        return tn <= tf;
    }

    // Binary FP32 BVH: visit one node (two child boxes) or pop the next node. Leaf children that the
    // ray enters are tested at once; of two internal children the nearer is visited next and the
    // farther pushed. Stack entries are node indices. Returns false when traversal is over.
    template <bool ANY, bool FIXED>
    __device__ __forceinline__ bool traverse_step_binary(const SceneView& sc, TraversalState& st, ColdSlot cold, uint32_t* stack, int stackCap,
                                                         bool& occluded, uint32_t* errorFlags, uint32_t& work)
    {
        uint32_t node;
        if (st.pending != kInvalid)
        {
            node = st.pending;
            st.pending = kInvalid;
        }
        else
        {
            if (st.sp == 0) return false;
            node = stack[--st.sp];
        }
        const uint4* nw = sc.nodes2[node].w;
        work += kVisit;
        const uint4 w0 = ldg4(nw + 0), w1 = ldg4(nw + 1), w2 = ldg4(nw + 2), w3 = ldg4(nw + 3);
        float tn0, tn1;
        const bool h0 = ((w3.z >> 24) & 1u) &&
                        slab_fp32(__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z), __uint_as_float(w0.w),
                                  __uint_as_float(w1.x), __uint_as_float(w1.y), st.ray, FIXED ? kMinT : st.ray.tmin, st.hitT, tn0);
        const bool h1 = ((w3.z >> 25) & 1u) &&
                        slab_fp32(__uint_as_float(w1.z), __uint_as_float(w1.w), __uint_as_float(w2.x), __uint_as_float(w2.y),
                                  __uint_as_float(w2.z), __uint_as_float(w2.w), st.ray, FIXED ? kMinT : st.ray.tmin, st.hitT, tn1);
        const uint32_t leafMask = (w3.z >> 16) & 3u;
        if (h0 && (leafMask & 1u))
            if (!leaf_tests<ANY, FIXED>(sc, st, cold, w3.x, w3.z & 0xFFu, occluded, work)) return false;
        if (h1 && (leafMask & 2u))
            if (!leaf_tests<ANY, FIXED>(sc, st, cold, w3.y, (w3.z >> 8) & 0xFFu, occluded, work)) return false;
        const bool in0 = h0 && !(leafMask & 1u), in1 = h1 && !(leafMask & 2u);
        if (in0 && in1)
        {
            if (st.sp >= stackCap)
            {
                atomicOr(errorFlags, static_cast<uint32_t>(kErrStackOverflow));
                return false;
            }
            const bool first0 = tn0 <= tn1;
            stack[st.sp++] = first0 ? w3.y : w3.x;
            st.pending = first0 ? w3.x : w3.y;
        }
        else if (in0)
            st.pending = w3.x;
        else if (in1)
            st.pending = w3.y;
        return true;
    }

    // Visit one node or pop the next child group. Returns false when traversal is over.
    // ANY: stops at the first triangle with tmin <= t < tmax.
    template <bool ANY, bool FIXED>
    __device__ __forceinline__ bool traverse_step(const SceneView& sc, TraversalState& st, ColdSlot cold, uint32_t* stack, uint32_t stride,
                                                  int stackCap, bool& occluded, uint32_t* errorFlags, uint32_t& work)
    {
        // stack entry = node << 8 | child slots still to visit (traversal order); an entry with no
        // slots is a node to visit itself (the root a ray starts with)
        if (st.sp == 0) return false;
        uint32_t* top = stack + static_cast<uint32_t>(st.sp - 1) * stride;
        const uint32_t entry = *top;
        uint32_t node;
        uint32_t m = entry & 0xFFu;
        if (m == 0)
        {
            node = entry >> 8;
            st.sp--;
        }
        else
        {
            const uint32_t i = static_cast<uint32_t>(__ffs(m) - 1);
            m &= m - 1u;
            if (m == 0) st.sp--;
            else *top = (entry & ~0xFFu) | m;
            const uint32_t parent = entry >> 8;
            const uint32_t* childRefs = reinterpret_cast<const uint32_t*>(&sc.nodes[parent].w[4]);
            node = __ldg(childRefs + (i ^ st.ray.oct));
        }
        const uint4* nw = sc.nodes[node].w;
        work += kVisit;
        uint4 w0, w1, w2, w3;
        ldg8(nw, w0, w1);
        ldg8(nw + 2, w2, w3);
        const uint32_t hitSlots = intersect_children(w0, w1, w2, w3, st.ray, FIXED ? kMinT : st.ray.tmin, st.hitT);
        const uint32_t innerSlots = hitSlots & (w0.w >> 24);
        uint32_t leafOrder = permute_mask(hitSlots & ~(w0.w >> 24), st.ray.oct);
        while (leafOrder)
        {
            const uint32_t i = static_cast<uint32_t>(__ffs(leafOrder) - 1);
            leafOrder &= leafOrder - 1u;
            const uint32_t slot = i ^ st.ray.oct;
            const uint32_t ref = __ldg(reinterpret_cast<const uint32_t*>(&nw[4]) + slot);
            if (!leaf_tests<ANY, FIXED>(sc, st, cold, ref & 0xFFFFFFu, ref >> 24, occluded, work)) return false;
        }
        if (innerSlots)
        {
            if (st.sp >= stackCap)
            {
                atomicOr(errorFlags, static_cast<uint32_t>(kErrStackOverflow));
                return false;
            }
            stack[static_cast<uint32_t>(st.sp) * stride] = (node << 8) | permute_mask(innerSlots, st.ray.oct);
            st.sp++;
        }
        return true;
    }

    // A path left its slot: counted for the iteration and recorded for regeneration, in the finished-slot
    // bitmap (frame renderer) or the regeneration queue (job engine).
    __device__ __forceinline__ void path_finished(const Wavefront& wf, Counters* ctr, uint32_t slot)
    {
        if (wf.regenBits != nullptr)
        {
            agg_push(&ctr->regenCount);
            atomicOr(&wf.regenBits[slot >> 5], 1u << (slot & 31u));
        }
        else
        {
            const uint32_t pos = agg_push(&ctr->regenCount);
            wf.regen[pos] = slot;
        }
    }

    // Work sources of the persistent traversal kernel.
    struct WavefrontClosest
    {
        SceneView sc;
        Wavefront wf;
        const SceneEntry* scenes;  // nullptr: one scene rooted at node 0
        int stackCap = 0;          // traversal stack entries a ray may use (0 = the kernel's whole stack)
        static constexpr int kPhase = 0;
        static constexpr bool kFixedTmin = true;   // every wavefront ray starts at kMinT
        __device__ uint32_t root(uint32_t tag) const { return scenes ? __ldg(&scenes[tag >> kSlotBits].root) : 0u; }
        __device__ Counters* counters() const { return wf.ctr; }
        __device__ uint32_t count() const { return wf.ctr->rayCount[wf.ctr->cur]; }
        __device__ uint32_t* cursor() const { return &wf.ctr->traceCursor; }
        __device__ void load(uint32_t i, float3& o, float3& d, float& tmin, float& tmax, uint32_t& tag) const
        {
            const uint32_t cur = wf.ctr->cur;
            const float4 a = wf.rayO[cur][i], b = wf.rayD[cur][i];
            o = make_float3(a.x, a.y, a.z);
            d = make_float3(b.x, b.y, b.z);
            tmin = kMinT;
            tmax = b.w;
            tag = __float_as_uint(a.w);
        }
        // A hit enters its shading model's queue with the ray (origin, tag, direction) beside it, so
        // the shading kernel reads one contiguous entry instead of gathering the ray and the hit.
        __device__ void finish(uint32_t, uint32_t tag, const HitRecord& h, bool, float3 o, float3 d) const
        {
            if (h.tri != kInvalid)
            {
                const uint32_t pos = agg_push_keyed(wf.ctr->matCount, h.model);
                float4* e = wf.matQ[h.model] + static_cast<size_t>(pos) * 3;
                e[0] = make_float4(o.x, o.y, o.z, __uint_as_float(tag));
                e[1] = make_float4(d.x, d.y, d.z, kMaxT);
                e[2] = make_float4(__uint_as_float(h.tri), h.u, h.v, h.t);
            }
            else
            {
                path_finished(wf, wf.ctr, tag & kSlotMask);
            }
        }
    };

    // Shadow radiance clamp, Intersect.cu:125-134.
    __device__ __forceinline__ float3 clamp_radiance(float3 radiance, float maxLength)
    {
        const float lengthSquared = dot(radiance, radiance);
        const float maxLengthSquared = maxLength * maxLength;
        if (lengthSquared > maxLengthSquared) radiance = radiance * (maxLength * rsqrt_f(lengthSquared));
        return radiance;
    }

    struct WavefrontShadow
    {
        SceneView sc;
        Wavefront wf;
        const SceneEntry* scenes;
        int stackCap = 0;
        static constexpr int kPhase = 2;
        static constexpr bool kFixedTmin = true;
        __device__ uint32_t root(uint32_t tag) const { return scenes ? __ldg(&scenes[tag >> kSlotBits].root) : 0u; }
        __device__ Counters* counters() const { return wf.ctr; }
        __device__ uint32_t count() const { return wf.ctr->shadowCount; }
        __device__ uint32_t* cursor() const { return &wf.ctr->shadowCursor; }
        __device__ void load(uint32_t i, float3& o, float3& d, float& tmin, float& tmax, uint32_t& tag) const
        {
            const float4 a = wf.shO[i], b = wf.shD[i];
            o = make_float3(a.x, a.y, a.z);
            d = make_float3(b.x, b.y, b.z);
            tmin = kMinT;
            tmax = b.w;
            tag = __float_as_uint(a.w);
        }
        __device__ void finish(uint32_t i, uint32_t tag, const HitRecord&, bool occluded, float3, float3) const
        {
            if (occluded) return;
            const uint32_t slot = tag & kSlotMask;
            const float4 l = wf.shL[i];
            const float3 add = clamp_radiance(make_float3(l.x, l.y, l.z), 20.0f);
            float4 acc = wf.slotL[slot];
            acc.x = acc.x + add.x;
            acc.y = acc.y + add.y;
            acc.z = acc.z + add.z;
            wf.slotL[slot] = acc;
        }
    };

    struct BatchRays
    {
        SceneView sc;
        const float* rays;
        uint32_t n;
        uint32_t* cursorPtr;
        uint32_t* triOut;
        float* uvtOut;
        uint8_t* occOut;
        uint32_t rootNode;
        int stackCap = 0;
        static constexpr int kPhase = 0;
        static constexpr bool kFixedTmin = false;  // per-ray tMin of the caller's batch
        __device__ uint32_t root(uint32_t) const { return rootNode; }
        __device__ Counters* counters() const { return nullptr; }
        __device__ uint32_t count() const { return n; }
        __device__ uint32_t* cursor() const { return cursorPtr; }
        __device__ void load(uint32_t i, float3& o, float3& d, float& tmin, float& tmax, uint32_t& tag) const
        {
            const float* r = rays + static_cast<size_t>(i) * 8;
            o = make_float3(r[0], r[1], r[2]);
            d = make_float3(r[3], r[4], r[5]);
            tmin = r[6];
            tmax = r[7];
            tag = i;
        }
        __device__ void finish(uint32_t i, uint32_t, const HitRecord& h, bool occluded, float3, float3) const
        {
            if (occOut)
            {
                occOut[i] = occluded ? 1 : 0;
                return;
            }
            triOut[i] = h.tri;
            uvtOut[static_cast<size_t>(i) * 3 + 0] = h.tri != kInvalid ? h.u : 0.0f;
            uvtOut[static_cast<size_t>(i) * 3 + 1] = h.tri != kInvalid ? h.v : 0.0f;
            uvtOut[static_cast<size_t>(i) * 3 + 2] = h.tri != kInvalid ? h.t : 0.0f;
        }
    };

    // Persistent traversal: each warp keeps 32 rays in flight; when at least `refill` lanes are
    // idle the warp takes that many new rays with one atomic (ballot + popc + shuffle), so lanes
    // that finished early are refilled instead of idling until the slowest ray of the warp ends.
    // Traversal stack: STACK entries per thread in shared memory, entry = node << 8 | child mask.
    // BINARY: the binary FP32 BVH with a per-thread stack of kMaxStack entries in local memory (the
    // plain format); otherwise the BVH8 with the shared-memory stack.
    // Shared memory: [cold slots: 2 x float4 per thread][BVH8 stack: STACK words per thread].
    template <int STACK, bool ANY, int MINB, bool BINARY, class Work>
    __global__ void __launch_bounds__(128, MINB) trace_kernel(Work work, uint32_t refill, uint32_t* errorFlags)
    {
        extern __shared__ float4 smem4[];
        uint32_t localStack[BINARY ? kMaxStack : 1];
        uint32_t* stack;
        uint32_t stride;
        const ColdSlot cold{smem4 + 2u * threadIdx.x};
        if constexpr (BINARY)
        {
            stack = localStack;
            stride = 1;
        }
        else
        {
            stack = reinterpret_cast<uint32_t*>(smem4 + 2u * blockDim.x) + threadIdx.x;
            stride = blockDim.x;
        }
        Counters* ctr = work.counters();
        phase_begin(ctr, Work::kPhase);
        const uint32_t n = work.count();
        // entries a ray may push: the stack's capacity, or the caller's smaller bound (pushes beyond it
        // are refused and reported as an overflow)
        const int cap = (work.stackCap > 0 && work.stackCap < STACK) ? work.stackCap : STACK;
        uint32_t counts = 0;  // node visits | triangle tests << 16
        const uint32_t lane = lane_id();
        TraversalState st;
        bool active = false;
        bool exhausted = false;
        for (;;)
        {
            const unsigned idle = __ballot_sync(0xFFFFFFFFu, !active);
            if (!exhausted && static_cast<uint32_t>(__popc(idle)) >= refill)
            {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(work.cursor(), static_cast<uint32_t>(__popc(idle)));
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= n) exhausted = true;
                if (!active)
                {
                    unsigned laneMaskLt;
                    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(laneMaskLt));
                    const uint32_t i = base + static_cast<uint32_t>(__popc(idle & laneMaskLt));
                    if (i < n)
                    {
                        float3 o, d;
                        float tmin, tmax;
                        uint32_t tag;
                        work.load(i, o, d, tmin, tmax, tag);
                        cold.p[0] = make_float4(d.x, d.y, d.z, __uint_as_float(tag));
                        cold.p[1] = make_float4(0.0f, 0.0f, __uint_as_float(kInvalid), __uint_as_float(i));
                        st.ray = make_ray(o, d, tmin);
                        // Any-hit rays visit a node's children far to near (from the light's end of the
                        // segment): the first occluder found ends the ray, and occluders lie nearer the
                        // light more often than near the shaded point (8.19M-triangle scene: 12.2 instead
                        // of 15.0 node visits per shadow ray). The order changes no result.
                        if (ANY) st.ray.oct ^= 7u;
                        st.hitT = tmax;
                        if constexpr (BINARY)
                        {
                            st.pending = work.root(tag);
                            st.sp = 0;
                        }
                        else
                        {
                            stack[0] = work.root(tag) << 8;
                            st.sp = 1;
                        }
                        active = true;
                    }
                }
            }
            if (__ballot_sync(0xFFFFFFFFu, active) == 0)
            {
                if (exhausted) break;
                continue;
            }
            if (active)
            {
                bool occluded = false;
                bool more = true;
#pragma unroll 1
                for (int k = 0; k < 4 && more; k++)
                {
                    if constexpr (BINARY)
                        more = traverse_step_binary<ANY, Work::kFixedTmin>(work.sc, st, cold, stack, cap, occluded, errorFlags, counts);
                    else
                        more = traverse_step<ANY, Work::kFixedTmin>(work.sc, st, cold, stack, stride, cap, occluded, errorFlags, counts);
                }
                if (!more)
                {
                    const float4 c0 = cold.p[0], c1 = cold.p[1];
                    const uint32_t best = __float_as_uint(c1.z);
                    HitRecord h;
                    h.t = st.hitT;
                    h.tri = best == kInvalid ? kInvalid : (best & 0xFFFFFFu);
                    h.u = c1.x;
                    h.v = c1.y;
                    h.model = best == kInvalid ? 0u : (best >> 24);
                    work.finish(__float_as_uint(c1.w), __float_as_uint(c0.w), h, occluded, st.ray.o, make_float3(c0.x, c0.y, c0.z));
                    active = false;
                }
                // a step adds at most 8 x 255 tests: flush the packed counters well before a field overflows
                if (ctr != nullptr && (counts & 0x80008000u))
                {
                    atomicAdd(&ctr->nodeVisits[ANY ? 1 : 0], static_cast<unsigned long long>(counts & 0xFFFFu));
                    atomicAdd(&ctr->triTests[ANY ? 1 : 0], static_cast<unsigned long long>(counts >> kTestShift));
                    counts = 0;
                }
            }
        }
        if (ctr != nullptr)
        {
            unsigned long long v = counts & 0xFFFFu, t = counts >> kTestShift;
            for (int o = 16; o > 0; o >>= 1)
            {
                v += __shfl_down_sync(0xFFFFFFFFu, v, o);
                t += __shfl_down_sync(0xFFFFFFFFu, t, o);
            }
            if (lane == 0)
            {
                atomicAdd(&ctr->nodeVisits[ANY ? 1 : 0], v);
                atomicAdd(&ctr->triTests[ANY ? 1 : 0], t);
            }
        }
        phase_end(ctr, Work::kPhase);
    }

    // ------------------------------------------------------------------ random numbers
    // A path's stream, positioned at the number of 32-bit words it has drawn (kept in the path slot).
    //   Philox (the reference's): cuRAND's device API, seed 1234, subsequence = sample index; the
    //     position is curand_init's offset, which continues the stream bit for bit.
    //   PCG32: PCG-XSH-RR with 64-bit state (O'Neill, "PCG: A Family of Simple Fast Space-Efficient
    //     Statistically Good Algorithms for Random Number Generation", 2014), one stream per sample,
    //     seeded by a hash of (seed, key) where key = pixel * spp + sample within the pixel (+ the
    //     shard offset) names (pixel, sample) uniquely, and positioned by the LCG's jump-ahead (Brown,
    //     "Random Number Generation with Arbitrary Strides", 1994). Uniforms are (w >> 8) 2^-24 +
    //     2^-25, in (0, 1]. Stateless per draw position, so a slot needs no stored generator state.
    __host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)  // splitmix64's finaliser (Steele, Lea, Flood, OOPSLA 2014)
    {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }

    constexpr uint64_t kPcgMultiplier = 6364136223846793005ull;

    struct Pcg32
    {
        uint64_t state, inc;
        __device__ __forceinline__ uint32_t next()
        {
            const uint64_t old = state;
            state = old * kPcgMultiplier + inc;
            const uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
            const uint32_t rot = static_cast<uint32_t>(old >> 59u);
            return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
        }
        __device__ __forceinline__ float uniform() { return static_cast<float>(next() >> 8) * 0x1p-24f + 0x1p-25f; }
        // state after `delta` more steps: the LCG's affine map raised to the delta-th power by squaring
        __device__ __forceinline__ void advance(uint64_t delta)
        {
            uint64_t accMult = 1, accPlus = 0, curMult = kPcgMultiplier, curPlus = inc;
            while (delta > 0)
            {
                if (delta & 1u)
                {
                    accMult *= curMult;
                    accPlus = accPlus * curMult + curPlus;
                }
                curPlus = (curMult + 1) * curPlus;
                curMult *= curMult;
                delta >>= 1;
            }
            state = accMult * state + accPlus;
        }
        // the generator's seeding: stream (increment) from initseq, then initstate mixed in over two steps
        __device__ __forceinline__ static Pcg32 seeded(uint64_t key)
        {
            Pcg32 g;
            const uint64_t initstate = mix64(kRandomSeed ^ mix64(key));
            const uint64_t initseq = mix64(key ^ 0x9E3779B97F4A7C15ull);
            g.state = 0;
            g.inc = (initseq << 1u) | 1u;
            g.next();
            g.state += initstate;
            g.next();
            return g;
        }
    };

    struct PathRng
    {
        curandStatePhilox4_32_10_t philox;
        Pcg32 pcg;
        bool usePcg;
        __device__ __forceinline__ void init(uint32_t policy, uint64_t key, uint32_t position)
        {
            usePcg = policy == kRngPcg32;
            if (usePcg)
            {
                pcg = Pcg32::seeded(key);
                pcg.advance(position);
            }
            else
                curand_init(kRandomSeed, static_cast<unsigned long long>(key), static_cast<unsigned long long>(position), &philox);
        }
        __device__ __forceinline__ float4 uniform4()
        {
            if (usePcg)
            {
                const float x = pcg.uniform();
                const float y = pcg.uniform();
                const float z = pcg.uniform();
                const float w = pcg.uniform();
                return make_float4(x, y, z, w);
            }
            return curand_uniform4(&philox);
        }
        __device__ __forceinline__ float uniform() { return usePcg ? pcg.uniform() : curand_uniform(&philox); }
    };

    // ------------------------------------------------------------------ paths
    __device__ __forceinline__ uint32_t pack_meta(uint32_t depth, bool delta, uint32_t job)
    {
        return depth | (delta ? 0x100u : 0u) | (job << 16);
    }

    // ComputePathSample + GenerateCameraRay (PathGeneration.cu:15-54).
    __device__ __forceinline__ void camera_ray(const JobView& job, uint64_t sampleIndex, float2 jitter, float3& o, float3& d)
    {
        const uint64_t spp = job.spp;
        const uint64_t pixelQ = sampleIndex / spp;
        const uint32_t pixelIndex = static_cast<uint32_t>(pixelQ);
        const uint32_t sampleGridIndex = static_cast<uint32_t>(sampleIndex - pixelQ * spp);
        const uint32_t yq = pixelIndex / job.width;
        const uint32_t x = pixelIndex - yq * job.width;
        const uint32_t y = yq;
        const uint32_t sgq = sampleGridIndex / job.spa;
        const uint32_t sgx = sampleGridIndex - sgq * job.spa;
        const uint32_t sgy = sgq;
        const float u = (static_cast<float>(x) + (static_cast<float>(sgx) + jitter.x) / static_cast<float>(job.spa)) / static_cast<float>(job.width);
        const float v = (static_cast<float>(y) + (static_cast<float>(sgy) + jitter.y) / static_cast<float>(job.spa)) / static_cast<float>(job.height);
        const float3 origin = make_float3(job.camera[0], job.camera[1], job.camera[2]);
        const float3 llc = make_float3(job.camera[3], job.camera[4], job.camera[5]);
        const float3 hor = make_float3(job.camera[6], job.camera[7], job.camera[8]);
        const float3 ver = make_float3(job.camera[9], job.camera[10], job.camera[11]);
        d = normalize(llc + u * hor + v * ver - origin);
        o = origin;
    }

    // New path for a sample in a slot: Philox stream (seed 1234, subsequence = sample), jitter from
    // the first uniform4, throughput 1, depth 0, delta flag set (PathGeneration.cu:56-102).
    __device__ __forceinline__ void start_path(const JobView& job, uint32_t jobIndex, const Wavefront& wf, uint32_t slot, uint32_t sample,
                                               uint32_t queue, uint32_t position)
    {
        PathRng rng;
        rng.init(job.rngPolicy, static_cast<uint64_t>(sample) + job.rngOffset, 0u);
        const float4 r = rng.uniform4();
        float3 o, d;
        camera_ray(job, sample, make_float2(r.x, r.y), o, d);
        wf.slotT[slot] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(pack_meta(0, true, jobIndex)));
        wf.slotL[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(4u));
        wf.slotSample[slot] = sample;
        wf.rayO[queue][position] = make_float4(o.x, o.y, o.z, __uint_as_float(slot | (job.scene << kSlotBits)));
        wf.rayD[queue][position] = make_float4(d.x, d.y, d.z, kMaxT);
    }

    __global__ void frame_init_kernel(Wavefront wf, const JobView* job, uint32_t pool)
    {
        Counters* c = wf.ctr;
        const uint64_t total = job->totalSamples;
        const uint32_t gen = static_cast<uint32_t>(total < pool ? total : pool);
        c->rayCount[0] = gen;
        c->rayCount[1] = 0;
        c->cur = 0;
        for (uint32_t m = 0; m < kModelCount; m++) c->matCount[m] = 0;
        c->shadowCount = 0;
        c->regenCount = 0;
        c->traceCursor = 0;
        c->shadowCursor = 0;
        c->regenCursor = 0;
        c->iteration = 0;
        c->done = gen == 0 ? 1u : 0u;
        c->errorFlags = 0;
        c->launched = gen;
        c->raysTraced = 0;
        c->shadowRaysTraced = 0;
        for (int p = 0; p < 4; p++)
        {
            c->tStart[p] = ~0ull;
            c->tEnd[p] = 0;
            c->tAccum[p] = 0;
        }
        for (int k = 0; k < 2; k++)
        {
            c->nodeVisits[k] = 0;
            c->triTests[k] = 0;
        }
    }

    __global__ void generate_kernel(Wavefront wf, const JobView* jobPtr)
    {
        const JobView job = *jobPtr;
        const uint32_t n = wf.ctr->rayCount[0];
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            start_path(job, 0, wf, i, i, 0, i);
        if (wf.regenBits != nullptr)
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (wf.capacity + 31u) >> 5; i += gridDim.x * blockDim.x)
                wf.regenBits[i] = 0u;
    }

    // Regeneration from the finished-slot bitmap: each warp takes a tile of 32 bitmap words (1,024
    // slots), reserves new samples for the tile's finished paths with one atomic, and walks the words in
    // slot order, so the slot records of finished and new paths are read and written in address order
    // (the queue holds them in the order paths finished, i.e. scattered). The set of new samples, their
    // ray-queue positions and every sample's result are those of the queue-driven regeneration; only
    // which slot a new sample lands in differs.
    constexpr uint32_t kRegenGroup = 4;  // bitmap words whose finished slots are loaded together

    __global__ void regen_bits_kernel(Wavefront wf, const JobView* jobPtr)
    {
        Counters* ctr = wf.ctr;
        phase_begin(ctr, 3);
        const unsigned long long launched = ctr->launched;
        const unsigned long long remaining = jobPtr->totalSamples - launched;
        const uint32_t regenerate = static_cast<uint32_t>(remaining < ctr->regenCount ? remaining : ctr->regenCount);
        const uint32_t nxt = ctr->cur ^ 1u;
        const uint32_t base = ctr->rayCount[nxt];
        float* out = jobPtr->sampleRadiance;
        const uint32_t words = (wf.capacity + 31u) >> 5;
        const uint32_t tiles = (words + 31u) >> 5;
        const uint32_t lane = lane_id();
        const uint32_t lanesBelow = (1u << lane) - 1u;
        const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
        for (uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < tiles; tile += warps)
        {
            const uint32_t wi = tile * 32u + lane;
            const uint32_t bits = wi < words ? wf.regenBits[wi] : 0u;
            if (bits) wf.regenBits[wi] = 0u;
            const uint32_t count = static_cast<uint32_t>(__popc(bits));
            uint32_t incl = count;
            for (int o = 1; o < 32; o <<= 1)
            {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (static_cast<int>(lane) >= o) incl += v;
            }
            const uint32_t tileTotal = __shfl_sync(0xFFFFFFFFu, incl, 31);
            if (tileTotal == 0) continue;
            uint32_t first = 0;
            if (lane == 0) first = atomicAdd(&ctr->regenCursor, tileTotal);
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            const uint32_t excl = incl - count;
            // words in groups of kRegenGroup: the finished slots' loads of a group are in flight together
            for (uint32_t jb = 0; jb < 32; jb += kRegenGroup)
            {
                uint32_t w[kRegenGroup], offset[kRegenGroup], sample[kRegenGroup];
                float4 L[kRegenGroup];
#pragma unroll
                for (uint32_t q = 0; q < kRegenGroup; q++)
                {
                    w[q] = __shfl_sync(0xFFFFFFFFu, bits, jb + q);
                    offset[q] = __shfl_sync(0xFFFFFFFFu, excl, jb + q);
                    L[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    sample[q] = 0;
                    if ((w[q] >> lane) & 1u)
                    {
                        const uint32_t slot = (tile * 32u + jb + q) * 32u + lane;
                        L[q] = wf.slotL[slot];
                        sample[q] = wf.slotSample[slot];
                    }
                }
#pragma unroll
                for (uint32_t q = 0; q < kRegenGroup; q++)
                {
                    if (!((w[q] >> lane) & 1u)) continue;
                    const uint32_t slot = (tile * 32u + jb + q) * 32u + lane;
                    float* dst = out + static_cast<size_t>(sample[q]) * 3;
                    dst[0] = L[q].x;
                    dst[1] = L[q].y;
                    dst[2] = L[q].z;
                    const uint32_t k = first + offset[q] + static_cast<uint32_t>(__popc(w[q] & lanesBelow));
                    if (k < regenerate) start_path(*jobPtr, 0, wf, slot, static_cast<uint32_t>(launched + k), nxt, base + k);
                }
            }
        }
        phase_end(ctr, 3);
    }

    // ------------------------------------------------------------------ shading (MaterialEval.cu)
    struct Frame
    {
        float3 tangent, bitangent, normal;
        __device__ float3 to_local(float3 v) const { return make_float3(dot(v, tangent), dot(v, bitangent), dot(v, normal)); }
        __device__ float3 from_local(float3 v) const { return v.x * tangent + v.y * bitangent + v.z * normal; }
    };

    __device__ __forceinline__ float3 safe_normalize(float3 v, float3 fallback)
    {
        const float l2 = dot(v, v);
        if (l2 > 1e-16f) return v * rsqrt_f(l2);
        return fallback;
    }

    __device__ __forceinline__ Frame frame_from_normal(float3 n)  // Math.hpp:120-134
    {
        float3 t;
        if (fabsf(n.x) > fabsf(n.z)) t = normalize(make_float3(n.y, -n.x, 0.0f));
        else t = normalize(make_float3(0.0f, n.z, -n.y));
        return Frame{t, cross(n, t), n};
    }

    __device__ __forceinline__ Frame frame_from(float3 n, float3 t, float sign)  // Math.hpp:136-148
    {
        n = safe_normalize(n, make_float3(0.0f, 0.0f, 1.0f));
        t = t - n * dot(n, t);
        const float l2 = dot(t, t);
        if (l2 > 1e-16f) t = t * rsqrt_f(l2);
        else t = frame_from_normal(n).tangent;
        return Frame{t, cross(n, t) * sign, n};
    }

    struct Surface
    {
        float3 position, gN, normal;
        float4 tangent;
        float2 uv;
        uint32_t material;
    };

    // LoadResolvedHit (MaterialEval.cu:54-87).
    __device__ __forceinline__ Surface resolve_hit(const SceneView& sc, float3 o, float3 d, float tHit, uint32_t tri, float u, float v)
    {
        const float4* rec = sc.shading + static_cast<size_t>(tri) * 9;
        const float b0 = 1.0f - u - v;
        const float b1 = u;
        const float b2 = v;
        Surface s;
        s.position = o + d * tHit;
        const float4 g = ldg4(rec + 6);
        float3 gn = make_float3(g.x, g.y, g.z);
        if (dot(gn, d) > 0.0f) gn = -gn;
        s.gN = gn;
        s.material = __float_as_uint(g.w);
        const float4 n0 = ldg4(rec + 0), n1 = ldg4(rec + 1), n2 = ldg4(rec + 2);
        s.normal = b0 * f3(n0) + b1 * f3(n1) + b2 * f3(n2);
        const float4 t0 = ldg4(rec + 3), t1 = ldg4(rec + 4), t2 = ldg4(rec + 5);
        s.tangent = b0 * t0 + b1 * t1 + b2 * t2;
        // uv only feeds texture lookups: without image textures every slot is a constant, so the
        // record's last 32 bytes are not read
        if (sc.textures != nullptr)
        {
            const float4 u01 = ldg4(rec + 7), u2 = ldg4(rec + 8);
            s.uv = b0 * make_float2(u01.x, u01.y) + b1 * make_float2(u01.z, u01.w) + b2 * make_float2(u2.x, u2.y);
        }
        else
            s.uv = make_float2(0.0f, 0.0f);
        return s;
    }

    // Material slot value: the slot's texture sampled at uv (TextureView::Sample, TextureView.hpp:17-20)
    // when the material has one, else its constant texel.
    __device__ __forceinline__ float3 slot_rgb(const SceneView& sc, uint32_t mat, int slot, float2 uv, const float* constant)
    {
        if (sc.textures != nullptr)
        {
            const unsigned long long t = __ldg(&sc.textures[mat].tex[slot]);
            if (t != 0)
            {
                const float4 v = tex2D<float4>(t, uv.x, uv.y);
                return make_float3(v.x, v.y, v.z);
            }
        }
        return make_float3(__ldg(constant), __ldg(constant + 1), __ldg(constant + 2));
    }

    __device__ __forceinline__ float slot_scalar(const SceneView& sc, uint32_t mat, int slot, float2 uv, const float* constant)
    {
        if (sc.textures != nullptr)
        {
            const unsigned long long t = __ldg(&sc.textures[mat].tex[slot]);
            if (t != 0) return tex2D<float>(t, uv.x, uv.y);
        }
        return __ldg(constant);
    }

    __device__ __forceinline__ float3 mat3(const float* v) { return make_float3(__ldg(v), __ldg(v + 1), __ldg(v + 2)); }

    // GetShadingFrame (MaterialEval.cu:89-115).
    __device__ __forceinline__ Frame shading_frame(const SceneView& sc, const Surface& s, const MaterialDev& m)
    {
        const float3 bt = make_float3(s.tangent.x, s.tangent.y, s.tangent.z);
        const float sign = s.tangent.w < 0.0f ? -1.0f : 1.0f;
        const Frame base = frame_from(s.normal, bt, sign);
        const float3 ts = normalize(slot_rgb(sc, s.material, 5, s.uv, m.normal) * 2.0f - 1.0f);
        const float3 sn = ts.x * base.tangent + ts.y * base.bitangent + ts.z * base.normal;
        return frame_from(sn, bt, sign);
    }

    __device__ __forceinline__ float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

    struct Continuation
    {
        bool terminated;
        uint32_t depth;
        float3 throughput;
    };

    // ComputePathContinuation (MaterialEval.cu:129-146).
    __device__ __forceinline__ Continuation continue_path(uint32_t depth, float3 T, uint32_t limit, float3 w, float rr)
    {
        const uint32_t next = depth + 1;
        if (next >= limit) return {true, next, f3(0.0f)};
        const float3 nt = T * w;
        if (next < kRussianRouletteStartDepth) return {false, next, nt};
        const float p = clampf(max3(nt), 0.0f, 1.0f);
        if (rr > p) return {true, next, f3(0.0f)};
        return {false, next, nt / p};
    }

    __device__ __forceinline__ float3 cosine_hemisphere(float2 u)  // :222-229
    {
        const float phi = 2.0f * kPi * u.x;
        const float cosTheta = sqrtf(u.y);
        const float sinTheta = sqrtf(1.0f - u.y);
        float s, c;
        sincos_f(phi, &s, &c);
        return make_float3(sinTheta * c, sinTheta * s, cosTheta);
    }

    struct LightHit
    {
        float3 position, gN, wi, emission;
        float distanceSquared, pdf;
    };

    // The lights of one resident scene: a slice of the packed light list and alias table.
    struct LightSet
    {
        uint32_t base, count;
        const uint4* bins;  // the job's alias table (area or power weights)
    };

    // SampleLightTriangle (MaterialEval.cu:171-192) with the alias table (AliasTableView.hpp:32-60).
    // Requires ls.count > 0 (NEE is off for scenes without emitters).
    __device__ __forceinline__ LightHit sample_light(const SceneView& sc, LightSet ls, float uSel, float2 xi, float3 hitPoint)
    {
        const uint32_t n = ls.count;
        const float scaledU = uSel * static_cast<float>(n);
        uint32_t bin = static_cast<uint32_t>(scaledU);
        bin = bin < n - 1u ? bin : n - 1u;
        const float up = fminf(scaledU - static_cast<float>(bin), kOneMinusEpsilon);
        bin += ls.base;
        const uint4 b = ldg4(ls.bins + bin);
        uint32_t index = bin;
        float pmf = __uint_as_float(b.y);
        if (!(up < __uint_as_float(b.x)))
        {
            index = b.z;
            pmf = __uint_as_float(__ldg(&ls.bins[index].y));
        }
        const float4* L = sc.lights + static_cast<size_t>(index) * 7;
        const float4 l0 = ldg4(L), l1 = ldg4(L + 1), l2 = ldg4(L + 2), l3 = ldg4(L + 3), l4 = ldg4(L + 4);
        const float s0 = sqrtf(xi.x);
        const float b1 = s0 * (1.0f - xi.y);
        const float b2 = s0 * xi.y;
        LightHit h;
        h.position = f3(l0) + b1 * f3(l1) + b2 * f3(l2);
        float3 emission = f3(l4);
        if (sc.textures != nullptr)
        {
            const float4 l5 = ldg4(L + 5), l6 = ldg4(L + 6);
            const uint32_t mat = __float_as_uint(l6.z);
            const unsigned long long t = __ldg(&sc.textures[mat].tex[4]);
            if (t != 0)
            {
                const float2 uv = make_float2(l5.x, l5.y) + b1 * make_float2(l5.z, l5.w) + b2 * make_float2(l6.x, l6.y);
                const float4 e = tex2D<float4>(t, uv.x, uv.y);
                emission = make_float3(e.x, e.y, e.z);
            }
        }
        const float3 toLight = h.position - hitPoint;
        h.distanceSquared = dot(toLight, toLight);
        h.wi = normalize(toLight);
        float3 gn = f3(l3);
        if (dot(gn, h.wi) > 0.0f) gn = -gn;
        h.gN = gn;
        h.emission = emission;
        h.pdf = pmf / l1.w;
        return h;
    }

    struct ShadowOut
    {
        bool valid;
        float3 origin, direction, radiance;
        float tMax;
    };

    __device__ __forceinline__ ShadowOut shadow_ray(float3 hitPosition, float3 gN, const LightHit& lh, float3 radiance)  // :261-267
    {
        ShadowOut s;
        s.valid = true;
        s.origin = hitPosition + gN * 1e-4f;
        const float3 v = lh.position - s.origin;
        const float dist = length(v);
        s.direction = v / dist;
        s.tMax = dist - 1e-4f;
        s.radiance = radiance;
        return s;
    }

    // Lambert NEE, EvaluateDiffuseDirect (:231-268); Phong NEE adds the lobe (:410-455).
    __device__ __forceinline__ ShadowOut direct_lambert_phong(const SceneView& sc, LightSet ls, float3 T, float3 dir, const Surface& s, const Frame& f,
                                                              float3 rs, float3 albedo, bool phong, float3 specular, float shininess)
    {
        ShadowOut none;
        none.valid = false;
        const LightHit lh = sample_light(sc, ls, rs.x, make_float2(rs.y, rs.z), s.position);
        if (lh.distanceSquared < 1e-6f) return none;
        const float cosThetaI = fmaxf(dot(f.normal, lh.wi), 0.0f);
        const float gCos = fmaxf(dot(s.gN, lh.wi), 0.0f);
        if (cosThetaI <= 0.0f || gCos <= 0.0f) return none;
        const float cosThetaLight = fmaxf(dot(lh.gN, f3(0.0f) - lh.wi), 0.0f);
        if (cosThetaLight <= 0.0f) return none;
        float3 brdf;
        if (phong)
        {
            const float3 refl = normalize(reflect(dir, f.normal));
            const float cosThetaR = fmaxf(dot(refl, lh.wi), 0.0f);
            const float3 diffuseBrdf = albedo / kPi;
            const float3 specularBrdf = specular * (shininess + 2.0f) * kInvTwoPi * pow_f(cosThetaR, shininess);
            brdf = diffuseBrdf + specularBrdf;
        }
        else
            brdf = albedo / kPi;
        const float geometryTerm = cosThetaI * cosThetaLight / lh.distanceSquared;
        const float3 radiance = lh.emission * T * brdf * geometryTerm / lh.pdf;
        return shadow_ray(s.position, s.gN, lh, radiance);
    }

    // GGX helpers (MaterialEval.cu:587-650) and Math.hpp:217-262.
    __device__ __forceinline__ float cos2_theta(float3 w) { return w.z * w.z; }
    __device__ __forceinline__ float sin2_theta(float3 w) { return fmaxf(0.0f, 1.0f - cos2_theta(w)); }
    __device__ __forceinline__ float sin_theta(float3 w) { return sqrtf(sin2_theta(w)); }
    __device__ __forceinline__ float tan2_theta(float3 w) { return sin2_theta(w) / cos2_theta(w); }
    __device__ __forceinline__ float cos_phi(float3 w)
    {
        const float st = sin_theta(w);
        return (st == 0) ? 1 : clampf(w.x / st, -1.f, 1.f);
    }
    __device__ __forceinline__ float sin_phi(float3 w)
    {
        const float st = sin_theta(w);
        return (st == 0) ? 0 : clampf(w.y / st, -1.f, 1.f);
    }
    __device__ __forceinline__ float ggx_lambda(float3 w, float alpha)
    {
        const float t2 = tan2_theta(w);
        if (t2 == INFINITY) return 0.0f;
        const float a2 = sqr(cos_phi(w) * alpha) + sqr(sin_phi(w) * alpha);
        return (sqrtf(1.0f + a2 * t2) - 1.0f) * 0.5f;
    }
    __device__ __forceinline__ float ggx_g1(float3 w, float alpha) { return 1.0f / (1.0f + ggx_lambda(w, alpha)); }
    __device__ __forceinline__ float ggx_g(float3 wo, float3 wi, float alpha) { return 1 / (1 + ggx_lambda(wo, alpha) + ggx_lambda(wi, alpha)); }
    __device__ __forceinline__ float ggx_d(float3 wm, float alpha)
    {
        const float t2 = tan2_theta(wm);
        if (t2 == INFINITY) return 0.0f;
        const float cos4 = sqr(cos2_theta(wm));
        if (cos4 < 1e-16f) return 0.0f;
        const float e = t2 * (sqr(cos_phi(wm) / alpha) + sqr(sin_phi(wm) / alpha));
        return 1 / (kPi * sqr(alpha) * cos4 * sqr(1 + e));
    }
    __device__ __forceinline__ float ggx_dv(float3 w, float3 wm, float alpha)
    {
        return ggx_g1(w, alpha) / fabsf(w.z) * ggx_d(wm, alpha) * fabsf(dot(w, wm));
    }
    __device__ __forceinline__ float3 fresnel_schlick(float3 f0, float c) { return f0 + (1.0f - f0) * pow5_f(1.0f - c); }

    __device__ __forceinline__ float3 trowbridge_sample(float3 w, float alpha, float2 u)
    {
        float3 wh = normalize(make_float3(alpha * w.x, alpha * w.y, w.z));
        if (wh.z < 0) wh = -wh;
        const float3 t = (wh.z < 0.999f) ? normalize(cross(wh, make_float3(0.0f, 0.0f, 1.0f))) : make_float3(1.0f, 0.0f, 0.0f);
        const float3 b = cross(wh, t);
        const float r = sqrtf(u.x);
        const float theta = 2.0f * kPi * u.y;
        float sn, cs;
        sincos_f(theta, &sn, &cs);
        float2 disk = make_float2(r * cs, r * sn);
        const float h = sqrtf(1.0f - disk.x * disk.x);
        disk.y = lerpf(h, disk.y, (1 + wh.z) * 0.5f);
        const float pz = sqrtf(fmaxf(0.0f, 1.0f - dot(disk, disk)));
        const float3 nh = disk.x * t + disk.y * b + pz * wh;
        return normalize(make_float3(alpha * nh.x, alpha * nh.y, fmaxf(1e-6f, nh.z)));
    }

    // EvaluateGgxDirect (:652-718)
    __device__ __forceinline__ ShadowOut direct_ggx(const SceneView& sc, LightSet ls, float3 T, float3 dir, const Surface& s, const Frame& f, float3 rs,
                                                    float3 base, float alpha, float metallic, float ior)
    {
        ShadowOut none;
        none.valid = false;
        const LightHit lh = sample_light(sc, ls, rs.x, make_float2(rs.y, rs.z), s.position);
        if (lh.distanceSquared < 1e-6f || lh.pdf <= 0.0f) return none;
        if (dot(s.gN, lh.wi) <= 0.0f) return none;
        const float cosThetaLight = fmaxf(dot(lh.gN, f3(0.0f) - lh.wi), 0.0f);
        if (cosThetaLight <= 0.0f) return none;
        const float3 wo = f.to_local(f3(0.0f) - dir);
        const float3 wi = f.to_local(lh.wi);
        const float cosThetaI = wi.z;
        const float cosThetaO = wo.z;
        if (cosThetaI <= 0.0f || cosThetaO <= 0.0f) return none;
        const float3 wm = normalize(wo + wi);
        if (wm.z <= 0.0f) return none;
        const float woDotWm = dot(wo, wm);
        const float wiDotWm = dot(wi, wm);
        if (woDotWm <= 1e-6f || wiDotWm <= 1e-6f) return none;
        const float dielectricF0 = sqr((1.0f - ior) / (1.0f + ior));
        const float3 f0 = lerp3(f3(dielectricF0), base, metallic);
        const float3 diffuseColor = base * (1.0f - metallic);
        const float3 F = fresnel_schlick(f0, clampf(woDotWm, 0.0f, 1.0f));
        const float3 diffuseBsdf = (1.0f - F) * diffuseColor * kInvPi;
        const float3 ggxBsdf = F * ggx_d(wm, alpha) * ggx_g(wo, wi, alpha) / (4.0f * cosThetaI * cosThetaO);
        const float3 bsdf = diffuseBsdf + ggxBsdf;
        const float geometryTerm = cosThetaI * cosThetaLight / lh.distanceSquared;
        const float3 radiance = lh.emission * T * bsdf * geometryTerm / lh.pdf;
        return shadow_ray(s.position, s.gN, lh, radiance);
    }

    struct Scatter
    {
        bool terminated;
        Continuation c;
        float3 direction;
    };

    __device__ __forceinline__ Scatter scatter_terminated()
    {
        Scatter s;
        s.terminated = true;
        return s;
    }

    // EvaluateGgxIndirect (:720-836)
    __device__ __forceinline__ Scatter indirect_ggx(uint32_t depth, float3 T, uint32_t limit, float3 dir, const Surface& s, const Frame& f,
                                                    float4 rs, float3 base, float alpha, float metallic, float ior)
    {
        const float3 wo = f.to_local(f3(0.0f) - dir);
        if (wo.z <= 0.0f) return scatter_terminated();
        const float dielectricF0 = sqr((1.0f - ior) / (1.0f + ior));
        const float3 f0 = lerp3(f3(dielectricF0), base, metallic);
        const float3 diffuseColor = base * (1.0f - metallic);
        const float dw = luminance(diffuseColor);
        const float sw = luminance(f0);
        const float ws = dw + sw;
        if (ws <= 1e-6f) return scatter_terminated();
        const float dsp = dw / ws;
        const float ssp = sw / ws;
        float3 wi;
        if (rs.z < dsp) wi = cosine_hemisphere(make_float2(rs.x, rs.y));
        else wi = reflect(-wo, trowbridge_sample(wo, alpha, make_float2(rs.x, rs.y)));
        const float cosThetaI = wi.z;
        const float cosThetaO = wo.z;
        if (cosThetaI <= 0.0f) return scatter_terminated();
        const float3 wm = normalize(wi + wo);
        if (wm.z <= 0.0f) return scatter_terminated();
        const float woDotWm = dot(wo, wm);
        if (woDotWm <= 1e-6f) return scatter_terminated();
        const float3 F = fresnel_schlick(f0, clampf(woDotWm, 0.0f, 1.0f));
        const float3 diffuseBsdf = (1.0f - F) * diffuseColor * kInvPi;
        const float3 ggxBsdf = F * ggx_d(wm, alpha) * ggx_g(wo, wi, alpha) / (4.0f * cosThetaI * cosThetaO);
        const float diffusePdf = cosThetaI * kInvPi;
        const float ggxPdf = ggx_dv(wo, wm, alpha) / (4.0f * woDotWm);
        const float pdf = dsp * diffusePdf + ssp * ggxPdf;
        if (pdf <= 1e-8f) return scatter_terminated();
        const float3 worldWi = f.from_local(wi);
        if (dot(worldWi, s.gN) <= 0.0f) return scatter_terminated();
        Scatter out;
        out.c = continue_path(depth, T, limit, (diffuseBsdf + ggxBsdf) * (cosThetaI / pdf), rs.w);
        out.terminated = out.c.terminated;
        out.direction = worldWi;
        return out;
    }

    // EvaluatePhongIndirect (:457-542)
    __device__ __forceinline__ Scatter indirect_phong(uint32_t depth, float3 T, uint32_t limit, float3 dir, const Surface& s, const Frame& f,
                                                      float4 rs, float3 albedo, float3 specular, float shininess)
    {
        const float dw = luminance(albedo);
        const float sw = luminance(specular);
        const float ws = dw + sw;
        if (ws <= 0.0f) return scatter_terminated();
        const float dsp = dw / ws;
        const float ssp = 1.0f - dsp;
        const float3 refl = normalize(reflect(dir, f.normal));
        float3 wi;
        if (rs.z < dsp)
            wi = f.from_local(cosine_hemisphere(make_float2(rs.x, rs.y)));
        else
        {
            const float phi = 2.0f * kPi * rs.x;
            const float cosTheta = pow_f(rs.y, 1.0f / (shininess + 1.0f));
            const float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
            float sn, cs;
            sincos_f(phi, &sn, &cs);
            wi = frame_from_normal(refl).from_local(make_float3(sinTheta * cs, sinTheta * sn, cosTheta));
        }
        const float cosThetaI = fmaxf(dot(f.normal, wi), 0.0f);
        const float gCos = fmaxf(dot(s.gN, wi), 0.0f);
        if (cosThetaI <= 0.0f || gCos <= 0.0f) return scatter_terminated();
        const float cosThetaR = fmaxf(dot(refl, wi), 0.0f);
        const float lobe = kInvTwoPi * pow_f(cosThetaR, shininess);
        const float diffusePdf = cosThetaI * kInvPi;
        const float specularPdf = (shininess + 1.0f) * lobe;
        const float pdf = dsp * diffusePdf + ssp * specularPdf;
        if (pdf <= 0.0f) return scatter_terminated();
        const float3 diffuseBrdf = albedo * kInvPi;
        const float3 specularBrdf = specular * (shininess + 2.0f) * lobe;
        Scatter out;
        out.c = continue_path(depth, T, limit, (diffuseBrdf + specularBrdf) * (cosThetaI / pdf), rs.w);
        out.terminated = out.c.terminated;
        out.direction = wi;
        return out;
    }

    // One kernel per shading model; blocks stride over the model's queue, one entry per thread. A
    // path's job (its depth limit, NEE switch and Philox offset) comes from its slot metadata, its
    // scene (lights) from the ray tag; NEE is off in scenes without emitters. Each block pushes its
    // extension rays and its shadow rays with one atomic each, grouped by direction octant: a
    // traversal warp then takes runs of rays leaving neighbouring surfaces (a block's entries come
    // from neighbouring hits) in the same octant. Queue order changes no result.
    template <uint32_t MODEL>
    __global__ void __launch_bounds__(128) shade_kernel(SceneView sc, Wavefront wf, const JobView* jobs, const SceneEntry* scenes)
    {
        Counters* ctr = wf.ctr;
        phase_begin(ctr, 1);
        const uint32_t n = ctr->matCount[MODEL];
        const uint32_t cur = ctr->cur;
        const uint32_t nxt = cur ^ 1u;
        const float4* queue = wf.matQ[MODEL];
        __shared__ uint32_t octCount[16], octBase[16], blockBase[2];
        for (uint32_t kb = blockIdx.x * blockDim.x; kb < n; kb += gridDim.x * blockDim.x)
        {
            const uint32_t k = kb + threadIdx.x;
            bool pushRay = false, pushShadow = false;
            float4 rayOut0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), rayOut1 = rayOut0;
            float4 shOut0 = rayOut0, shOut1 = rayOut0, shOut2 = rayOut0;
            if (k < n)
            {
                const float4* entry = queue + static_cast<size_t>(k) * 3;
                const float4 o4 = entry[0];
                const float4 d4 = entry[1];
                const float4 h4 = entry[2];
                const uint32_t tag = __float_as_uint(o4.w);
                const uint32_t slot = tag & kSlotMask;
                const float3 o = f3(o4), d = f3(d4);
                const float tHit = h4.w;
                const uint32_t tri = __float_as_uint(h4.x);
                const float4 T4 = wf.slotT[slot];
                float4 L4 = wf.slotL[slot];
                const uint32_t meta = __float_as_uint(T4.w);
                const uint32_t depth = meta & 0xFFu;
                const bool delta = (meta & 0x100u) != 0;
                const uint32_t jobIndex = meta >> 16;
                const JobView& job = jobs[jobIndex];
                const uint32_t limit = __ldg(&job.depthLimit);
                const uint4 se = __ldg(reinterpret_cast<const uint4*>(scenes) + (tag >> kSlotBits));
                const LightSet ls{se.y, se.z, __ldg(&job.lightMode) == kLightsPower ? sc.binsPower : sc.bins};
                const bool nee = __ldg(&job.nee) != 0 && ls.count > 0;
                const float3 T = f3(T4);
                uint32_t rngPos = __float_as_uint(L4.w);
                bool terminated = true;
                float3 nextDir = f3(0.0f);
                float3 nextGn = f3(0.0f);
                Continuation cont{true, 0, f3(0.0f)};
                bool nextDelta = false;
                ShadowOut sh;
                sh.valid = false;
                float3 hitPos = f3(0.0f);

                if (MODEL == 5)  // Emissive (:882-912)
                {
                    if (!(nee && !delta))
                    {
                        // LoadPartiallyResolvedHit (MaterialEval.cu:32-52): material and interpolated uv
                        const float4* rec = sc.shading + static_cast<size_t>(tri) * 9;
                        const uint32_t mat = __float_as_uint(__ldg(&rec[6].w));
                        const float b0 = 1.0f - h4.y - h4.z;
                        float2 uv = make_float2(0.0f, 0.0f);
                        if (sc.textures != nullptr)
                        {
                            const float4 u01 = ldg4(rec + 7), u2 = ldg4(rec + 8);
                            uv = b0 * make_float2(u01.x, u01.y) + h4.y * make_float2(u01.z, u01.w) + h4.z * make_float2(u2.x, u2.y);
                        }
                        const float3 em = slot_rgb(sc, mat, 4, uv, sc.materials[mat].emission);
                        const float3 c = T * em;
                        L4.x = L4.x + c.x;
                        L4.y = L4.y + c.y;
                        L4.z = L4.z + c.z;
                    }
                }
                else if (MODEL == 0)  // Normal (:194-220)
                {
                    const Surface s = resolve_hit(sc, o, d, tHit, tri, h4.y, h4.z);
                    const float3 c = T * s.normal * 0.5f + 0.5f;
                    L4.x = L4.x + c.x;
                    L4.y = L4.y + c.y;
                    L4.z = L4.z + c.z;
                }
                else
                {
                    const Surface s = resolve_hit(sc, o, d, tHit, tri, h4.y, h4.z);
                    hitPos = s.position;
                    nextGn = s.gN;
                    const MaterialDev& m = sc.materials[s.material];
                    const Frame f = shading_frame(sc, s, m);
                    PathRng rng;
                    rng.init(__ldg(&job.rngPolicy), static_cast<uint64_t>(wf.slotSample[slot]) + __ldg(&job.rngOffset), rngPos);
                    if (MODEL == 1)  // Diffuse (:311-350, :270-309)
                    {
                        const float3 albedo = slot_rgb(sc, s.material, 0, s.uv, m.color);
                        const float4 ind = rng.uniform4();
                        rngPos += 4;
                        if (nee)
                        {
                            const float4 dir4 = rng.uniform4();
                            rngPos += 4;
                            sh = direct_lambert_phong(sc, ls, T, d, s, f, f3(dir4), albedo, false, f3(0.0f), 0.0f);
                        }
                        const float3 wi = f.from_local(cosine_hemisphere(make_float2(ind.x, ind.y)));
                        const float cosThetaI = fmaxf(dot(f.normal, wi), 0.0f);
                        const float gCos = fmaxf(dot(s.gN, wi), 0.0f);
                        if (!(cosThetaI <= 0.0f || gCos <= 0.0f))
                        {
                            cont = continue_path(depth, T, limit, albedo, ind.z);
                            terminated = cont.terminated;
                            nextDir = wi;
                            nextDelta = false;
                        }
                    }
                    else if (MODEL == 2)  // Mirror (:352-392)
                    {
                        const float3 reflectance = slot_rgb(sc, s.material, 1, s.uv, m.specular);
                        const float rr = rng.uniform();
                        rngPos += 1;
                        const float3 wi = reflect(d, f.normal);
                        cont = continue_path(depth, T, limit, reflectance, rr);
                        terminated = cont.terminated;
                        nextDir = wi;
                        nextDelta = true;
                    }
                    else if (MODEL == 3)  // Phong (:544-585)
                    {
                        const float3 albedo = slot_rgb(sc, s.material, 0, s.uv, m.color);
                        const float3 specular = slot_rgb(sc, s.material, 1, s.uv, m.specular);
                        const float shininess = slot_scalar(sc, s.material, 2, s.uv, &m.shininess) * (1000.0f - 1.0f) + 1.0f;
                        const float4 ind = rng.uniform4();
                        rngPos += 4;
                        if (nee) sh = direct_lambert_phong(sc, ls, T, d, s, f, f3(ind), albedo, true, specular, shininess);
                        const Scatter sc2 = indirect_phong(depth, T, limit, d, s, f, ind, albedo, specular, shininess);
                        terminated = sc2.terminated;
                        cont = sc2.c;
                        nextDir = sc2.direction;
                        nextDelta = false;
                    }
                    else if (MODEL == 4)  // GGX (:838-880)
                    {
                        const float3 base = slot_rgb(sc, s.material, 0, s.uv, m.color);
                        const float3 rma = slot_rgb(sc, s.material, 3, s.uv, m.rma);
                        const float alpha = fmaxf(rma.x * rma.x, 0.001f);
                        const float metallic = rma.y;
                        const float ior = __ldg(&m.ior);
                        const float4 ind = rng.uniform4();
                        rngPos += 4;
                        if (nee)
                        {
                            const float4 dir4 = rng.uniform4();
                            rngPos += 4;
                            sh = direct_ggx(sc, ls, T, d, s, f, f3(dir4), base, alpha, metallic, ior);
                        }
                        const Scatter sc2 = indirect_ggx(depth, T, limit, d, s, f, ind, base, alpha, metallic, ior);
                        terminated = sc2.terminated;
                        cont = sc2.c;
                        nextDir = sc2.direction;
                        nextDelta = false;
                    }
                }
                L4.w = __uint_as_float(rngPos);
                wf.slotL[slot] = L4;
                if (sh.valid)
                {
                    pushShadow = true;
                    shOut0 = make_float4(sh.origin.x, sh.origin.y, sh.origin.z, __uint_as_float(tag));
                    shOut1 = make_float4(sh.direction.x, sh.direction.y, sh.direction.z, sh.tMax);
                    shOut2 = make_float4(sh.radiance.x, sh.radiance.y, sh.radiance.z, 0.0f);
                }
                if (terminated) path_finished(wf, ctr, slot);
                else
                {
                    // SpawnScatteredRay (:148-156)
                    const float3 origin = o + d * tHit + nextGn * 1e-4f;
                    wf.slotT[slot] = make_float4(cont.throughput.x, cont.throughput.y, cont.throughput.z,
                                                 __uint_as_float(pack_meta(cont.depth, nextDelta, jobIndex)));
                    pushRay = true;
                    rayOut0 = make_float4(origin.x, origin.y, origin.z, __uint_as_float(tag));
                    rayOut1 = make_float4(nextDir.x, nextDir.y, nextDir.z, kMaxT);
                }
                (void)hitPos;
            }
            // the block's extension rays and shadow rays, each grouped by direction octant, take one
            // range of their queue each
            if (threadIdx.x < 16) octCount[threadIdx.x] = 0;
            __syncthreads();
            uint32_t oct = 0, rank = 0, soct = 0, srank = 0;
            if (pushRay)
            {
                oct = (rayOut1.x < 0.0f ? 1u : 0u) | (rayOut1.y < 0.0f ? 2u : 0u) | (rayOut1.z < 0.0f ? 4u : 0u);
                rank = atomicAdd(&octCount[oct], 1u);
            }
            if (pushShadow)
            {
                soct = 8u | (shOut1.x < 0.0f ? 1u : 0u) | (shOut1.y < 0.0f ? 2u : 0u) | (shOut1.z < 0.0f ? 4u : 0u);
                srank = atomicAdd(&octCount[soct], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0)
            {
                uint32_t total = 0, stotal = 0;
                for (int q = 0; q < 8; q++)
                {
                    octBase[q] = total;
                    total += octCount[q];
                    octBase[8 + q] = stotal;
                    stotal += octCount[8 + q];
                }
                blockBase[0] = total ? atomicAdd(&ctr->rayCount[nxt], total) : 0u;
                blockBase[1] = stotal ? atomicAdd(&ctr->shadowCount, stotal) : 0u;
            }
            __syncthreads();
            if (pushRay)
            {
                const uint32_t pos = blockBase[0] + octBase[oct] + rank;
                wf.rayO[nxt][pos] = rayOut0;
                wf.rayD[nxt][pos] = rayOut1;
            }
            if (pushShadow)
            {
                const uint32_t pos = blockBase[1] + octBase[soct] + srank;
                wf.shO[pos] = shOut0;
                wf.shD[pos] = shOut1;
                wf.shL[pos] = shOut2;
            }
            __syncthreads();
        }
        phase_end(ctr, 1);
    }

    // Finished paths write their radiance to the per-sample buffer; the first
    // min(terminated, remaining) slots start new samples behind the extension rays
    // (RegeneratePathsKernel, PathGeneration.cu:78-102).
    __global__ void regen_kernel(Wavefront wf, const JobView* jobPtr)
    {
        Counters* ctr = wf.ctr;
        phase_begin(ctr, 3);
        const uint32_t n = ctr->regenCount;
        const unsigned long long launched = ctr->launched;
        const unsigned long long total = jobPtr->totalSamples;
        const unsigned long long remaining = total - launched;
        const uint32_t regenerate = static_cast<uint32_t>(remaining < n ? remaining : n);
        const uint32_t nxt = ctr->cur ^ 1u;
        const uint32_t base = ctr->rayCount[nxt];
        float* out = jobPtr->sampleRadiance;
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        {
            const uint32_t slot = wf.regen[k];
            const float4 L = wf.slotL[slot];
            const uint32_t sample = wf.slotSample[slot];
            float* dst = out + static_cast<size_t>(sample) * 3;
            dst[0] = L.x;
            dst[1] = L.y;
            dst[2] = L.z;
            if (k < regenerate)
                start_path(*jobPtr, 0, wf, slot, static_cast<uint32_t>(launched + k), nxt, base + k);
        }
        phase_end(ctr, 3);
    }

    __global__ void advance_kernel(Wavefront wf, const JobView* jobPtr, cudaGraphConditionalHandle handle, bool graphLoop)
    {
        Counters* c = wf.ctr;
        const uint32_t cur = c->cur;
        const uint32_t nxt = cur ^ 1u;
        const unsigned long long remaining = jobPtr->totalSamples - c->launched;
        const uint32_t regenerate = static_cast<uint32_t>(remaining < c->regenCount ? remaining : c->regenCount);
        const uint32_t next = c->rayCount[nxt] + regenerate;
        if (c->iteration < wf.logCapacity)
        {
            uint32_t* row = wf.queueLog + static_cast<size_t>(c->iteration) * kQueueLogColumns;
            row[0] = c->rayCount[cur];
            for (uint32_t m = 0; m < kModelCount; m++) row[1 + m] = c->matCount[m];
            row[7] = c->shadowCount;
            row[8] = c->regenCount;
        }
        c->raysTraced += c->rayCount[cur];
        c->shadowRaysTraced += c->shadowCount;
        for (int p = 0; p < 4; p++)
        {
            if (c->tEnd[p] > c->tStart[p] && c->tStart[p] != ~0ull) c->tAccum[p] += c->tEnd[p] - c->tStart[p];
            c->tStart[p] = ~0ull;
            c->tEnd[p] = 0;
        }
        c->launched += regenerate;
        c->rayCount[cur] = 0;
        c->rayCount[nxt] = next;
        c->cur = nxt;
        for (uint32_t m = 0; m < kModelCount; m++) c->matCount[m] = 0;
        c->shadowCount = 0;
        c->regenCount = 0;
        c->traceCursor = 0;
        c->shadowCursor = 0;
        c->regenCursor = 0;
        c->iteration += 1;
        const bool cancelled = wf.cancel != nullptr && *wf.cancel != 0u;
        // Every path ends within depthLimit iterations, so the frame needs at most
        // depthLimit * (ceil(samples / pool) + 2) iterations; the cap turns a logic error
        // into an error flag instead of an endless device loop.
        const bool capped = c->iteration >= jobPtr->maxIterations;
        if (capped && next != 0) c->errorFlags |= kErrIterationCap;
        c->done = (next == 0 || cancelled || capped) ? 1u : 0u;
        if (wf.progress != nullptr)
        {
            wf.progress[0] = c->launched;
            wf.progress[1] = c->iteration;
        }
        if (graphLoop) cudaGraphSetConditional(handle, c->done ? 0u : 1u);
    }

    // PostprocessKernel's tonemap (Image.cu:22-54): x/spp, Reinhard, x^(1/2.2), u8 truncation.
    __device__ __forceinline__ uint32_t tonemap_rgba8(const float* acc, float invSpp)
    {
        uint32_t rgb[3];
        for (int ch = 0; ch < 3; ch++)
        {
            const float hdr = acc[ch] * invSpp;
            const float ldr = hdr / (hdr + 1.0f);
            const float g = pow_f(ldr, 1.0f / 2.2f);
            rgb[ch] = static_cast<uint32_t>(static_cast<unsigned char>(clampf(g * 255.0f, 0.0f, 255.0f)));
        }
        return rgb[0] | (rgb[1] << 8) | (rgb[2] << 16) | (255u << 24);
    }

    // One step of the compensated (Kahan) sum.
    __device__ __forceinline__ void kahan_add(float& sum, float& comp, float x)
    {
        const float y = x - comp;
        const float t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }

    // Per pixel: compensated (Kahan) FP32 sum of its samples in sample order, then the tonemap.
    __global__ void resolve_kernel(const JobView* jobPtr, float4* accumulation, uint32_t* framebuffer)
    {
        const JobView job = *jobPtr;
        const uint32_t pixels = job.width * job.height;
        const float invSpp = 1.0f / static_cast<float>(job.spp);
        // A pixel's samples are contiguous (sample = pixel * spp + k). With spp a multiple of 4 and a
        // whole frame, a pixel's 12 * spp bytes start 16-byte aligned and are read as float4 triples
        // (4 samples each) in sample order; every channel's Kahan sum sees the same sequence either way.
        const bool vec = (job.spp % 4u) == 0u && job.totalSamples == static_cast<uint64_t>(pixels) * job.spp;
        for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += gridDim.x * blockDim.x)
        {
            float sum[3] = {0.0f, 0.0f, 0.0f}, comp[3] = {0.0f, 0.0f, 0.0f};
            const uint64_t first = static_cast<uint64_t>(p) * job.spp;
            if (vec)
            {
                const float4* src = reinterpret_cast<const float4*>(job.sampleRadiance + first * 3);
                for (uint32_t q = 0; q < job.spp / 4u; q++)
                {
                    const float4 a = __ldg(src + 3u * q), b = __ldg(src + 3u * q + 1u), c = __ldg(src + 3u * q + 2u);
                    kahan_add(sum[0], comp[0], a.x);
                    kahan_add(sum[1], comp[1], a.y);
                    kahan_add(sum[2], comp[2], a.z);
                    kahan_add(sum[0], comp[0], a.w);
                    kahan_add(sum[1], comp[1], b.x);
                    kahan_add(sum[2], comp[2], b.y);
                    kahan_add(sum[0], comp[0], b.z);
                    kahan_add(sum[1], comp[1], b.w);
                    kahan_add(sum[2], comp[2], c.x);
                    kahan_add(sum[0], comp[0], c.y);
                    kahan_add(sum[1], comp[1], c.z);
                    kahan_add(sum[2], comp[2], c.w);
                }
            }
            else
            {
                for (uint32_t k = 0; k < job.spp; k++)
                {
                    const uint64_t si = first + k;
                    if (si >= job.totalSamples) break;
                    for (int ch = 0; ch < 3; ch++) kahan_add(sum[ch], comp[ch], job.sampleRadiance[si * 3 + ch]);
                }
            }
            accumulation[p] = make_float4(sum[0], sum[1], sum[2], 0.0f);
            framebuffer[p] = tonemap_rgba8(sum, invSpp);
        }
    }

    // ------------------------------------------------------------------ job engine
    // Jobs share one pool of path slots. A job hands out launch indices g in pass-major order:
    // pass g / pixels (= the stratum), pixel g % pixels, sample pixel * spp + pass. The sample,
    // and with it the Philox stream and the path, is the one the frame renderer traces, so the
    // per-sample radiance is identical. Finished samples land in a ring of `ring` pass buffers;
    // complete passes are folded in order into a per-pixel Kahan accumulator, which therefore
    // adds every pixel's samples in the same order as resolve_kernel: the image of a job is the
    // same alone, mixed with other jobs, and rendered by the frame renderer.

    __device__ __forceinline__ uint64_t job_passes(const JobView& J)
    {
        return (J.totalSamples + J.pixels - 1) / J.pixels;
    }

    // Number of consecutive complete passes starting at the first unfolded one (at most `ring`).
    __device__ __forceinline__ uint32_t foldable_passes(const JobView& J)
    {
        const uint64_t passes = job_passes(J);
        uint32_t c = 0;
        while (c < J.ring && J.folded + c < passes)
        {
            const uint64_t p = J.folded + c;
            const uint64_t rem = J.totalSamples - p * J.pixels;
            const uint32_t size = rem < J.pixels ? static_cast<uint32_t>(rem) : J.pixels;
            if (J.passDone[p % J.ring] != size) break;
            c++;
        }
        return c;
    }

    __device__ __forceinline__ uint64_t job_window_end(const JobView& J)
    {
        const uint64_t window = static_cast<uint64_t>(J.folded + J.ring) * J.pixels;
        return window < J.totalSamples ? window : J.totalSamples;
    }

    __global__ void engine_init_kernel(Wavefront wf, EngineView ev, uint32_t pool)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pool; i += gridDim.x * blockDim.x) ev.freeList[i] = pool - 1u - i;
        if (blockIdx.x != 0 || threadIdx.x != 0) return;
        Counters* c = wf.ctr;
        *c = Counters{};
        for (int p = 0; p < 4; p++) c->tStart[p] = ~0ull;
        EngineCtl* e = ev.ctl;
        e->freeCount = pool;
        e->launchCount = 0;
        e->segmentCount = 0;
        e->stalled = 0;
    }

    // One thread: hands the iteration's idle slots (finished paths + free list) to the active
    // jobs, oldest first, within each job's ring window.
    __global__ void plan_kernel(Wavefront wf, EngineView ev)
    {
        EngineCtl* e = ev.ctl;
        const uint32_t avail = wf.ctr->regenCount + e->freeCount;
        uint32_t launch = 0, segments = 0;
        // a job marked kOrderInTurn gets slots only once every marked job before it has launched all
        // its samples (its turn has come), even if an earlier one's pass window holds it back for now
        bool waitTurn = false;
        for (uint32_t i = 0; i < e->orderCount && launch < avail; i++)
        {
            const uint32_t o = ev.order[i];
            const uint32_t j = o & ~kOrderInTurn;
            JobView& J = ev.jobs[j];
            if (J.state != kJobActive) continue;
            const bool inTurn = (o & kOrderInTurn) != 0;
            if (inTurn && waitTurn) continue;
            const uint64_t end = job_window_end(J);
            if (end > J.launched)
            {
                const uint64_t can = end - J.launched;
                const uint32_t take = static_cast<uint32_t>(can < static_cast<uint64_t>(avail - launch) ? can : avail - launch);
                ev.segments[segments] = LaunchSegment{j, launch, J.launched};
                segments++;
                J.launched += take;
                launch += take;
            }
            if (inTurn && J.launched < J.totalSamples) waitTurn = true;
        }
        e->launchCount = launch;
        e->segmentCount = segments;
    }

    // Finished samples per (job, ring buffer) are counted per block in shared memory first: every path
    // of a job's pass increments the same counter, and a global atomic per warp and key piles up on a
    // few addresses (worst with one job). A block flushes its table once, at the end of the kernel.
    constexpr uint32_t kPassTable = 256;

    __device__ __forceinline__ void count_finished(uint32_t* tableKey, uint32_t* tableCount, uint32_t* globalCounter, uint32_t key)
    {
        const unsigned active = __activemask();
        const unsigned peers = __match_any_sync(active, key);
        if (static_cast<int>(lane_id()) != __ffs(peers) - 1) return;
        const uint32_t n = static_cast<uint32_t>(__popc(peers));
        const uint32_t h = (key * 2654435761u) >> 24;
        for (uint32_t probe = 0; probe < 8; probe++)
        {
            const uint32_t s = (h + probe) & (kPassTable - 1u);
            const uint32_t prev = atomicCAS(&tableKey[s], kInvalid, key);
            if (prev == kInvalid || prev == key)
            {
                atomicAdd(&tableCount[s], n);
                return;
            }
        }
        atomicAdd(globalCounter, n);  // table crowded: count directly
    }

    // A finished path writes its radiance into its job's pass ring and counts towards the pass.
    // meta: the slot's path metadata (job in bits 16-31), sample and L: its sample index and radiance.
    __device__ __forceinline__ void engine_retire_path(const EngineView& ev, uint32_t meta, uint32_t sample, float4 L, uint32_t* tableKey,
                                                       uint32_t* tableCount)
    {
        const uint32_t j = meta >> 16;
        JobView& J = ev.jobs[j];
        const uint32_t pixel = sample / J.spp;
        const uint32_t pass = sample - pixel * J.spp;
        const uint32_t r = pass % J.ring;
        float* dst = J.sampleRadiance + (static_cast<size_t>(r) * J.pixels + pixel) * 3;
        dst[0] = L.x;
        dst[1] = L.y;
        dst[2] = L.z;
        count_finished(tableKey, tableCount, &J.passDone[r], (j << 8) | r);
    }

    // Planned launch k of the iteration starts in `slot` (the plan's segments map k to a job and launch index).
    // segments: the plan's segments (a shared-memory copy when they fit, else ev.segments).
    __device__ __forceinline__ void engine_start_launch(const Wavefront& wf, const EngineView& ev, const LaunchSegment* segments, uint32_t k,
                                                        uint32_t slot, uint32_t segmentCount, uint32_t nxt, uint32_t base)
    {
        uint32_t lo = 0, hi = segmentCount - 1u;
        while (lo < hi)
        {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (segments[mid].start <= k) lo = mid;
            else hi = mid - 1u;
        }
        const LaunchSegment sg = segments[lo];
        const JobView& J = ev.jobs[sg.job];
        const uint64_t g = sg.first + (k - sg.start);
        const uint32_t pass = static_cast<uint32_t>(g / J.pixels);
        const uint32_t pixel = static_cast<uint32_t>(g - static_cast<uint64_t>(pass) * J.pixels);
        start_path(J, sg.job, wf, slot, pixel * J.spp + pass, nxt, base + k);
    }

    // Job-engine regeneration from the finished-slot bitmap (same tiling as regen_bits_kernel): the
    // finished slot of rank k takes planned launch k, or goes onto the free list when k >= the plan;
    // launches beyond the finished slots take slots from the free list.
    constexpr uint32_t kSharedSegments = 512;  // plan segments held in shared memory by the engine's regeneration

    __global__ void engine_regen_bits_kernel(Wavefront wf, EngineView ev)
    {
        Counters* ctr = wf.ctr;
        phase_begin(ctr, 3);
        const uint32_t n = ctr->regenCount;
        const EngineCtl* e = ev.ctl;
        const uint32_t launch = e->launchCount;
        const uint32_t freeCount = e->freeCount;
        const uint32_t segmentCount = e->segmentCount;
        const uint32_t nxt = ctr->cur ^ 1u;
        const uint32_t base = ctr->rayCount[nxt];
        const uint32_t words = (wf.capacity + 31u) >> 5;
        const uint32_t tiles = (words + 31u) >> 5;
        const uint32_t lane = lane_id();
        const uint32_t lanesBelow = (1u << lane) - 1u;
        const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
        // the plan's segments, searched once per launch, from shared memory when they fit
        __shared__ LaunchSegment localSegments[kSharedSegments];
        __shared__ uint32_t passKey[kPassTable], passCount[kPassTable];
        const bool shared = segmentCount <= kSharedSegments;
        if (shared)
            for (uint32_t i = threadIdx.x; i < segmentCount; i += blockDim.x) localSegments[i] = ev.segments[i];
        for (uint32_t i = threadIdx.x; i < kPassTable; i += blockDim.x)
        {
            passKey[i] = kInvalid;
            passCount[i] = 0;
        }
        __syncthreads();
        const LaunchSegment* segments = shared ? localSegments : ev.segments;
        for (uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < tiles; tile += warps)
        {
            const uint32_t wi = tile * 32u + lane;
            const uint32_t bits = wi < words ? wf.regenBits[wi] : 0u;
            if (bits) wf.regenBits[wi] = 0u;
            const uint32_t count = static_cast<uint32_t>(__popc(bits));
            uint32_t incl = count;
            for (int o = 1; o < 32; o <<= 1)
            {
                const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (static_cast<int>(lane) >= o) incl += v;
            }
            const uint32_t tileTotal = __shfl_sync(0xFFFFFFFFu, incl, 31);
            if (tileTotal == 0) continue;
            uint32_t first = 0;
            if (lane == 0) first = atomicAdd(&ctr->regenCursor, tileTotal);
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            const uint32_t excl = incl - count;
            // words in groups of kRegenGroup: the finished slots' loads of a group are in flight together
            for (uint32_t jb = 0; jb < 32; jb += kRegenGroup)
            {
                uint32_t w[kRegenGroup], offset[kRegenGroup], meta[kRegenGroup], sample[kRegenGroup];
                float4 L[kRegenGroup];
#pragma unroll
                for (uint32_t q = 0; q < kRegenGroup; q++)
                {
                    w[q] = __shfl_sync(0xFFFFFFFFu, bits, jb + q);
                    offset[q] = __shfl_sync(0xFFFFFFFFu, excl, jb + q);
                    L[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    meta[q] = 0;
                    sample[q] = 0;
                    if ((w[q] >> lane) & 1u)
                    {
                        const uint32_t slot = (tile * 32u + jb + q) * 32u + lane;
                        meta[q] = __float_as_uint(wf.slotT[slot].w);
                        sample[q] = wf.slotSample[slot];
                        L[q] = wf.slotL[slot];
                    }
                }
#pragma unroll
                for (uint32_t q = 0; q < kRegenGroup; q++)
                {
                    if (!((w[q] >> lane) & 1u)) continue;
                    const uint32_t slot = (tile * 32u + jb + q) * 32u + lane;
                    engine_retire_path(ev, meta[q], sample[q], L[q], passKey, passCount);
                    const uint32_t k = first + offset[q] + static_cast<uint32_t>(__popc(w[q] & lanesBelow));
                    if (k < launch) engine_start_launch(wf, ev, segments, k, slot, segmentCount, nxt, base);
                    else ev.freeList[freeCount + (k - launch)] = slot;
                }
            }
        }
        for (uint32_t k = n + blockIdx.x * blockDim.x + threadIdx.x; k < launch; k += gridDim.x * blockDim.x)
            engine_start_launch(wf, ev, segments, k, ev.freeList[freeCount - 1u - (k - n)], segmentCount, nxt, base);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kPassTable; i += blockDim.x)
        {
            const uint32_t key = passKey[i];
            if (key != kInvalid) atomicAdd(&ev.jobs[key >> 8].passDone[key & 0xFFu], passCount[i]);
        }
        phase_end(ctr, 3);
    }

    // Folds every job's complete passes, in pass order, into its Kahan accumulator; the job's
    // last fold also writes its tone-mapped RGBA8 image.
    __global__ void fold_kernel(EngineView ev)
    {
        // jobs in blocks of blockDim.x: their foldable pass counts are found side by side first
        __shared__ uint32_t jobOf[256], countOf[256];
        const uint32_t orderCount = ev.ctl->orderCount;
        for (uint32_t base = 0; base < orderCount; base += blockDim.x)
        {
            const uint32_t i = base + threadIdx.x;
            uint32_t count = 0, j = 0;
            if (i < orderCount)
            {
                j = ev.order[i] & ~kOrderInTurn;
                const JobView& J = ev.jobs[j];
                if (J.state == kJobActive) count = foldable_passes(J);
            }
            jobOf[threadIdx.x] = j;
            countOf[threadIdx.x] = count;
            __syncthreads();
            const uint32_t chunk = orderCount - base < blockDim.x ? orderCount - base : blockDim.x;
            for (uint32_t t = 0; t < chunk; t++)
            {
                const uint32_t count_t = countOf[t];
                if (count_t == 0) continue;
                const JobView& J = ev.jobs[jobOf[t]];
                const bool last = J.folded + count_t == job_passes(J);
                const float invSpp = 1.0f / static_cast<float>(J.spp);
                for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < J.pixels; px += gridDim.x * blockDim.x)
                {
                    const float4 s4 = J.accum[2 * static_cast<size_t>(px)];
                    const float4 c4 = J.accum[2 * static_cast<size_t>(px) + 1];
                    float sum[3] = {s4.x, s4.y, s4.z}, comp[3] = {c4.x, c4.y, c4.z};
                    for (uint32_t q = 0; q < count_t; q++)
                    {
                        const uint64_t p = static_cast<uint64_t>(J.folded) + q;
                        if (p * J.pixels + px >= J.totalSamples) break;
                        const float* x = J.sampleRadiance + (static_cast<size_t>(p % J.ring) * J.pixels + px) * 3;
                        for (int ch = 0; ch < 3; ch++) kahan_add(sum[ch], comp[ch], x[ch]);
                    }
                    J.accum[2 * static_cast<size_t>(px)] = make_float4(sum[0], sum[1], sum[2], 0.0f);
                    J.accum[2 * static_cast<size_t>(px) + 1] = make_float4(comp[0], comp[1], comp[2], 0.0f);
                    if (last) J.framebuffer[px] = tonemap_rgba8(sum, invSpp);
                }
            }
            __syncthreads();
        }
    }

    // One block: fold accounting and job completion, one thread per job, then (thread 0) queue
    // bookkeeping and the slice's loop condition. The slice ends when a job completes (so the host can
    // hand out its result and admit waiting jobs), when the host rings the doorbell (a job arrived),
    // when there is nothing left to do, or after maxSliceIterations iterations.
    __global__ void engine_advance_kernel(Wavefront wf, EngineView ev, cudaGraphConditionalHandle handle, bool graphLoop)
    {
        __shared__ uint32_t completedJobs, unfinishedJobs, launchableJobs;
        if (threadIdx.x == 0)
        {
            completedJobs = 0;
            unfinishedJobs = 0;
            launchableJobs = 0;
        }
        __syncthreads();
        {
            const uint32_t orderCount = ev.ctl->orderCount;
            for (uint32_t i = threadIdx.x; i < orderCount; i += blockDim.x)
            {
                JobView& J = ev.jobs[ev.order[i] & ~kOrderInTurn];
                if (J.state != kJobActive) continue;
                const uint32_t count = foldable_passes(J);
                for (uint32_t q = 0; q < count; q++) J.passDone[(static_cast<uint64_t>(J.folded) + q) % J.ring] = 0;
                J.folded += count;
                if (J.folded == job_passes(J))
                {
                    J.state = kJobDone;
                    atomicAdd(&completedJobs, 1u);
                    continue;
                }
                atomicOr(&unfinishedJobs, 1u);
                if (job_window_end(J) > J.launched) atomicOr(&launchableJobs, 1u);
            }
        }
        __syncthreads();
        if (threadIdx.x != 0) return;
        Counters* c = wf.ctr;
        EngineCtl* e = ev.ctl;
        const uint32_t cur = c->cur;
        const uint32_t nxt = cur ^ 1u;
        const uint32_t launch = e->launchCount;
        const uint32_t next = c->rayCount[nxt] + launch;
        c->raysTraced += c->rayCount[cur];
        c->shadowRaysTraced += c->shadowCount;
        for (int p = 0; p < 4; p++)
        {
            if (c->tEnd[p] > c->tStart[p] && c->tStart[p] != ~0ull) c->tAccum[p] += c->tEnd[p] - c->tStart[p];
            c->tStart[p] = ~0ull;
            c->tEnd[p] = 0;
        }
        e->freeCount = e->freeCount + c->regenCount - launch;
        c->launched += launch;
        c->rayCount[cur] = 0;
        c->rayCount[nxt] = next;
        c->cur = nxt;
        for (uint32_t m = 0; m < kModelCount; m++) c->matCount[m] = 0;
        c->shadowCount = 0;
        c->regenCount = 0;
        c->traceCursor = 0;
        c->shadowCursor = 0;
        c->regenCursor = 0;
        c->iteration += 1;
        e->launchCount = 0;
        e->segmentCount = 0;
        const uint32_t completed = completedJobs;
        const bool launchable = launchableJobs != 0, unfinished = unfinishedJobs != 0;
        e->completed += completed;
        e->sliceIterations += 1;
        const bool idle = next == 0 && !launchable;
        if (idle && unfinished) e->stalled = 1;
        const bool bell = ev.doorbell != nullptr && *ev.doorbell != 0u;
        c->done = (completed > 0 || bell || idle || e->sliceIterations >= e->maxSliceIterations) ? 1u : 0u;
        if (wf.progress != nullptr)
        {
            wf.progress[0] = c->launched;
            wf.progress[1] = c->iteration;
        }
        if (graphLoop) cudaGraphSetConditional(handle, c->done ? 0u : 1u);
    }

    // Packing resident scenes into one set of arrays: add `offset` to one 32-bit field of every
    // record (base points at the field of record 0, records are strideWords apart). Entries equal
    // to kInvalid stay invalid when skipInvalid is set (alias entries without an alias).
    __global__ void rebase_field_kernel(uint32_t* base, uint32_t n, uint32_t strideWords, uint32_t offset, bool skipInvalid)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        {
            uint32_t* f = base + static_cast<size_t>(i) * strideWords;
            if (skipInvalid && *f == kInvalid) continue;
            *f += offset;
        }
    }

    // Child references of BVH8 nodes: inner children by nodeOffset, leaf ranges by triOffset.
    __global__ void rebase_nodes_kernel(Node8* nodes, uint32_t n, uint32_t nodeOffset, uint32_t triOffset)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        {
            Node8& nd = nodes[i];
            const uint32_t inner = nd.w[0].w >> 24;
            const uint32_t leaf = nd.w[6].z & 0xFFu;
            uint32_t* refs = reinterpret_cast<uint32_t*>(&nd.w[4]);
            for (int k = 0; k < 8; k++)
            {
                if ((inner >> k) & 1u) refs[k] += nodeOffset;
                else if ((leaf >> k) & 1u) refs[k] += triOffset;
            }
        }
    }

    // The FP64 reference accumulation of a frame: per pixel, the sum of its per-sample radiance in FP64,
    // in sample order (the same order the FP32 Kahan resolve uses), for measuring the FP32 accumulation
    // error on the device. sums: [pixels][3].
    __global__ void resolve_fp64_kernel(const JobView* jobPtr, double* sums)
    {
        const JobView job = *jobPtr;
        const uint32_t pixels = job.width * job.height;
        for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += gridDim.x * blockDim.x)
        {
            double acc[3] = {0.0, 0.0, 0.0};
            const uint64_t first = static_cast<uint64_t>(p) * job.spp;
            for (uint32_t k = 0; k < job.spp; k++)
            {
                const uint64_t si = first + k;
                if (si >= job.totalSamples) break;
                for (int ch = 0; ch < 3; ch++) acc[ch] += static_cast<double>(job.sampleRadiance[si * 3 + ch]);
            }
            for (int ch = 0; ch < 3; ch++) sums[static_cast<size_t>(p) * 3 + ch] = acc[ch];
        }
    }

    __global__ void clear_kernel(uint32_t* framebuffer, uint32_t n, uint32_t value)  // ClearKernel (Image.cu:7-13)
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) framebuffer[i] = value;
    }

    // ------------------------------------------------------------------ host launchers
    namespace
    {
        constexpr size_t kColdBytes = 2 * sizeof(float4);  // shared-memory cold slot per traversal thread

        // Traversal kernel variants: stack capacity (>= BVH8 depth) x occupancy target. MINB is the
        // minimum resident 128-thread blocks per SM the compiler must allow (1 = registers unconstrained,
        // 10 = <= 48 registers, 12 = <= 40 registers); the best one is measured, not assumed.
        template <int STACK, bool ANY, int MINB, class Work>
        cudaError_t launch_trace_t(const Work& w, int blocks, int threads, uint32_t refill, uint32_t* err, cudaStream_t s)
        {
            const size_t smem = static_cast<size_t>(STACK) * threads * sizeof(uint32_t) + kColdBytes * threads;
            trace_kernel<STACK, ANY, MINB, false, Work><<<blocks, threads, smem, s>>>(w, refill, err);
            return cudaGetLastError();
        }

        // Binary FP32 BVH (local-memory stack of kMaxStack entries, no shared memory).
        template <bool ANY, class Work>
        cudaError_t launch_trace_binary(const Work& w, int blocks, int threads, uint32_t refill, uint32_t* err, cudaStream_t s)
        {
            trace_kernel<kMaxStack, ANY, 1, true, Work><<<blocks, threads, kColdBytes * threads, s>>>(w, refill, err);
            return cudaGetLastError();
        }

        template <int STACK, bool ANY, class Work>
        cudaError_t launch_trace_m(const Work& w, int occupancy, int blocks, int threads, uint32_t refill, uint32_t* err, cudaStream_t s)
        {
            if (occupancy >= 12) return launch_trace_t<STACK, ANY, 12>(w, blocks, threads, refill, err, s);
            if (occupancy >= 10) return launch_trace_t<STACK, ANY, 10>(w, blocks, threads, refill, err, s);
            return launch_trace_t<STACK, ANY, 1>(w, blocks, threads, refill, err, s);
        }

        template <bool ANY, class Work>
        cudaError_t launch_trace(const Work& w, uint32_t depth, int occupancy, int blocks, int threads, uint32_t refill, uint32_t* err,
                                 cudaStream_t s)
        {
            if (depth <= 8) return launch_trace_m<8, ANY>(w, occupancy, blocks, threads, refill, err, s);
            if (depth <= 16) return launch_trace_m<16, ANY>(w, occupancy, blocks, threads, refill, err, s);
            if (depth <= 32) return launch_trace_m<32, ANY>(w, occupancy, blocks, threads, refill, err, s);
            return launch_trace_m<64, ANY>(w, occupancy, blocks, threads, refill, err, s);
        }

        template <int STACK, int MINB>
        int resident_blocks(int threads)
        {
            int perSm = 0;
            const size_t smem = static_cast<size_t>(STACK) * threads * sizeof(uint32_t) + kColdBytes * threads;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, trace_kernel<STACK, false, MINB, false, WavefrontClosest>, threads, smem);
            return perSm;
        }

        template <int STACK>
        int resident_blocks_m(int occupancy, int threads)
        {
            if (occupancy >= 12) return resident_blocks<STACK, 12>(threads);
            if (occupancy >= 10) return resident_blocks<STACK, 10>(threads);
            return resident_blocks<STACK, 1>(threads);
        }
    }

    int trace_grid_blocks(int device, int threads, uint32_t depth, int occupancy, uint32_t bvhFormat)
    {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        int perSm;
        if (bvhFormat == kBvh2Fp32)
        {
            perSm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, trace_kernel<kMaxStack, false, 1, true, WavefrontClosest>, threads,
                                                          kColdBytes * threads);
            return sms * (perSm < 1 ? 1 : perSm);
        }
        if (depth <= 8) perSm = resident_blocks_m<8>(occupancy, threads);
        else if (depth <= 16) perSm = resident_blocks_m<16>(occupancy, threads);
        else if (depth <= 32) perSm = resident_blocks_m<32>(occupancy, threads);
        else perSm = resident_blocks_m<64>(occupancy, threads);
        if (perSm < 1) perSm = 1;
        return sms * perSm;
    }

    // Resident 128-thread blocks per SM of shade_kernel<M> (its registers decide: 32 to 96 per thread),
    // at most 8. The shading loop strides over its queue by the grid, so a grid larger than what is
    // resident at once leaves the blocks that start late with a full share of the work.
    template <uint32_t M>
    static int shade_blocks_per_sm()
    {
        static const int perSm = []
        {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, shade_kernel<M>, 128, 0) != cudaSuccess) b = 8;
            return b < 1 ? 1 : (b > 8 ? 8 : b);
        }();
        return perSm;
    }

    // Resident 256-thread blocks per SM of a regeneration kernel, at most 8 (its tiles are handed out
    // by a grid stride, so a grid larger than what is resident leaves late blocks a full share).
    template <class K>
    static int resident_blocks_256(K kernel)
    {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 256, 0) != cudaSuccess) b = 8;
        return b < 1 ? 1 : (b > 8 ? 8 : b);
    }
    static int regen_blocks_per_sm()
    {
        static const int perSm = resident_blocks_256(regen_bits_kernel);
        return perSm;
    }
    static int engine_regen_blocks_per_sm()
    {
        static const int perSm = resident_blocks_256(engine_regen_bits_kernel);
        return perSm;
    }

    static cudaError_t launch_shade(uint32_t m, int sms, const SceneView& sc, const Wavefront& wf, const JobView* jobs,
                                    const SceneEntry* scenes, cudaStream_t s)
    {
        switch (m)
        {
            case 0: shade_kernel<0><<<sms * shade_blocks_per_sm<0>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
            case 1: shade_kernel<1><<<sms * shade_blocks_per_sm<1>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
            case 2: shade_kernel<2><<<sms * shade_blocks_per_sm<2>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
            case 3: shade_kernel<3><<<sms * shade_blocks_per_sm<3>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
            case 4: shade_kernel<4><<<sms * shade_blocks_per_sm<4>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
            default: shade_kernel<5><<<sms * shade_blocks_per_sm<5>(), 128, 0, s>>>(sc, wf, jobs, scenes); break;
        }
        return cudaGetLastError();
    }

    // The shading kernels of the models present: with a fork event they run on their own streams side
    // by side (parallel branches when captured into a graph; they touch disjoint queue entries and push
    // with atomics) and join the launching stream again; without one, in order on it.
    static cudaError_t launch_shading(const bool* modelPresent, cudaEvent_t fork, const cudaEvent_t* join, const cudaStream_t* streams,
                                      int sms, const SceneView& sc, const Wavefront& wf, const JobView* jobs, const SceneEntry* scenes,
                                      cudaStream_t s)
    {
        cudaError_t e;
        uint32_t models = 0;
        for (uint32_t m = 0; m < kModelCount; m++) models += modelPresent[m] ? 1u : 0u;
        if (fork && models > 1)
        {
            if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
            for (uint32_t m = 0; m < kModelCount; m++)
            {
                if (!modelPresent[m]) continue;
                if ((e = cudaStreamWaitEvent(streams[m], fork, 0)) != cudaSuccess) return e;
                if ((e = launch_shade(m, sms, sc, wf, jobs, scenes, streams[m])) != cudaSuccess) return e;
                if ((e = cudaEventRecord(join[m], streams[m])) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(s, join[m], 0)) != cudaSuccess) return e;
            }
            return cudaSuccess;
        }
        for (uint32_t m = 0; m < kModelCount; m++)
        {
            if (!modelPresent[m]) continue;
            if ((e = launch_shade(m, sms, sc, wf, jobs, scenes, s)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    cudaError_t launch_iteration(const IterationLaunch& L, cudaStream_t s)
    {
        cudaError_t e;
        WavefrontClosest wc{L.scene, L.wf, nullptr, L.stackCap};
        const bool binary = L.bvhFormat == kBvh2Fp32;
        if (L.traceStart && (e = cudaEventRecord(L.traceStart, s)) != cudaSuccess) return e;
        if (binary)
            e = launch_trace_binary<false>(wc, L.traceBlocks, L.traceThreads, L.refill, &L.wf.ctr->errorFlags, s);
        else
            e = launch_trace<false>(wc, L.scene.depth, L.occupancy, L.traceBlocks, L.traceThreads, L.refill, &L.wf.ctr->errorFlags, s);
        if (e != cudaSuccess) return e;
        if (L.traceStop && (e = cudaEventRecord(L.traceStop, s)) != cudaSuccess) return e;
        if ((e = launch_shading(L.modelPresent, L.shadeFork, L.shadeJoin, L.shadeStreams, L.sms, L.scene, L.wf, L.job, L.scenes, s)) != cudaSuccess)
            return e;
        if (L.nee && L.scene.lightCount > 0)
        {
            WavefrontShadow ws{L.scene, L.wf, nullptr, L.stackCap};
            if (binary)
                e = launch_trace_binary<true>(ws, L.traceBlocks, L.traceThreads, L.refillShadow, &L.wf.ctr->errorFlags, s);
            else
                e = launch_trace<true>(ws, L.scene.depth, L.occupancy, L.traceBlocks, L.traceThreads, L.refillShadow, &L.wf.ctr->errorFlags, s);
            if (e != cudaSuccess) return e;
        }
        if (L.wf.regenBits != nullptr)
            regen_bits_kernel<<<L.sms * regen_blocks_per_sm(), 256, 0, s>>>(L.wf, L.job);
        else
            regen_kernel<<<L.shadeBlocks, 256, 0, s>>>(L.wf, L.job);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        advance_kernel<<<1, 1, 0, s>>>(L.wf, L.job, L.handle, L.graphLoop);
        return cudaGetLastError();
    }

    cudaError_t launch_engine_init(const Wavefront& wf, const EngineView& ev, uint32_t pool, cudaStream_t s)
    {
        const uint32_t blocks = (pool + 255) / 256 < 4096 ? (pool + 255) / 256 : 4096;
        engine_init_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(wf, ev, pool);
        return cudaGetLastError();
    }

    cudaError_t launch_engine_iteration(const EngineLaunch& L, cudaStream_t s)
    {
        cudaError_t e;
        WavefrontClosest wc{L.scene, L.wf, L.ev.scenes};
        e = launch_trace<false>(wc, L.scene.depth, L.occupancy, L.traceBlocks, L.traceThreads, L.refill, &L.wf.ctr->errorFlags, s);
        if (e != cudaSuccess) return e;
        if ((e = launch_shading(L.modelPresent, L.shadeFork, L.shadeJoin, L.shadeStreams, L.sms, L.scene, L.wf, L.ev.jobs, L.ev.scenes, s)) !=
            cudaSuccess)
            return e;
        if (L.anyLights)
        {
            WavefrontShadow ws{L.scene, L.wf, L.ev.scenes};
            e = launch_trace<true>(ws, L.scene.depth, L.occupancy, L.traceBlocks, L.traceThreads, L.refillShadow, &L.wf.ctr->errorFlags, s);
            if (e != cudaSuccess) return e;
        }
        plan_kernel<<<1, 1, 0, s>>>(L.wf, L.ev);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        engine_regen_bits_kernel<<<L.sms * engine_regen_blocks_per_sm(), 256, 0, s>>>(L.wf, L.ev);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        fold_kernel<<<L.shadeBlocks, 256, 0, s>>>(L.ev);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        engine_advance_kernel<<<1, 256, 0, s>>>(L.wf, L.ev, L.handle, L.graphLoop);
        return cudaGetLastError();
    }

    cudaError_t launch_rebase_field(uint32_t* base, uint32_t n, uint32_t strideWords, uint32_t offset, bool skipInvalid, cudaStream_t s)
    {
        if (n == 0 || (offset == 0 && !skipInvalid)) return cudaSuccess;
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        rebase_field_kernel<<<blocks, 256, 0, s>>>(base, n, strideWords, offset, skipInvalid);
        return cudaGetLastError();
    }

    cudaError_t launch_rebase_nodes(Node8* nodes, uint32_t n, uint32_t nodeOffset, uint32_t triOffset, cudaStream_t s)
    {
        if (n == 0) return cudaSuccess;
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        rebase_nodes_kernel<<<blocks, 256, 0, s>>>(nodes, n, nodeOffset, triOffset);
        return cudaGetLastError();
    }

    cudaError_t launch_frame_prologue(const Wavefront& wf, const JobView* job, uint32_t pool, int blocks, cudaStream_t s)
    {
        frame_init_kernel<<<1, 1, 0, s>>>(wf, job, pool);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        generate_kernel<<<blocks, 256, 0, s>>>(wf, job);
        return cudaGetLastError();
    }

    cudaError_t launch_resolve(const JobView* job, float4* accumulation, uint32_t* framebuffer, int blocks, cudaStream_t s)
    {
        resolve_kernel<<<blocks, 128, 0, s>>>(job, accumulation, framebuffer);
        return cudaGetLastError();
    }

    cudaError_t launch_resolve_fp64(const JobView* job, double* sums, int blocks, cudaStream_t s)
    {
        resolve_fp64_kernel<<<blocks, 128, 0, s>>>(job, sums);
        return cudaGetLastError();
    }

    cudaError_t launch_clear(uint32_t* framebuffer, uint32_t n, uint32_t value, cudaStream_t s)
    {
        if (n == 0) return cudaSuccess;
        clear_kernel<<<(n + 511) / 512 < 4096 ? (n + 511) / 512 : 4096, 512, 0, s>>>(framebuffer, n, value);
        return cudaGetLastError();
    }

    cudaError_t launch_batch_trace(const SceneView& sc, uint32_t root, const float* rays, uint32_t n, uint32_t* cursor, uint32_t* triOut,
                                   float* uvtOut, uint8_t* occOut, int blocks, int threads, uint32_t* errorFlags, cudaStream_t s,
                                   uint32_t bvhFormat)
    {
        BatchRays b{sc, rays, n, cursor, triOut, uvtOut, occOut, root};
        if (bvhFormat == kBvh2Fp32)
        {
            if (occOut) return launch_trace_binary<true>(b, blocks, threads, 32, errorFlags, s);
            return launch_trace_binary<false>(b, blocks, threads, 32, errorFlags, s);
        }
        if (occOut) return launch_trace<true>(b, sc.depth, 1, blocks, threads, 32, errorFlags, s);
        return launch_trace<false>(b, sc.depth, 1, blocks, threads, 32, errorFlags, s);
    }
}

