// Device construction of the BVH8 (gpt_set_bvh_build(GPT_BVH_BUILD_DEVICE)). It writes the node
// format, single-triangle leaves and triangle records of the host builder (bvh8.cpp) and uses its
// surface-area-optimal 8-wide collapse, slot assignment and quantisation; the binary tree the wide
// tree is collapsed from is built on the GPU by clustering instead of the host's binned SAH:
//
// 1. Triangle boxes and centroids, and the centroids' bounds (two-pass reduction).
// 2. 30-bit Morton codes of the centroids; triangles sorted by code (cub::DeviceRadixSort).
// 3. PLOC (Meister and Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
//    Construction", IEEE TVCG 2018): the clusters stay in Morton order; each finds the cluster within
//    kPlocRadius positions whose merged box has the smallest surface area (the nearer position wins a
//    tie), mutual nearest neighbours merge, and the survivors are compacted in order by prefix sums,
//    until one cluster is left. The nodes of one round get consecutive indices after those of the
//    rounds before, so every node has a larger index than its children.
// 4. The collapse's cost table (Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on
//    GPUs Through Compressed Wide BVHs", HPG 2017), bottom-up one round of nodes at a time.
// 5. Wide nodes level by level from the root: each collects its children from the cost table,
//    assigns them to slots by octant, quantises their boxes in double precision with outward
//    rounding and reserves consecutive indices for its inner children with one atomic.
// 6. Triangle records in Morton order (leaf position k holds the k-th triangle of the sort).
//
// Hits do not depend on the tree (the traversal is conservative and ties go to the smaller input
// index), so frames equal those of a host-built BVH bit for bit; only the traversal work differs.
#include <cfloat>
#include <cstdint>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "bvh_device.hpp"

namespace pt
{
    namespace
    {
        constexpr int kPlocRadius = 16;
        constexpr int kPlocBlock = 256;
        constexpr float kCollapseNodeCost = 2.0f;  // a wide-node visit against one triangle test (bvh8.cpp)
        constexpr int kCollectStack = 24;
        constexpr uint32_t kBuildErrExponent = 1u;  // quantisation exponent overflow
        constexpr uint32_t kBuildErrCollect = 2u;   // a node's child list did not fit its slots
        constexpr uint32_t kBuildErrCapacity = 4u;  // a wide-node index beyond the node array

        __device__ __forceinline__ float box_area(float4 lo, float4 hi)
        {
            const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
            if (dx < 0.0f || dy < 0.0f || dz < 0.0f) return 0.0f;
            return 2.0f * (dx * dy + dy * dz + dz * dx);
        }

        __device__ __forceinline__ float4 fmin4(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.0f); }
        __device__ __forceinline__ float4 fmax4(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), 0.0f); }

        // Triangle boxes (leaf k of the sort is written later, by permutation) and centroids; per-block
        // bounds of the centroids.
        __global__ void triangle_boxes_kernel(const float* pos, uint32_t n, float4* triLo, float4* triHi, float4* cent, float4* partLo, float4* partHi)
        {
            __shared__ float4 sLo[256], sHi[256];
            float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.0f), hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.0f);
            for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
            {
                const float* p = pos + static_cast<size_t>(t) * 9;
                float4 bl = make_float4(p[0], p[1], p[2], 0.0f), bh = bl;
                for (int k = 1; k < 3; k++)
                {
                    const float4 v = make_float4(p[3 * k], p[3 * k + 1], p[3 * k + 2], 0.0f);
                    bl = fmin4(bl, v);
                    bh = fmax4(bh, v);
                }
                triLo[t] = bl;
                triHi[t] = bh;
                const float4 c = make_float4(0.5f * (bl.x + bh.x), 0.5f * (bl.y + bh.y), 0.5f * (bl.z + bh.z), 0.0f);
                cent[t] = c;
                lo = fmin4(lo, c);
                hi = fmax4(hi, c);
            }
            sLo[threadIdx.x] = lo;
            sHi[threadIdx.x] = hi;
            __syncthreads();
            for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1)
            {
                if (threadIdx.x < s)
                {
                    sLo[threadIdx.x] = fmin4(sLo[threadIdx.x], sLo[threadIdx.x + s]);
                    sHi[threadIdx.x] = fmax4(sHi[threadIdx.x], sHi[threadIdx.x + s]);
                }
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                partLo[blockIdx.x] = sLo[0];
                partHi[blockIdx.x] = sHi[0];
            }
        }

        __device__ __forceinline__ uint32_t expand_bits10(uint32_t v)
        {
            v = (v * 0x00010001u) & 0xFF0000FFu;
            v = (v * 0x00000101u) & 0x0F00F00Fu;
            v = (v * 0x00000011u) & 0xC30C30C3u;
            v = (v * 0x00000005u) & 0x49249249u;
            return v;
        }

        // One block of 256 threads: the bounds of the per-block bounds, into entry 0.
        __global__ void bounds_final_kernel(float4* partLo, float4* partHi, uint32_t parts)
        {
            __shared__ float4 sLo[256], sHi[256];
            float4 lo = partLo[0], hi = partHi[0];
            for (uint32_t i = threadIdx.x; i < parts; i += blockDim.x)
            {
                lo = fmin4(lo, partLo[i]);
                hi = fmax4(hi, partHi[i]);
            }
            sLo[threadIdx.x] = lo;
            sHi[threadIdx.x] = hi;
            __syncthreads();
            for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1)
            {
                if (threadIdx.x < s)
                {
                    sLo[threadIdx.x] = fmin4(sLo[threadIdx.x], sLo[threadIdx.x + s]);
                    sHi[threadIdx.x] = fmax4(sHi[threadIdx.x], sHi[threadIdx.x + s]);
                }
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                partLo[0] = sLo[0];
                partHi[0] = sHi[0];
            }
        }

        // The Morton code of every centroid within the centroids' bounds.
        __global__ void morton_kernel(const float4* cent, uint32_t n, const float4* boundsLo, const float4* boundsHi, uint32_t* keys, uint32_t* values)
        {
            const float4 lo = boundsLo[0], hi = boundsHi[0];
            const float ex = hi.x - lo.x, ey = hi.y - lo.y, ez = hi.z - lo.z;
            const float sx = ex > 0.0f ? 1023.0f / ex : 0.0f, sy = ey > 0.0f ? 1023.0f / ey : 0.0f, sz = ez > 0.0f ? 1023.0f / ez : 0.0f;
            for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
            {
                const float4 c = cent[t];
                const uint32_t x = static_cast<uint32_t>(fminf(fmaxf((c.x - lo.x) * sx, 0.0f), 1023.0f));
                const uint32_t y = static_cast<uint32_t>(fminf(fmaxf((c.y - lo.y) * sy, 0.0f), 1023.0f));
                const uint32_t z = static_cast<uint32_t>(fminf(fmaxf((c.z - lo.z) * sz, 0.0f), 1023.0f));
                keys[t] = (expand_bits10(x) << 2) | (expand_bits10(y) << 1) | expand_bits10(z);
                values[t] = t;
            }
        }

        // Leaf k = the k-th triangle of the sort; every cluster starts as one leaf.
        __global__ void leaves_kernel(const uint32_t* sorted, uint32_t n, const float4* triLo, const float4* triHi, float4* lo, float4* hi,
                                      uint2* child, uint32_t* clusters)
        {
            for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
            {
                const uint32_t t = sorted[k];
                lo[k] = triLo[t];
                hi[k] = triHi[t];
                child[k] = make_uint2(kInvalid, kInvalid);
                clusters[k] = k;
            }
        }

        // Nearest neighbour of every cluster within kPlocRadius positions (surface area of the merged box).
        __global__ void __launch_bounds__(kPlocBlock) ploc_nearest_kernel(const uint32_t* clusters, uint32_t m, const float4* lo, const float4* hi,
                                                                          uint32_t* nn)
        {
            __shared__ float4 sLo[kPlocBlock + 2 * kPlocRadius], sHi[kPlocBlock + 2 * kPlocRadius];
            const int start = static_cast<int>(blockIdx.x) * kPlocBlock - kPlocRadius;
            for (int k = threadIdx.x; k < kPlocBlock + 2 * kPlocRadius; k += kPlocBlock)
            {
                const int i = start + k;
                if (i >= 0 && i < static_cast<int>(m))
                {
                    const uint32_t c = clusters[i];
                    sLo[k] = lo[c];
                    sHi[k] = hi[c];
                }
            }
            __syncthreads();
            const int i = static_cast<int>(blockIdx.x) * kPlocBlock + static_cast<int>(threadIdx.x);
            if (i >= static_cast<int>(m)) return;
            const int si = i - start;
            const float4 myLo = sLo[si], myHi = sHi[si];
            const int jLo = i - kPlocRadius < 0 ? 0 : i - kPlocRadius;
            const int jHi = i + kPlocRadius > static_cast<int>(m) - 1 ? static_cast<int>(m) - 1 : i + kPlocRadius;
            float best = FLT_MAX;
            int bj = i == 0 ? 1 : i - 1;
            for (int j = jLo; j <= jHi; j++)
            {
                if (j == i) continue;
                const float a = box_area(fmin4(myLo, sLo[j - start]), fmax4(myHi, sHi[j - start]));
                if (a < best)
                {
                    best = a;
                    bj = j;
                }
            }
            nn[i] = static_cast<uint32_t>(bj);
        }

        // merge[i]: cluster i merges with its neighbour into a new node (mutual pair, i the smaller);
        // keep[i]: a cluster survives at position i (unpaired, or the smaller of a pair). Entry m is 0,
        // so the exclusive sums over m + 1 entries end with the totals.
        __global__ void ploc_flags_kernel(const uint32_t* nn, uint32_t m, uint32_t* merge, uint32_t* keep)
        {
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += gridDim.x * blockDim.x)
            {
                if (i == m)
                {
                    merge[i] = 0;
                    keep[i] = 0;
                    continue;
                }
                const uint32_t j = nn[i];
                const bool mutual = nn[j] == i;
                merge[i] = mutual && i < j ? 1u : 0u;
                keep[i] = mutual && i > j ? 0u : 1u;
            }
        }

        __global__ void ploc_merge_kernel(const uint32_t* clusters, uint32_t m, const uint32_t* nn, const uint32_t* merge, const uint32_t* mergePos,
                                          const uint32_t* keep, const uint32_t* keepPos, uint32_t nodeBase, float4* lo, float4* hi, uint2* child,
                                          uint32_t* next)
        {
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
            {
                if (!keep[i]) continue;
                uint32_t id = clusters[i];
                if (merge[i])
                {
                    const uint32_t other = clusters[nn[i]];
                    const uint32_t fresh = nodeBase + mergePos[i];
                    child[fresh] = make_uint2(id, other);
                    lo[fresh] = fmin4(lo[id], lo[other]);
                    hi[fresh] = fmax4(hi[id], hi[other]);
                    id = fresh;
                }
                next[keepPos[i]] = id;
            }
        }

        // Collapse costs (bvh8.cpp, CollapsePlan::plan): cost[8 i + j - 1] = cost of node i taking j slots
        // of its parent, how[] the choice, split[i] the left child's share when i becomes a wide node.
        __global__ void collapse_leaf_kernel(uint32_t n, const float4* lo, const float4* hi, float* cost, uint8_t* how)
        {
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const float A = box_area(lo[i], hi[i]);
                for (int k = 0; k < 8; k++)
                {
                    cost[static_cast<size_t>(i) * 8 + k] = A;  // area x one triangle
                    how[static_cast<size_t>(i) * 8 + k] = 0;
                }
            }
        }

        __global__ void collapse_node_kernel(uint32_t first, uint32_t end, const float4* lo, const float4* hi, const uint2* child, float* cost,
                                             uint8_t* how, uint8_t* split)
        {
            for (uint32_t i = first + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x)
            {
                const float A = box_area(lo[i], hi[i]);
                const uint2 c = child[i];
                const float* L = cost + static_cast<size_t>(c.x) * 8;
                const float* R = cost + static_cast<size_t>(c.y) * 8;
                float l[8], r[8];
                for (int k = 0; k < 8; k++)
                {
                    l[k] = L[k];
                    r[k] = R[k];
                }
                float D[9];
                uint8_t Dk[9] = {};
                for (int j = 2; j <= 8; j++)
                {
                    D[j] = FLT_MAX;
                    for (int k = 1; k < j; k++)
                    {
                        const float v = l[k - 1] + r[j - k - 1];
                        if (v < D[j])
                        {
                            D[j] = v;
                            Dk[j] = static_cast<uint8_t>(k);
                        }
                    }
                }
                split[i] = Dk[8];
                float C[8];
                uint8_t H[8];
                C[0] = A * kCollapseNodeCost + D[8];  // two or more triangles: never one leaf slot
                H[0] = 1;
                for (int s = 2; s <= 8; s++)
                {
                    if (D[s] < C[s - 2])
                    {
                        C[s - 1] = D[s];
                        H[s - 1] = Dk[s];
                    }
                    else
                    {
                        C[s - 1] = C[s - 2];
                        H[s - 1] = 0;
                    }
                }
                for (int k = 0; k < 8; k++)
                {
                    cost[static_cast<size_t>(i) * 8 + k] = C[k];
                    how[static_cast<size_t>(i) * 8 + k] = H[k];
                }
            }
        }

        // Box padding of bvh8.cpp (WideBuilder::padBox).
        __device__ void pad_box(float4 lo, float4 hi, double dlo[3], double dhi[3])
        {
            const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
            float ext = 0.0f, mag = 0.0f;
            for (int k = 0; k < 3; k++)
            {
                ext = fmaxf(ext, h[k] - l[k]);
                mag = fmaxf(mag, fmaxf(fabsf(l[k]), fabsf(h[k])));
            }
            const double pad = 1e-5 * static_cast<double>(ext) + 1e-7 * static_cast<double>(mag) + 1e-30;
            for (int k = 0; k < 3; k++)
            {
                dlo[k] = static_cast<double>(l[k]) - pad;
                dhi[k] = static_cast<double>(h[k]) + pad;
            }
        }

        __device__ __forceinline__ uint32_t pack4(const uint8_t* q)
        {
            return static_cast<uint32_t>(q[0]) | (static_cast<uint32_t>(q[1]) << 8) | (static_cast<uint32_t>(q[2]) << 16) | (static_cast<uint32_t>(q[3]) << 24);
        }

        // One level of wide nodes: node `levelBase + w` is binary node level[w]. Inner children get
        // consecutive indices from *counter and enter nextLevel at (index - nextBase).
        // capacity: entries of `out` and of nextLevel (an index beyond it is refused and reported).
        __global__ void emit_level_kernel(const uint32_t* level, uint32_t count, uint32_t levelBase, uint32_t nextBase, uint32_t n,
                                          const float4* lo, const float4* hi, const uint2* child, const uint8_t* how, const uint8_t* split,
                                          uint32_t* counter, uint32_t* nextLevel, Node8* out, uint32_t capacity, uint32_t* errorFlags)
        {
            for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x)
            {
                const uint32_t b = level[w];
                uint32_t kids[8];
                bool kidLeaf[8];
                int nk = 0;
                if (b < n)
                {
                    kids[0] = b;
                    kidLeaf[0] = true;
                    nk = 1;
                }
                else
                {
                    // CollapsePlan::children / collect, left before right
                    uint32_t stNode[kCollectStack];
                    uint8_t stSlots[kCollectStack];
                    int sp = 0;
                    const uint2 c = child[b];
                    const int s = split[b];
                    stNode[sp] = c.y;
                    stSlots[sp++] = static_cast<uint8_t>(8 - s);
                    stNode[sp] = c.x;
                    stSlots[sp++] = static_cast<uint8_t>(s);
                    bool bad = false;
                    while (sp > 0)
                    {
                        const uint32_t x = stNode[--sp];
                        const int i = stSlots[sp];
                        const uint8_t h = how[static_cast<size_t>(x) * 8 + i - 1];
                        if (i == 1)
                        {
                            if (nk >= 8)
                            {
                                bad = true;
                                break;
                            }
                            kids[nk] = x;
                            kidLeaf[nk] = h == 0;
                            nk++;
                        }
                        else if (h == 0)
                        {
                            stNode[sp] = x;
                            stSlots[sp++] = static_cast<uint8_t>(i - 1);
                        }
                        else
                        {
                            if (sp + 2 > kCollectStack)
                            {
                                bad = true;
                                break;
                            }
                            const uint2 cx = child[x];
                            stNode[sp] = cx.y;
                            stSlots[sp++] = static_cast<uint8_t>(i - h);
                            stNode[sp] = cx.x;
                            stSlots[sp++] = h;
                        }
                    }
                    if (bad)
                    {
                        atomicOr(errorFlags, kBuildErrCollect);
                        continue;
                    }
                }
                // slot assignment by octant (WideBuilder::emit)
                float4 nlo = lo[kids[0]], nhi = hi[kids[0]];
                for (int i = 1; i < nk; i++)
                {
                    nlo = fmin4(nlo, lo[kids[i]]);
                    nhi = fmax4(nhi, hi[kids[i]]);
                }
                const float center[3] = {0.5f * (nlo.x + nhi.x), 0.5f * (nlo.y + nhi.y), 0.5f * (nlo.z + nhi.z)};
                int slotOf[8] = {};
                bool slotUsed[8] = {}, kidUsed[8] = {};
                for (int round = 0; round < nk; round++)
                {
                    float bestScore = -FLT_MAX;
                    int bk = -1, bs = -1;
                    for (int i = 0; i < nk; i++)
                    {
                        if (kidUsed[i]) continue;
                        const float4 cl = lo[kids[i]], ch = hi[kids[i]];
                        const float v[3] = {0.5f * (cl.x + ch.x) - center[0], 0.5f * (cl.y + ch.y) - center[1], 0.5f * (cl.z + ch.z) - center[2]};
                        for (int s = 0; s < 8; s++)
                        {
                            if (slotUsed[s]) continue;
                            const float score = ((s & 1) ? v[0] : -v[0]) + ((s & 2) ? v[1] : -v[1]) + ((s & 4) ? v[2] : -v[2]);
                            if (score > bestScore)
                            {
                                bestScore = score;
                                bk = i;
                                bs = s;
                            }
                        }
                    }
                    kidUsed[bk] = true;
                    slotUsed[bs] = true;
                    slotOf[bk] = bs;
                }
                // child references: inner children take consecutive indices in the order of the child list
                int inner = 0;
                for (int i = 0; i < nk; i++) inner += kidLeaf[i] ? 0 : 1;
                const uint32_t firstInner = inner ? atomicAdd(counter, static_cast<uint32_t>(inner)) : 0u;
                uint32_t childRef[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                uint8_t counts[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                uint32_t innerMask = 0, leafMask = 0;
                int r = 0;
                for (int i = 0; i < nk; i++)
                {
                    const int s = slotOf[i];
                    if (kidLeaf[i])
                    {
                        childRef[s] = kids[i] | (1u << 24);  // leaf position (24 bits), one triangle
                        counts[s] = 1;
                        leafMask |= 1u << s;
                    }
                    else
                    {
                        const uint32_t at = firstInner + static_cast<uint32_t>(r++);
                        childRef[s] = at;
                        if (at < capacity && at >= nextBase) nextLevel[at - nextBase] = kids[i];
                        else atomicOr(errorFlags, kBuildErrCapacity);
                        innerMask |= 1u << s;
                    }
                }
                if (levelBase + w >= capacity)
                {
                    atomicOr(errorFlags, kBuildErrCapacity);
                    continue;
                }
                // quantisation (WideBuilder::emit): origin rounded down to float, power-of-two scales, every
                // quantised box checked in double to contain its padded child box
                double clo[8][3], chi[8][3];
                bool valid[8] = {};
                double plo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, phi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
                for (int i = 0; i < nk; i++)
                {
                    const int s = slotOf[i];
                    pad_box(lo[kids[i]], hi[kids[i]], clo[s], chi[s]);
                    valid[s] = true;
                    for (int a = 0; a < 3; a++)
                    {
                        plo[a] = fmin(plo[a], clo[s][a]);
                        phi[a] = fmax(phi[a], chi[s][a]);
                    }
                }
                float p[3];
                int expo[3];
                uint8_t qlo[3][8], qhi[3][8];
                bool overflow = false;
                for (int a = 0; a < 3; a++)
                {
                    float pf = __double2float_rd(plo[a]);
                    p[a] = pf;
                    const double ext = phi[a] - static_cast<double>(pf);
                    int e = -126;
                    if (ext > 0.0)
                    {
                        int fe;
                        frexp(ext / 255.0, &fe);
                        e = max(-126, min(127, fe));
                    }
                    for (;;)
                    {
                        const double scale = ldexp(1.0, e);
                        bool ok = true;
                        for (int s = 0; s < 8 && ok; s++)
                        {
                            if (!valid[s])
                            {
                                qlo[a][s] = 255;
                                qhi[a][s] = 0;
                                continue;
                            }
                            double ql = floor((clo[s][a] - pf) / scale);
                            double qh = ceil((chi[s][a] - pf) / scale);
                            ql = fmax(0.0, ql);
                            while (ql > 0 && static_cast<double>(pf) + ql * scale > clo[s][a]) ql -= 1.0;
                            while (static_cast<double>(pf) + qh * scale < chi[s][a]) qh += 1.0;
                            if (qh > 255.0 || static_cast<double>(pf) + ql * scale > clo[s][a])
                            {
                                ok = false;
                                break;
                            }
                            qlo[a][s] = static_cast<uint8_t>(ql);
                            qhi[a][s] = static_cast<uint8_t>(qh);
                        }
                        if (ok) break;
                        e++;
                        if (e > 127)
                        {
                            overflow = true;
                            break;
                        }
                    }
                    if (overflow) break;
                    expo[a] = e;
                }
                if (overflow)
                {
                    atomicOr(errorFlags, kBuildErrExponent);
                    continue;
                }
                Node8 node;
                const uint32_t header = static_cast<uint32_t>(expo[0] + 127) | (static_cast<uint32_t>(expo[1] + 127) << 8) |
                                        (static_cast<uint32_t>(expo[2] + 127) << 16) | (innerMask << 24);
                node.w[0] = make_uint4(__float_as_uint(p[0]), __float_as_uint(p[1]), __float_as_uint(p[2]), header);
                node.w[1] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
                node.w[2] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
                node.w[3] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
                node.w[4] = make_uint4(childRef[0], childRef[1], childRef[2], childRef[3]);
                node.w[5] = make_uint4(childRef[4], childRef[5], childRef[6], childRef[7]);
                node.w[6] = make_uint4(pack4(counts), pack4(counts + 4), leafMask, 0);
                node.w[7] = make_uint4(0, 0, 0, 0);
                out[levelBase + w] = node;
            }
        }

        // Triangle records in leaf order (bvh8.cpp, BuildBvh8): (v0, input index), (e1, model), (e2, 0), 0.
        __global__ void triangle_records_kernel(const float* pos, const uint32_t* models, const uint32_t* sorted, uint32_t n, float4* tris)
        {
            for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
            {
                const uint32_t t = sorted[k];
                const float* p = pos + static_cast<size_t>(t) * 9;
                tris[static_cast<size_t>(k) * kTriangleVec4 + 0] = make_float4(p[0], p[1], p[2], __uint_as_float(t));
                tris[static_cast<size_t>(k) * kTriangleVec4 + 1] = make_float4(p[3] - p[0], p[4] - p[1], p[5] - p[2], __uint_as_float(models[t]));
                tris[static_cast<size_t>(k) * kTriangleVec4 + 2] = make_float4(p[6] - p[0], p[7] - p[1], p[8] - p[2], 0.0f);
                tris[static_cast<size_t>(k) * kTriangleVec4 + 3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }

        uint32_t grid_for(uint32_t items, uint32_t threads, uint32_t cap = 65535u)
        {
            const uint32_t g = (items + threads - 1) / threads;
            return g < 1 ? 1 : (g > cap ? cap : g);
        }
    }

    Status BuildBvh8Device(const float* positions, const uint32_t* models, uint32_t n, cudaStream_t s, DeviceBvh& out)
    {
        if (n == 0) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "BVH build failed: scene has no triangles");
        if (n > kMaxTriangles) return Status::Err(GPT_ERR_CAPACITY, "BVH build failed: scene has more than 2^24 triangles");
        const uint32_t nodes = 2 * n - 1;
        DeviceBuffer triLo, triHi, cent, partLo, partHi, keys, keysSorted, values, sorted, lo, hi, child, clustersA, clustersB, nn, merge, mergePos, keep,
            keepPos, cost, how, split, levelA, levelB, counter, errorFlags, temp, wide;
        const uint32_t parts = grid_for(n, 256, 1024);
        PT_TRY(triLo.allocate(size_t(n) * 16));
        PT_TRY(triHi.allocate(size_t(n) * 16));
        PT_TRY(cent.allocate(size_t(n) * 16));
        PT_TRY(partLo.allocate(size_t(parts) * 16));
        PT_TRY(partHi.allocate(size_t(parts) * 16));
        PT_TRY(keys.allocate(size_t(n) * 4));
        PT_TRY(keysSorted.allocate(size_t(n) * 4));
        PT_TRY(values.allocate(size_t(n) * 4));
        PT_TRY(sorted.allocate(size_t(n) * 4));
        PT_TRY(lo.allocate(size_t(nodes) * 16));
        PT_TRY(hi.allocate(size_t(nodes) * 16));
        PT_TRY(child.allocate(size_t(nodes) * 8));
        PT_TRY(clustersA.allocate(size_t(n) * 4));
        PT_TRY(clustersB.allocate(size_t(n) * 4));
        PT_TRY(nn.allocate(size_t(n) * 4));
        PT_TRY(merge.allocate(size_t(n + 1) * 4));
        PT_TRY(mergePos.allocate(size_t(n + 1) * 4));
        PT_TRY(keep.allocate(size_t(n + 1) * 4));
        PT_TRY(keepPos.allocate(size_t(n + 1) * 4));
        PT_TRY(cost.allocate(size_t(nodes) * 8 * 4));
        PT_TRY(how.allocate(size_t(nodes) * 8));
        PT_TRY(split.allocate(size_t(nodes)));
        PT_TRY(levelA.allocate(size_t(n) * 4));
        PT_TRY(levelB.allocate(size_t(n) * 4));
        PT_TRY(counter.allocate(16));
        PT_TRY(errorFlags.allocate(16));
        PT_TRY(wide.allocate(size_t(n) * sizeof(Node8)));  // at most one wide node per binary inner node (one for n = 1)
        size_t sortBytes = 0, scanBytes = 0;
        PT_CUDA("cub::DeviceRadixSort::SortPairs", cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, keys.get<uint32_t>(), keysSorted.get<uint32_t>(),
                                                                                 values.get<uint32_t>(), sorted.get<uint32_t>(), static_cast<int>(n), 0, 30, s));
        PT_CUDA("cub::DeviceScan::ExclusiveSum", cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, merge.get<uint32_t>(), mergePos.get<uint32_t>(),
                                                                              static_cast<int>(n + 1), s));
        PT_TRY(temp.allocate(sortBytes > scanBytes ? sortBytes : scanBytes));
        PT_CUDA("cudaMemsetAsync", cudaMemsetAsync(errorFlags.get<void>(), 0, 16, s));

        // 1-2: boxes, centroids, Morton order
        triangle_boxes_kernel<<<parts, 256, 0, s>>>(positions, n, triLo.get<float4>(), triHi.get<float4>(), cent.get<float4>(), partLo.get<float4>(),
                                                    partHi.get<float4>());
        PT_CUDA("triangle boxes", cudaGetLastError());
        bounds_final_kernel<<<1, 256, 0, s>>>(partLo.get<float4>(), partHi.get<float4>(), parts);
        PT_CUDA("centroid bounds", cudaGetLastError());
        morton_kernel<<<grid_for(n, 256, 4096), 256, 0, s>>>(cent.get<float4>(), n, partLo.get<float4>(), partHi.get<float4>(),
                                                             keys.get<uint32_t>(), values.get<uint32_t>());
        PT_CUDA("morton codes", cudaGetLastError());
        size_t tb = temp.bytes();
        PT_CUDA("cub::DeviceRadixSort::SortPairs", cub::DeviceRadixSort::SortPairs(temp.get<void>(), tb, keys.get<uint32_t>(), keysSorted.get<uint32_t>(),
                                                                                 values.get<uint32_t>(), sorted.get<uint32_t>(), static_cast<int>(n), 0, 30, s));
        leaves_kernel<<<grid_for(n, 256, 4096), 256, 0, s>>>(sorted.get<uint32_t>(), n, triLo.get<float4>(), triHi.get<float4>(), lo.get<float4>(),
                                                             hi.get<float4>(), child.get<uint2>(), clustersA.get<uint32_t>());
        PT_CUDA("leaves", cudaGetLastError());

        // 3: clustering rounds; rounds[r] = first node index of round r (nodes of round r: [rounds[r], rounds[r + 1]))
        std::vector<uint32_t> rounds{n};
        uint32_t m = n, nodeBase = n;
        uint32_t* cur = clustersA.get<uint32_t>();
        uint32_t* nxt = clustersB.get<uint32_t>();
        uint32_t totals[2] = {0, 0};
        const uint32_t maxRounds = n + 8;  // every round merges at least the closest pair of its windows
        while (m > 1)
        {
            if (rounds.size() > maxRounds) return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: clustering did not converge");
            ploc_nearest_kernel<<<(m + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, s>>>(cur, m, lo.get<float4>(), hi.get<float4>(), nn.get<uint32_t>());
            PT_CUDA("nearest clusters", cudaGetLastError());
            ploc_flags_kernel<<<grid_for(m + 1, 256, 8192), 256, 0, s>>>(nn.get<uint32_t>(), m, merge.get<uint32_t>(), keep.get<uint32_t>());
            PT_CUDA("cluster flags", cudaGetLastError());
            tb = temp.bytes();
            PT_CUDA("cub::DeviceScan::ExclusiveSum", cub::DeviceScan::ExclusiveSum(temp.get<void>(), tb, merge.get<uint32_t>(), mergePos.get<uint32_t>(),
                                                                                  static_cast<int>(m + 1), s));
            tb = temp.bytes();
            PT_CUDA("cub::DeviceScan::ExclusiveSum", cub::DeviceScan::ExclusiveSum(temp.get<void>(), tb, keep.get<uint32_t>(), keepPos.get<uint32_t>(),
                                                                                  static_cast<int>(m + 1), s));
            ploc_merge_kernel<<<grid_for(m, 256, 8192), 256, 0, s>>>(cur, m, nn.get<uint32_t>(), merge.get<uint32_t>(), mergePos.get<uint32_t>(),
                                                                     keep.get<uint32_t>(), keepPos.get<uint32_t>(), nodeBase, lo.get<float4>(),
                                                                     hi.get<float4>(), child.get<uint2>(), nxt);
            PT_CUDA("cluster merge", cudaGetLastError());
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&totals[0], mergePos.get<uint32_t>() + m, 4, cudaMemcpyDeviceToHost, s));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&totals[1], keepPos.get<uint32_t>() + m, 4, cudaMemcpyDeviceToHost, s));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(s));
            if (totals[0] == 0 || totals[1] != m - totals[0])
                return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: a clustering round merged no pair");
            nodeBase += totals[0];
            m = totals[1];
            rounds.push_back(nodeBase);
            std::swap(cur, nxt);
        }
        if (nodeBase != nodes) return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: clustering left the wrong number of nodes");
        const uint32_t root = nodes - 1;

        // 4: collapse costs, one round at a time (children before parents)
        collapse_leaf_kernel<<<grid_for(n, 256, 8192), 256, 0, s>>>(n, lo.get<float4>(), hi.get<float4>(), cost.get<float>(), how.get<uint8_t>());
        PT_CUDA("collapse leaves", cudaGetLastError());
        for (size_t r = 0; r + 1 < rounds.size(); r++)
        {
            const uint32_t a = rounds[r], b = rounds[r + 1];
            collapse_node_kernel<<<grid_for(b - a, 128, 8192), 128, 0, s>>>(a, b, lo.get<float4>(), hi.get<float4>(), child.get<uint2>(), cost.get<float>(),
                                                                            how.get<uint8_t>(), split.get<uint8_t>());
            PT_CUDA("collapse nodes", cudaGetLastError());
        }

        // 5: wide nodes level by level
        const uint32_t one = 1;
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(levelA.get<uint32_t>(), &root, 4, cudaMemcpyHostToDevice, s));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(counter.get<uint32_t>(), &one, 4, cudaMemcpyHostToDevice, s));
        uint32_t levelBase = 0, count = 1, depth = 0, allocated = 1;
        uint32_t* level = levelA.get<uint32_t>();
        uint32_t* nextLevel = levelB.get<uint32_t>();
        while (count > 0)
        {
            depth++;
            if (depth > kMaxStack) return Status::Err(GPT_ERR_CAPACITY, "BVH8 deeper than the traversal stack");
            emit_level_kernel<<<grid_for(count, 128, 16384), 128, 0, s>>>(level, count, levelBase, levelBase + count, n, lo.get<float4>(), hi.get<float4>(),
                                                                          child.get<uint2>(), how.get<uint8_t>(), split.get<uint8_t>(),
                                                                          counter.get<uint32_t>(), nextLevel, wide.get<Node8>(), n,
                                                                          errorFlags.get<uint32_t>());
            PT_CUDA("wide nodes", cudaGetLastError());
            uint32_t levelFlags = 0;
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&allocated, counter.get<uint32_t>(), 4, cudaMemcpyDeviceToHost, s));
            PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(&levelFlags, errorFlags.get<uint32_t>(), 4, cudaMemcpyDeviceToHost, s));
            PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(s));
            if (allocated > n) return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: more wide nodes than the bound");
            if (levelFlags) break;  // reported below; the next level's list is incomplete
            levelBase += count;
            count = allocated - levelBase;
            std::swap(level, nextLevel);
        }
        uint32_t flags = 0;
        PT_CUDA("cudaMemcpy", cudaMemcpy(&flags, errorFlags.get<void>(), 4, cudaMemcpyDeviceToHost));
        if (flags & kBuildErrExponent) return Status::Err(GPT_ERR_INVALID_ARGUMENT, "BVH build failed: BVH quantisation exponent overflow");
        if (flags & kBuildErrCapacity) return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: a wide-node index beyond the node array");
        if (flags) return Status::Err(GPT_ERR_DEVICE_FAULT, "BVH build failed: a wide node's child list did not fit");
        if (allocated >= (1u << 24)) return Status::Err(GPT_ERR_CAPACITY, "BVH8 has more than 2^24 nodes");

        // 6: triangle records; the wide nodes move into an allocation of their exact size
        PT_TRY(out.tris.allocate(size_t(n) * kTriangleVec4 * sizeof(float4)));
        triangle_records_kernel<<<grid_for(n, 256, 8192), 256, 0, s>>>(positions, models, sorted.get<uint32_t>(), n, out.tris.get<float4>());
        PT_CUDA("triangle records", cudaGetLastError());
        PT_TRY(out.nodes.allocate(size_t(allocated) * sizeof(Node8)));
        PT_CUDA("cudaMemcpyAsync", cudaMemcpyAsync(out.nodes.get<void>(), wide.get<void>(), size_t(allocated) * sizeof(Node8), cudaMemcpyDeviceToDevice, s));
        PT_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(s));
        out.nodeCount = allocated;
        out.depth = depth;
        out.binaryNodes = nodes;
        out.rounds = static_cast<uint32_t>(rounds.size() - 1);
        return Status::Ok();
    }
}
