// Host construction of the 8-wide, 8-bit-quantised BVH.
//
// Replaces the reference's median-split binary BVH (Core/Source/Graphics/Cuda/Bvh/HostBvh.cpp:22-100)
// and its DFS flattening to 40-byte nodes (Core/Source/Graphics/Cuda/Bvh/DeviceBvh.cpp:7-52).
//  1. Binary BVH by binned SAH (32 bins, all three axes), one triangle per leaf: the 8-wide node's
//     quantised box test then culls single triangles, which costs less than their triangle tests
//     (on a 1.3M-triangle frame, leaves of up to 4 triangles took 3.46 triangle tests and 7.84 node
//     visits per closest-hit ray; single-triangle leaves take 2.70 and 8.23, and the frame is 2% faster).
//  2. Collapse to 8-wide by the surface-area-optimal distribution of binary subtrees over child slots
//     (the dynamic programme of Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on
//     GPUs Through Compressed Wide BVHs", HPG 2017): for every binary node and every slot budget
//     i = 1..8, the least expected cost of its subtree in at most i slots of the parent wide node,
//     where a wide node costs its area x kNodeCost and a leaf its area x its triangle count. On the
//     1.3M-triangle frame this gives 256K instead of 422K nodes (6.1 instead of 4.1 children per node)
//     and 7.91 instead of 8.23 node visits per closest-hit ray against greedily opening the child of
//     largest area, and a 2.7% faster frame. Leaves stay single triangles: letting the programme
//     choose leaves of 2 or 3 triangles gave fewer nodes but more triangle tests and slower frames.
//  3. Child slots are assigned by octant (greedy on dot(child centre - node centre, octant
//     direction)) so a ray visiting slot i ^ octant(ray) goes roughly front to back.
//  4. Child boxes are padded (1e-5 of their largest extent, plus a relative 1e-7 of their
//     coordinates) and quantised to 8 bits per axis against the node origin with a power-of-two
//     scale, rounding outward; every quantised box is checked in exact arithmetic to contain the
//     padded child box.
#include "bvh8.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <future>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace pt
{
    namespace
    {
        struct Box
        {
            float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
            float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            void grow(const Box& b)
            {
                for (int k = 0; k < 3; k++)
                {
                    lo[k] = std::min(lo[k], b.lo[k]);
                    hi[k] = std::max(hi[k], b.hi[k]);
                }
            }
            void grow(const float* p)
            {
                for (int k = 0; k < 3; k++)
                {
                    lo[k] = std::min(lo[k], p[k]);
                    hi[k] = std::max(hi[k], p[k]);
                }
            }
            float area() const
            {
                float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
                if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
                return 2.0f * (dx * dy + dy * dz + dz * dx);
            }
        };

        struct BNode
        {
            Box box;
            uint32_t left = kInvalid, right = kInvalid;
            uint32_t first = 0, count = 0;
            bool leaf() const { return left == kInvalid; }
        };

        constexpr int kBins = 32;
        constexpr uint32_t kMaxLeaf = 1;
        constexpr float kTraversalCost = 1.2f;
        // Nodes of at least this many triangles compute their bounds, bins and partition on several
        // threads, in fixed chunks of kChunk triangles (the tree does not depend on the thread count).
        // Near the root the SAH peels off one cluster of triangles at a time, so a serial build spends
        // most of its time in a chain of large nodes that no subtree-level parallelism shortens.
        constexpr uint32_t kParallelNode = 1u << 18;
        constexpr uint32_t kChunk = 1u << 16;

        // f(c) for every chunk c in [0, chunks), on at most `threads` threads
        template <class F>
        void for_chunks(uint32_t chunks, int threads, F&& f)
        {
            std::atomic<uint32_t> next{0};
            auto worker = [&]
            {
                for (uint32_t c; (c = next.fetch_add(1)) < chunks;) f(c);
            };
            const int t = static_cast<int>(std::min<uint32_t>(static_cast<uint32_t>(std::max(threads, 1)), chunks));
            std::vector<std::thread> pool;
            for (int i = 1; i < t; i++) pool.emplace_back(worker);
            worker();
            for (auto& th : pool) th.join();
        }

        // Bins of one range of triangles along all three axes.
        struct Bins
        {
            uint32_t cnt[3][kBins] = {};
            Box box[3][kBins];
            void merge(const Bins& o)
            {
                for (int k = 0; k < 3; k++)
                    for (int b = 0; b < kBins; b++)
                    {
                        cnt[k][b] += o.cnt[k][b];
                        box[k][b].grow(o.box[k][b]);
                    }
            }
        };

        struct BinaryBuilder
        {
            const float* pos;
            uint32_t n;
            std::vector<Box> triBox;
            std::vector<float> cent;  // 3 per triangle
            std::vector<uint32_t> idx;
            std::vector<BNode> nodes;
            std::atomic<uint32_t> nodeCount{0};
            std::atomic<int> spawned{0};
            int maxThreads = 1;

            uint32_t alloc()
            {
                uint32_t i = nodeCount.fetch_add(1);
                if (i >= nodes.size()) throw std::runtime_error("BVH node pool exhausted");
                return i;
            }

            int bin_of(uint32_t t, int k, float lo, float scale) const
            {
                const int b = static_cast<int>((cent[static_cast<size_t>(t) * 3 + k] - lo) * scale);
                return std::min(std::max(b, 0), kBins - 1);
            }

            void bin_range(uint32_t begin, uint32_t end, const Box& cbox, const float scale[3], Bins& out) const
            {
                for (uint32_t i = begin; i < end; i++)
                {
                    const uint32_t t = idx[i];
                    for (int k = 0; k < 3; k++)
                    {
                        if (!(scale[k] > 0.0f)) continue;
                        const int b = bin_of(t, k, cbox.lo[k], scale[k]);
                        out.cnt[k][b]++;
                        out.box[k][b].grow(triBox[t]);
                    }
                }
            }

            uint32_t build(uint32_t first, uint32_t count, int depth)
            {
                const uint32_t me = alloc();
                const bool parallel = count >= kParallelNode && maxThreads > 1;
                const uint32_t chunks = (count + kChunk - 1) / kChunk;
                Box box, cbox;
                if (parallel)
                {
                    std::vector<Box> boxes(chunks), cboxes(chunks);
                    for_chunks(chunks, maxThreads, [&](uint32_t c)
                    {
                        const uint32_t b = first + c * kChunk, e = std::min(first + count, b + kChunk);
                        for (uint32_t i = b; i < e; i++)
                        {
                            boxes[c].grow(triBox[idx[i]]);
                            cboxes[c].grow(&cent[static_cast<size_t>(idx[i]) * 3]);
                        }
                    });
                    for (uint32_t c = 0; c < chunks; c++)
                    {
                        box.grow(boxes[c]);
                        cbox.grow(cboxes[c]);
                    }
                }
                else
                    for (uint32_t i = first; i < first + count; i++)
                    {
                        const uint32_t t = idx[i];
                        box.grow(triBox[t]);
                        cbox.grow(&cent[static_cast<size_t>(t) * 3]);
                    }
                BNode node;
                node.box = box;
                node.first = first;
                node.count = count;
                if (count <= 1 || depth >= 60)
                {
                    nodes[me] = node;
                    return me;
                }
                // binned SAH over the three axes, one pass over the triangles for all three
                float bestCost = FLT_MAX;
                int bestAxis = -1, bestBin = -1;
                const float parentArea = std::max(box.area(), 1e-30f);
                float scales[3];
                for (int k = 0; k < 3; k++)
                {
                    const float ext = cbox.hi[k] - cbox.lo[k];
                    scales[k] = ext > 0.0f ? kBins / ext : 0.0f;
                }
                Bins bins;
                if (parallel)
                {
                    std::vector<Bins> part(chunks);
                    for_chunks(chunks, maxThreads, [&](uint32_t c)
                    {
                        const uint32_t b = first + c * kChunk, e = std::min(first + count, b + kChunk);
                        bin_range(b, e, cbox, scales, part[c]);
                    });
                    for (uint32_t c = 0; c < chunks; c++) bins.merge(part[c]);
                }
                else
                    bin_range(first, first + count, cbox, scales, bins);
                for (int k = 0; k < 3; k++)
                {
                    if (!(scales[k] > 0.0f)) continue;
                    const uint32_t* cnt = bins.cnt[k];
                    const Box* bb = bins.box[k];
                    float areaL[kBins], areaR[kBins];
                    uint32_t cntL[kBins], cntR[kBins];
                    Box acc;
                    uint32_t c = 0;
                    for (int b = 0; b < kBins; b++)
                    {
                        acc.grow(bb[b]);
                        c += cnt[b];
                        areaL[b] = acc.area();
                        cntL[b] = c;
                    }
                    acc = Box();
                    c = 0;
                    for (int b = kBins - 1; b >= 0; b--)
                    {
                        acc.grow(bb[b]);
                        c += cnt[b];
                        areaR[b] = acc.area();
                        cntR[b] = c;
                    }
                    for (int b = 0; b < kBins - 1; b++)
                    {
                        if (cntL[b] == 0 || cntR[b + 1] == 0) continue;
                        float cost = kTraversalCost + (areaL[b] * cntL[b] + areaR[b + 1] * cntR[b + 1]) / parentArea;
                        if (cost < bestCost)
                        {
                            bestCost = cost;
                            bestAxis = k;
                            bestBin = b;
                        }
                    }
                }
                if (count <= kMaxLeaf && static_cast<float>(count) <= bestCost)
                {
                    nodes[me] = node;
                    return me;
                }
                uint32_t mid;
                if (bestAxis < 0)
                {
                    if (count <= kMaxLeaf)
                    {
                        nodes[me] = node;
                        return me;
                    }
                    mid = first + count / 2;  // identical centroids: split the range
                }
                else
                {
                    const float lo = cbox.lo[bestAxis];
                    const float scale = scales[bestAxis];
                    auto left = [&](uint32_t t) { return bin_of(t, bestAxis, lo, scale) <= bestBin; };
                    if (parallel)
                    {
                        // stable partition by chunks: left entries of every chunk in order, then the right ones
                        std::vector<uint32_t> nLeft(chunks + 1, 0);
                        for_chunks(chunks, maxThreads, [&](uint32_t c)
                        {
                            const uint32_t b = first + c * kChunk, e = std::min(first + count, b + kChunk);
                            uint32_t n = 0;
                            for (uint32_t i = b; i < e; i++) n += left(idx[i]) ? 1u : 0u;
                            nLeft[c + 1] = n;
                        });
                        for (uint32_t c = 0; c < chunks; c++) nLeft[c + 1] += nLeft[c];
                        const uint32_t totalLeft = nLeft[chunks];
                        std::vector<uint32_t> tmp(count);
                        for_chunks(chunks, maxThreads, [&](uint32_t c)
                        {
                            const uint32_t b = first + c * kChunk, e = std::min(first + count, b + kChunk);
                            uint32_t l = nLeft[c], r = totalLeft + (b - first) - nLeft[c];
                            for (uint32_t i = b; i < e; i++)
                            {
                                const uint32_t t = idx[i];
                                if (left(t)) tmp[l++] = t;
                                else tmp[r++] = t;
                            }
                        });
                        std::copy(tmp.begin(), tmp.end(), idx.begin() + first);
                        mid = first + totalLeft;
                    }
                    else
                    {
                        auto it = std::partition(idx.begin() + first, idx.begin() + first + count, left);
                        mid = static_cast<uint32_t>(it - idx.begin());
                    }
                    if (mid == first || mid == first + count) mid = first + count / 2;
                }
                uint32_t l, r;
                if (count > 65536 && spawned.fetch_add(1) < maxThreads)
                {
                    // a subtree on its own thread; the slot is given back when it is done
                    auto fut = std::async(std::launch::async, [&, first, mid, depth]()
                    {
                        const uint32_t res = build(first, mid - first, depth + 1);
                        spawned.fetch_sub(1);
                        return res;
                    });
                    r = build(mid, first + count - mid, depth + 1);
                    l = fut.get();
                }
                else if (count > 65536)
                {
                    spawned.fetch_sub(1);
                    l = build(first, mid - first, depth + 1);
                    r = build(mid, first + count - mid, depth + 1);
                }
                else
                {
                    l = build(first, mid - first, depth + 1);
                    r = build(mid, first + count - mid, depth + 1);
                }
                node.left = l;
                node.right = r;
                nodes[me] = node;
                return me;
            }
        };

        constexpr float kNodeCost = 2.0f;     // wide-node visit against one triangle test
        constexpr uint32_t kWideLeafMax = 1;   // most triangles in one leaf slot of a wide node

        // Surface-area-optimal distribution of binary subtrees over the 8 child slots of wide nodes.
        struct CollapsePlan
        {
            const BinaryBuilder& bin;
            std::vector<float> cost;     // [node * 8 + i - 1]: least cost of the subtree in at most i slots
            std::vector<uint8_t> how;    // i == 1: 0 leaf, 1 wide node; i > 1: 0 = as in i - 1 slots, k = k slots to the left child
            std::vector<uint8_t> split;  // slots of the left child in the node's own wide node
            std::vector<uint32_t> wide;  // wide nodes of the subtree of a binary node that becomes a wide node
            int maxThreads = 1;
            std::atomic<int> spawned{0};

            // a subtree on another thread while one is free (large subtrees only)
            template <class F>
            bool spawn_if_free(uint32_t triangles, F&& f, std::future<void>& fut)
            {
                if (triangles < kParallelNode) return false;
                if (spawned.fetch_add(1) >= maxThreads)
                {
                    spawned.fetch_sub(1);
                    return false;
                }
                fut = std::async(std::launch::async, [this, f]()
                {
                    f();
                    spawned.fetch_sub(1);
                });
                return true;
            }

            void plan(uint32_t n)
            {
                const BNode& b = bin.nodes[n];
                const float A = b.box.area();
                float* C = &cost[static_cast<size_t>(n) * 8];
                uint8_t* H = &how[static_cast<size_t>(n) * 8];
                if (b.leaf())
                {
                    for (int i = 0; i < 8; i++)
                    {
                        C[i] = A * static_cast<float>(b.count);
                        H[i] = 0;
                    }
                    return;
                }
                std::future<void> fut;
                const uint32_t left = b.left;
                const bool async = spawn_if_free(bin.nodes[left].count, [this, left] { plan(left); }, fut);
                if (!async) plan(b.left);
                plan(b.right);
                if (async) fut.get();
                const float* L = &cost[static_cast<size_t>(b.left) * 8];
                const float* R = &cost[static_cast<size_t>(b.right) * 8];
                float D[9];
                uint8_t Dk[9] = {};
                for (int j = 2; j <= 8; j++)
                {
                    D[j] = FLT_MAX;
                    for (int k = 1; k < j; k++)
                    {
                        const float v = L[k - 1] + R[j - k - 1];
                        if (v < D[j])
                        {
                            D[j] = v;
                            Dk[j] = static_cast<uint8_t>(k);
                        }
                    }
                }
                split[n] = Dk[8];
                const float nodeCost = A * kNodeCost + D[8];
                const float leafCost = b.count <= kWideLeafMax ? A * static_cast<float>(b.count) : FLT_MAX;
                C[0] = std::min(leafCost, nodeCost);
                H[0] = leafCost <= nodeCost ? 0 : 1;
                for (int i = 2; i <= 8; i++)
                {
                    if (D[i] < C[i - 2])
                    {
                        C[i - 1] = D[i];
                        H[i - 1] = Dk[i];
                    }
                    else
                    {
                        C[i - 1] = C[i - 2];
                        H[i - 1] = 0;
                    }
                }
            }

            // The children that node n contributes with i slots: binary nodes, each a leaf slot or a wide node.
            void collect(uint32_t n, int i, std::vector<uint32_t>& kids, std::vector<uint8_t>& leaf) const
            {
                const uint8_t h = how[static_cast<size_t>(n) * 8 + i - 1];
                if (i == 1)
                {
                    kids.push_back(n);
                    leaf.push_back(h == 0 ? 1 : 0);
                    return;
                }
                if (h == 0)
                {
                    collect(n, i - 1, kids, leaf);
                    return;
                }
                const BNode& b = bin.nodes[n];
                collect(b.left, h, kids, leaf);
                collect(b.right, i - h, kids, leaf);
            }

            // The child list of the wide node a binary node becomes.
            void children(uint32_t n, std::vector<uint32_t>& kids, std::vector<uint8_t>& leaf) const
            {
                kids.clear();
                leaf.clear();
                const BNode& b = bin.nodes[n];
                if (b.leaf())
                {
                    kids.push_back(n);
                    leaf.push_back(1);
                    return;
                }
                collect(b.left, split[n], kids, leaf);
                collect(b.right, 8 - split[n], kids, leaf);
            }

            // wide[n] for binary node n and every wide node below it; returns it
            uint32_t count_wide(uint32_t n)
            {
                std::vector<uint32_t> kids;
                std::vector<uint8_t> leaf;
                children(n, kids, leaf);
                uint32_t total = 1;
                std::vector<std::future<void>> futs;
                for (size_t i = 0; i < kids.size(); i++)
                {
                    if (leaf[i]) continue;
                    const uint32_t k = kids[i];
                    std::future<void> fut;
                    if (spawn_if_free(bin.nodes[k].count, [this, k] { count_wide(k); }, fut)) futs.push_back(std::move(fut));
                    else count_wide(k);
                }
                for (auto& f : futs) f.get();
                for (size_t i = 0; i < kids.size(); i++)
                    if (!leaf[i]) total += wide[kids[i]];
                wide[n] = total;
                return total;
            }
        };

        // Wide nodes in depth-first pre-order (a node, then the subtrees of its inner children in slot
        // assignment order). Every subtree's place is known from the plan's node counts, so large
        // subtrees are written by other threads into their own ranges of the preallocated array.
        struct WideBuilder
        {
            const BinaryBuilder& bin;
            CollapsePlan& plan;
            std::vector<Node8> out;
            std::atomic<uint32_t> maxDepth{0};

            static void padBox(const Box& in, double lo[3], double hi[3])
            {
                float ext = 0.0f, mag = 0.0f;
                for (int k = 0; k < 3; k++)
                {
                    ext = std::max(ext, in.hi[k] - in.lo[k]);
                    mag = std::max(mag, std::max(std::fabs(in.lo[k]), std::fabs(in.hi[k])));
                }
                const double pad = 1e-5 * ext + 1e-7 * mag + 1e-30;
                for (int k = 0; k < 3; k++)
                {
                    lo[k] = static_cast<double>(in.lo[k]) - pad;
                    hi[k] = static_cast<double>(in.hi[k]) + pad;
                }
            }

            void emit(uint32_t bnode, uint32_t depth, uint32_t me)
            {
                uint32_t seen = maxDepth.load();
                while (seen < depth + 1 && !maxDepth.compare_exchange_weak(seen, depth + 1)) {}
                // children list
                std::vector<uint32_t> kids;
                std::vector<uint8_t> kidLeaf;
                plan.children(bnode, kids, kidLeaf);
                // slot assignment by octant
                Box nodeBox;
                for (uint32_t k : kids) nodeBox.grow(bin.nodes[k].box);
                float center[3];
                for (int a = 0; a < 3; a++) center[a] = 0.5f * (nodeBox.lo[a] + nodeBox.hi[a]);
                int slotOf[8];
                bool slotUsed[8] = {};
                bool kidUsed[8] = {};
                for (size_t round = 0; round < kids.size(); round++)
                {
                    float bestScore = -FLT_MAX;
                    int bk = -1, bs = -1;
                    for (size_t i = 0; i < kids.size(); i++)
                    {
                        if (kidUsed[i]) continue;
                        const Box& b = bin.nodes[kids[i]].box;
                        float v[3];
                        for (int a = 0; a < 3; a++) v[a] = 0.5f * (b.lo[a] + b.hi[a]) - center[a];
                        for (int s = 0; s < 8; s++)
                        {
                            if (slotUsed[s]) continue;
                            float score = ((s & 1) ? v[0] : -v[0]) + ((s & 2) ? v[1] : -v[1]) + ((s & 4) ? v[2] : -v[2]);
                            if (score > bestScore)
                            {
                                bestScore = score;
                                bk = static_cast<int>(i);
                                bs = s;
                            }
                        }
                    }
                    kidUsed[bk] = true;
                    slotUsed[bs] = true;
                    slotOf[bk] = bs;
                }
                // child references: inner children's subtrees follow this node in the order of the children list
                uint32_t childRef[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                uint8_t counts[8] = {};
                uint8_t innerMask = 0, leafMask = 0;
                uint32_t next = me + 1;
                std::vector<std::future<void>> futs;
                for (size_t i = 0; i < kids.size(); i++)
                {
                    const BNode& c = bin.nodes[kids[i]];
                    const int s = slotOf[i];
                    if (kidLeaf[i])
                    {
                        if (c.count > 255) throw std::runtime_error("BVH leaf larger than 255 triangles");
                        childRef[s] = c.first | (c.count << 24);  // first triangle (24 bits), count (8 bits)
                        counts[s] = static_cast<uint8_t>(c.count);
                        leafMask |= static_cast<uint8_t>(1u << s);
                    }
                    else
                    {
                        const uint32_t at = next, k = kids[i];
                        next += plan.wide[k];
                        childRef[s] = at;
                        innerMask |= static_cast<uint8_t>(1u << s);
                        std::future<void> fut;
                        if (plan.spawn_if_free(c.count, [this, k, depth, at] { emit(k, depth + 1, at); }, fut)) futs.push_back(std::move(fut));
                        else emit(k, depth + 1, at);
                    }
                }
                for (auto& f : futs) f.get();
                // quantisation
                double clo[8][3], chi[8][3];
                bool valid[8] = {};
                double plo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, phi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
                for (size_t i = 0; i < kids.size(); i++)
                {
                    const int s = slotOf[i];
                    padBox(bin.nodes[kids[i]].box, clo[s], chi[s]);
                    valid[s] = true;
                    for (int a = 0; a < 3; a++)
                    {
                        plo[a] = std::min(plo[a], clo[s][a]);
                        phi[a] = std::max(phi[a], chi[s][a]);
                    }
                }
                float p[3];
                int expo[3];
                uint8_t qlo[3][8], qhi[3][8];
                for (int a = 0; a < 3; a++)
                {
                    // origin rounded down to float
                    float pf = static_cast<float>(plo[a]);
                    if (static_cast<double>(pf) > plo[a]) pf = std::nextafter(pf, -FLT_MAX);
                    p[a] = pf;
                    const double ext = phi[a] - static_cast<double>(pf);
                    int e = -126;
                    if (ext > 0.0)
                    {
                        int fe;
                        std::frexp(ext / 255.0, &fe);  // ext/255 = m * 2^fe, m in [0.5, 1)
                        e = std::max(-126, std::min(127, fe));
                    }
                    for (;;)
                    {
                        const double scale = std::ldexp(1.0, e);
                        bool ok = true;
                        for (int s = 0; s < 8 && ok; s++)
                        {
                            if (!valid[s])
                            {
                                qlo[a][s] = 255;
                                qhi[a][s] = 0;
                                continue;
                            }
                            double ql = std::floor((clo[s][a] - pf) / scale);
                            double qh = std::ceil((chi[s][a] - pf) / scale);
                            ql = std::max(0.0, ql);
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
                        if (e > 127) throw std::runtime_error("BVH quantisation exponent overflow");
                    }
                    expo[a] = e;
                }
                Node8 node{};
                uint32_t header = static_cast<uint32_t>(expo[0] + 127) | (static_cast<uint32_t>(expo[1] + 127) << 8) |
                                  (static_cast<uint32_t>(expo[2] + 127) << 16) | (static_cast<uint32_t>(innerMask) << 24);
                uint32_t pb[3];
                std::memcpy(pb, p, sizeof(pb));
                node.w[0] = make_uint4(pb[0], pb[1], pb[2], header);
                auto pack8 = [](const uint8_t* q, uint32_t& lo, uint32_t& hi)
                {
                    lo = static_cast<uint32_t>(q[0]) | (static_cast<uint32_t>(q[1]) << 8) | (static_cast<uint32_t>(q[2]) << 16) | (static_cast<uint32_t>(q[3]) << 24);
                    hi = static_cast<uint32_t>(q[4]) | (static_cast<uint32_t>(q[5]) << 8) | (static_cast<uint32_t>(q[6]) << 16) | (static_cast<uint32_t>(q[7]) << 24);
                };
                uint32_t a0, a1, b0, b1;
                pack8(qlo[0], a0, a1);
                pack8(qlo[1], b0, b1);
                node.w[1] = make_uint4(a0, a1, b0, b1);
                pack8(qlo[2], a0, a1);
                pack8(qhi[0], b0, b1);
                node.w[2] = make_uint4(a0, a1, b0, b1);
                pack8(qhi[1], a0, a1);
                pack8(qhi[2], b0, b1);
                node.w[3] = make_uint4(a0, a1, b0, b1);
                node.w[4] = make_uint4(childRef[0], childRef[1], childRef[2], childRef[3]);
                node.w[5] = make_uint4(childRef[4], childRef[5], childRef[6], childRef[7]);
                pack8(counts, a0, a1);
                node.w[6] = make_uint4(a0, a1, leafMask, 0);
                node.w[7] = make_uint4(0, 0, 0, 0);
                out[me] = node;
            }
        };

        // The binary tree itself as 64-byte FP32 nodes in depth-first order (the plain format): each
        // node holds the boxes of its two children, padded like the BVH8's (WideBuilder::padBox) and
        // rounded outward to float, so the boxes contain their subtrees. A single-leaf root becomes a
        // node with one valid child.
        struct BinaryFlattener
        {
            const BinaryBuilder& bin;
            std::vector<Node2> out;
            uint32_t maxDepth = 0;

            static void outwardBox(const Box& b, float lo[3], float hi[3])
            {
                double dlo[3], dhi[3];
                WideBuilder::padBox(b, dlo, dhi);
                for (int k = 0; k < 3; k++)
                {
                    float l = static_cast<float>(dlo[k]);
                    if (static_cast<double>(l) > dlo[k]) l = std::nextafter(l, -FLT_MAX);
                    float h = static_cast<float>(dhi[k]);
                    if (static_cast<double>(h) < dhi[k]) h = std::nextafter(h, FLT_MAX);
                    lo[k] = l;
                    hi[k] = h;
                }
            }

            uint32_t emit(uint32_t bnode, uint32_t depth)
            {
                maxDepth = std::max(maxDepth, depth + 1);
                const uint32_t me = static_cast<uint32_t>(out.size());
                out.push_back(Node2{});
                const BNode& nd = bin.nodes[bnode];
                uint32_t kids[2] = {bnode, kInvalid};
                if (!nd.leaf())
                {
                    kids[0] = nd.left;
                    kids[1] = nd.right;
                }
                float lo[2][3], hi[2][3];
                uint32_t ref[2] = {0, 0}, count[2] = {0, 0}, leafMask = 0, validMask = 0;
                for (int i = 0; i < 2; i++)
                {
                    if (kids[i] == kInvalid)
                    {
                        for (int k = 0; k < 3; k++)
                        {
                            lo[i][k] = FLT_MAX;
                            hi[i][k] = -FLT_MAX;
                        }
                        continue;
                    }
                    const BNode& c = bin.nodes[kids[i]];
                    outwardBox(c.box, lo[i], hi[i]);
                    validMask |= 1u << i;
                    if (c.leaf())
                    {
                        if (c.count > 255) throw std::runtime_error("BVH leaf larger than 255 triangles");
                        ref[i] = c.first;
                        count[i] = c.count;
                        leafMask |= 1u << i;
                    }
                    else
                    {
                        ref[i] = emit(kids[i], depth + 1);
                    }
                }
                auto bits = [](float f)
                {
                    uint32_t u;
                    std::memcpy(&u, &f, 4);
                    return u;
                };
                Node2 node{};
                node.w[0] = make_uint4(bits(lo[0][0]), bits(lo[0][1]), bits(lo[0][2]), bits(hi[0][0]));
                node.w[1] = make_uint4(bits(hi[0][1]), bits(hi[0][2]), bits(lo[1][0]), bits(lo[1][1]));
                node.w[2] = make_uint4(bits(lo[1][2]), bits(hi[1][0]), bits(hi[1][1]), bits(hi[1][2]));
                node.w[3] = make_uint4(ref[0], ref[1], count[0] | (count[1] << 8) | (leafMask << 16) | (validMask << 24), 0u);
                out[me] = node;
                return me;
            }
        };
    }

    Bvh8 BuildBvh8(const float* positions, const uint32_t* models, uint32_t n, int threads, bool withBinary)
    {
        if (n == 0) throw std::runtime_error("scene has no triangles");
        if (n > kMaxTriangles) throw std::runtime_error("scene has more than 2^24 triangles");
        BinaryBuilder b;
        b.pos = positions;
        b.n = n;
        b.maxThreads = std::max(1, threads);
        b.triBox.resize(n);
        b.cent.resize(static_cast<size_t>(n) * 3);
        for_chunks((n + kChunk - 1) / kChunk, b.maxThreads, [&](uint32_t c)
        {
            for (uint32_t t = c * kChunk; t < std::min(n, (c + 1) * kChunk); t++)
            {
                Box box;
                for (int k = 0; k < 3; k++) box.grow(positions + (static_cast<size_t>(t) * 3 + k) * 3);
                b.triBox[t] = box;
                for (int a = 0; a < 3; a++) b.cent[static_cast<size_t>(t) * 3 + a] = 0.5f * (box.lo[a] + box.hi[a]);
            }
        });
        b.idx.resize(n);
        std::iota(b.idx.begin(), b.idx.end(), 0u);
        b.nodes.resize(static_cast<size_t>(n) * 2);
        const uint32_t root = b.build(0, n, 0);
        if (root != 0) throw std::runtime_error("BVH root index");
        CollapsePlan plan{b, {}, {}, {}, {}};
        plan.maxThreads = b.maxThreads;
        const size_t binaryNodes = b.nodeCount.load();
        plan.cost.assign(binaryNodes * 8, 0.0f);
        plan.how.assign(binaryNodes * 8, 0);
        plan.split.assign(binaryNodes, 1);
        plan.wide.assign(binaryNodes, 0);
        plan.plan(root);
        WideBuilder w{b, plan, {}};
        w.out.resize(plan.count_wide(root));
        w.emit(root, 0, 0);
        Bvh8 result;
        result.nodes = std::move(w.out);
        result.depth = w.maxDepth.load();
        if (withBinary)
        {
            BinaryFlattener f{b, {}, 0};
            f.out.reserve(b.nodeCount.load() / 2 + 1);
            f.emit(root, 0);
            result.nodes2 = std::move(f.out);
            result.depth2 = f.maxDepth;
        }
        result.order = b.idx;
        result.tris.assign(static_cast<size_t>(n) * kTriangleVec4, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        for (uint32_t j = 0; j < n; j++)
        {
            const uint32_t t = b.idx[j];
            const float* p0 = positions + (static_cast<size_t>(t) * 3 + 0) * 3;
            const float* p1 = positions + (static_cast<size_t>(t) * 3 + 1) * 3;
            const float* p2 = positions + (static_cast<size_t>(t) * 3 + 2) * 3;
            uint32_t ob = t, mb = models[t];
            float of, mf;
            std::memcpy(&of, &ob, 4);
            std::memcpy(&mf, &mb, 4);
            result.tris[static_cast<size_t>(j) * kTriangleVec4 + 0] = make_float4(p0[0], p0[1], p0[2], of);
            result.tris[static_cast<size_t>(j) * kTriangleVec4 + 1] = make_float4(p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2], mf);
            result.tris[static_cast<size_t>(j) * kTriangleVec4 + 2] = make_float4(p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2], 0.0f);
        }
        return result;
    }
}

namespace pt
{
    namespace
    {
        struct CheckState
        {
            const Bvh8& b;
            const float* positions;
            std::vector<uint32_t> seen;
            uint64_t violations = 0;
            uint64_t leafTriangles = 0;
        };

        // Exact bounds of a subtree; checks each quantised child box against its subtree.
        void check_node(CheckState& cs, uint32_t node, double lo[3], double hi[3])
        {
            const Node8& n = cs.b.nodes[node];
            float p[3];
            std::memcpy(p, &n.w[0], 12);
            const uint32_t header = n.w[0].w;
            const uint32_t innerMask = header >> 24;
            const uint32_t leafMask = n.w[6].z & 0xFFu;
            const uint32_t* child = reinterpret_cast<const uint32_t*>(&n.w[4]);
            const uint8_t* counts = reinterpret_cast<const uint8_t*>(&n.w[6]);
            const uint8_t* q = reinterpret_cast<const uint8_t*>(&n.w[1]);  // qlo x,y,z then qhi x,y,z, 8 each
            for (int k = 0; k < 3; k++)
            {
                lo[k] = DBL_MAX;
                hi[k] = -DBL_MAX;
            }
            for (int s = 0; s < 8; s++)
            {
                const bool isInner = (innerMask >> s) & 1u, isLeaf = (leafMask >> s) & 1u;
                if (!isInner && !isLeaf) continue;
                double clo[3], chi[3];
                if (isInner)
                    check_node(cs, child[s], clo, chi);
                else
                {
                    for (int k = 0; k < 3; k++)
                    {
                        clo[k] = DBL_MAX;
                        chi[k] = -DBL_MAX;
                    }
                    if ((child[s] >> 24) != counts[s]) cs.violations++;
                    for (uint32_t j = 0; j < counts[s]; j++)
                    {
                        const uint32_t t = cs.b.order[(child[s] & 0xFFFFFFu) + j];
                        cs.seen[t]++;
                        cs.leafTriangles++;
                        for (int v = 0; v < 3; v++)
                            for (int k = 0; k < 3; k++)
                            {
                                const double c = cs.positions[(static_cast<size_t>(t) * 3 + v) * 3 + k];
                                clo[k] = std::min(clo[k], c);
                                chi[k] = std::max(chi[k], c);
                            }
                    }
                }
                for (int k = 0; k < 3; k++)
                {
                    const int e = static_cast<int>((header >> (8 * k)) & 0xFFu) - 127;
                    const double scale = std::ldexp(1.0, e);
                    const double qlo = q[k * 8 + s], qhi = q[24 + k * 8 + s];
                    const double blo = static_cast<double>(p[k]) + qlo * scale;
                    const double bhi = static_cast<double>(p[k]) + qhi * scale;
                    if (!(blo <= clo[k] && bhi >= chi[k])) cs.violations++;
                    lo[k] = std::min(lo[k], clo[k]);
                    hi[k] = std::max(hi[k], chi[k]);
                }
            }
        }

        // Same for the binary FP32 tree: each child box (exact float values) must contain its subtree.
        void check_binary(CheckState& cs, uint32_t node, double lo[3], double hi[3])
        {
            const Node2& n = cs.b.nodes2[node];
            float f[12];
            std::memcpy(f, &n.w[0], 48);  // lo0 xyz, hi0 xyz, lo1 xyz, hi1 xyz
            const uint32_t meta = n.w[3].z;
            const uint32_t ref[2] = {n.w[3].x, n.w[3].y};
            for (int k = 0; k < 3; k++)
            {
                lo[k] = DBL_MAX;
                hi[k] = -DBL_MAX;
            }
            for (int c = 0; c < 2; c++)
            {
                if (!((meta >> (24 + c)) & 1u)) continue;
                double clo[3], chi[3];
                if ((meta >> (16 + c)) & 1u)
                {
                    for (int k = 0; k < 3; k++)
                    {
                        clo[k] = DBL_MAX;
                        chi[k] = -DBL_MAX;
                    }
                    const uint32_t count = (meta >> (8 * c)) & 0xFFu;
                    for (uint32_t j = 0; j < count; j++)
                    {
                        const uint32_t t = cs.b.order[ref[c] + j];
                        cs.seen[t]++;
                        cs.leafTriangles++;
                        for (int v = 0; v < 3; v++)
                            for (int k = 0; k < 3; k++)
                            {
                                const double x = cs.positions[(static_cast<size_t>(t) * 3 + v) * 3 + k];
                                clo[k] = std::min(clo[k], x);
                                chi[k] = std::max(chi[k], x);
                            }
                    }
                }
                else
                    check_binary(cs, ref[c], clo, chi);
                for (int k = 0; k < 3; k++)
                {
                    if (!(static_cast<double>(f[c * 6 + k]) <= clo[k] && static_cast<double>(f[c * 6 + 3 + k]) >= chi[k])) cs.violations++;
                    lo[k] = std::min(lo[k], clo[k]);
                    hi[k] = std::max(hi[k], chi[k]);
                }
            }
        }
    }

    Bvh8Check CheckBvh8(const Bvh8& b, const float* positions, uint32_t n)
    {
        CheckState cs{b, positions, std::vector<uint32_t>(n, 0)};
        double lo[3], hi[3];
        check_node(cs, 0, lo, hi);
        Bvh8Check r;
        r.containmentViolations = cs.violations;
        r.leafTriangles = cs.leafTriangles;
        r.trianglesNotExactlyOnce = 0;
        for (uint32_t t = 0; t < n; t++)
            if (cs.seen[t] != 1) r.trianglesNotExactlyOnce++;
        if (!b.nodes2.empty())
        {
            CheckState bs{b, positions, std::vector<uint32_t>(n, 0)};
            check_binary(bs, 0, lo, hi);
            r.containmentViolations += bs.violations;
            for (uint32_t t = 0; t < n; t++)
                if (bs.seen[t] != 1) r.trianglesNotExactlyOnce++;
        }
        return r;
    }
}
