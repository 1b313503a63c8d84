// ORACLE — test infrastructure only.
//
// A CPU restatement of KrzystekMatej/gpu-path-tracer's CUDA wavefront path
// tracer, used by tests/ (as the parity checker) and by bench.py (as the timed
// CPU baseline). It is never linked into, called by, or shipped with the
// product library. Every function cites the reference file:line it follows;
// all paths are relative to the reference project root.
//
// Deviations from the reference, each deliberate and shared with the GPU product:
//  * Transcendentals follow the deterministic specification in
//    oracle_detmath.h instead of CUDA's sinf/cosf/powf/rsqrtf.
//  * Closest-hit ties (two triangles at bit-identical t) resolve to the smaller
//    ORIGINAL triangle index; the reference keeps the first one its DFS visits
//    (Intersect.cu:60,110-111), which depends on the BVH.
//  * Hit triangle ids are reported in the caller's input order, not in the
//    reference's BVH-permuted order (HostBvh.cpp:90-96, Intersect.cu:101).
//  * Materials are constant per material: the decoded texel values a 1x1 CUDA
//    texture would return are passed in directly (Manager.cpp:321-380,
//    TextureView.hpp:17-20).
//  * Radiance is accumulated per path (per sample) and summed per pixel in
//    sample order after the frame, instead of float atomics per contribution
//    (Kernels/Common.hpp:8-16). At spp = 1 the two are identical.
//
// Production modes of the product that the reference does not have (restated here
// from the product's definition, so the checker covers them too):
//  * RNG policy PCG32: PCG-XSH-RR 64/32 (O'Neill 2014) per sample, seeded by a
//    splitmix64 hash of (seed, sample key) and positioned by LCG jump-ahead.
//  * Power-weighted light selection: weights area x luminance(emission) in FP64, the
//    alias table built by the parallel sweep; the prefix sums are taken in the
//    product's device order (its block scan), so the table is bit-for-bit the same.
//
// Compile with -ffp-contract=off (see oracle/Makefile): no FMA contraction.
#include "oracle_detmath.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

namespace oracle
{
    // ------------------------------------------------------------------
    // Vector algebra, restating External/cuda-samples/Common/helper_math.h
    // (operator order kept: e.g. dot = a.x*b.x + a.y*b.y + a.z*b.z, :1264).
    // ------------------------------------------------------------------
    struct float2 { float x, y; };
    struct float3 { float x, y, z; };
    struct float4 { float x, y, z, w; };

    inline float2 make_float2(float x, float y) { return {x, y}; }
    inline float3 make_float3(float x, float y, float z) { return {x, y, z}; }
    inline float3 make_float3(float s) { return {s, s, s}; }
    inline float3 make_float3(float4 a) { return {a.x, a.y, a.z}; }
    inline float4 make_float4(float x, float y, float z, float w) { return {x, y, z, w}; }

    inline float3 operator+(float3 a, float3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
    inline float3 operator-(float3 a, float3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    inline float3 operator*(float3 a, float3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
    inline float3 operator/(float3 a, float3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
    inline float3 operator*(float3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
    inline float3 operator*(float b, float3 a) { return {b * a.x, b * a.y, b * a.z}; }
    inline float3 operator/(float3 a, float b) { return {a.x / b, a.y / b, a.z / b}; }
    inline float3 operator+(float3 a, float b) { return {a.x + b, a.y + b, a.z + b}; }
    inline float3 operator-(float3 a, float b) { return {a.x - b, a.y - b, a.z - b}; }
    inline float3 operator-(float b, float3 a) { return {b - a.x, b - a.y, b - a.z}; }
    inline float3 operator-(float3 a) { return {-a.x, -a.y, -a.z}; }
    inline float2 operator+(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
    inline float2 operator*(float b, float2 a) { return {b * a.x, b * a.y}; }
    inline float4 operator+(float4 a, float4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
    inline float4 operator*(float b, float4 a) { return {b * a.x, b * a.y, b * a.z, b * a.w}; }

    inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
    inline float3 cross(float3 a, float3 b)
    {
        return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    }
    inline float length(float3 v) { return std::sqrt(dot(v, v)); }
    inline float3 normalize(float3 v)
    {
        float invLen = dm_rsqrt(dot(v, v));
        return v * invLen;
    }
    inline float3 reflect(float3 i, float3 n) { return i - 2.0f * n * dot(n, i); }
    inline float3 fminf3(float3 a, float3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
    inline float3 fmaxf3(float3 a, float3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
    inline float clampf(float f, float a, float b) { return std::fmax(a, std::fmin(f, b)); }
    inline float lerpf(float a, float b, float t) { return a + t * (b - a); }
    inline float3 lerp3(float3 a, float3 b, float t) { return a + t * (b - a); }
    inline float MinComponent(float3 v) { return std::fmin(v.x, std::fmin(v.y, v.z)); }
    inline float MaxComponent(float3 v) { return std::fmax(v.x, std::fmax(v.y, v.z)); }
    inline float Sqr(float v) { return v * v; }

    // Core/Include/Core/Graphics/Cuda/Utils/Math.hpp:8-11 and math_constants.h
    constexpr float PiF = 3.141592654f;
    constexpr float InvPi = 1.0f / PiF;
    constexpr float TwoPi = 2.0f * PiF;
    constexpr float InvTwoPi = 1.0f / TwoPi;
    constexpr float OneMinusEpsilon = 0x1.fffffep-1f;

    // PathTracerDefaults.hpp:9-35
    constexpr uint32_t RussianRouletteStartDepth = 3;
    constexpr uint32_t InvalidIndex = 0xFFFFFFFFu;
    constexpr float MinT = 1e-4f;
    constexpr float MaxT = 1e34f;
    constexpr uint64_t RandomSeed = 1234;
    // Common/Material.hpp:187-195
    constexpr float MinShininess = 1.0f;
    constexpr float MaxShininess = 1000.0f;
    constexpr float DefaultIor = 1.0f;

    // Math.hpp:91-148
    struct Frame
    {
        float3 tangent, bitangent, normal;
        float3 ToLocal(float3 d) const { return make_float3(dot(d, tangent), dot(d, bitangent), dot(d, normal)); }
        float3 FromLocal(float3 d) const { return d.x * tangent + d.y * bitangent + d.z * normal; }
    };

    inline float3 SafeNormalize(float3 v, float3 fallback)
    {
        float lengthSquared = dot(v, v);
        if (lengthSquared > 1e-16f)
            return v * dm_rsqrt(lengthSquared);
        return fallback;
    }

    inline Frame BuildFrame(float3 normal)
    {
        float3 tangent;
        if (std::fabs(normal.x) > std::fabs(normal.z))
            tangent = normalize(make_float3(normal.y, -normal.x, 0.0f));
        else
            tangent = normalize(make_float3(0.0f, normal.z, -normal.y));
        float3 bitangent = cross(normal, tangent);
        return Frame{tangent, bitangent, normal};
    }

    inline Frame BuildFrame(float3 normal, float3 tangent, float tangentSign)
    {
        normal = SafeNormalize(normal, make_float3(0.0f, 0.0f, 1.0f));
        Frame fallback = BuildFrame(normal);
        tangent = tangent - normal * dot(normal, tangent);
        tangent = SafeNormalize(tangent, fallback.tangent);
        float3 bitangent = cross(normal, tangent) * tangentSign;
        return Frame{tangent, bitangent, normal};
    }

    // Math.hpp:217-262
    inline float CosTheta(float3 w) { return w.z; }
    inline float Cos2Theta(float3 w) { return w.z * w.z; }
    inline float AbsCosTheta(float3 w) { return std::fabs(w.z); }
    inline float Sin2Theta(float3 w) { return std::fmax(0.0f, 1.0f - Cos2Theta(w)); }
    inline float SinTheta(float3 w) { return std::sqrt(Sin2Theta(w)); }
    inline float Tan2Theta(float3 w) { return Sin2Theta(w) / Cos2Theta(w); }
    inline float CosPhi(float3 w)
    {
        float sinTheta = SinTheta(w);
        return (sinTheta == 0) ? 1 : clampf(w.x / sinTheta, -1.f, 1.f);
    }
    inline float SinPhi(float3 w)
    {
        float sinTheta = SinTheta(w);
        return (sinTheta == 0) ? 0 : clampf(w.y / sinTheta, -1.f, 1.f);
    }

    // ------------------------------------------------------------------
    // Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel Random Numbers: As
    // Easy as 1, 2, 3", SC'11), arranged as the counter stream the reference
    // draws from through cuRAND (PathData.hpp:37-73; curand_init(1234,
    // sampleIndex, 0) at PathGeneration.cu:66,93). Key = 64-bit seed; counter =
    // (position / 4 as 64 bits, subsequence as 64 bits); the stream is the
    // sequence of 32-bit words; a uniform is u * 2^-32 + 2^-33 in (0, 1].
    // The GPU parity tests pin this against device curand output.
    // ------------------------------------------------------------------
    struct PhiloxBlock { uint32_t v[4]; };

    inline PhiloxBlock Philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
    {
        const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
        const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
        for (int round = 0; round < 10; round++)
        {
            uint64_t p0 = static_cast<uint64_t>(M0) * c0;
            uint64_t p1 = static_cast<uint64_t>(M1) * c2;
            uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
            uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
            uint32_t n0 = hi1 ^ c1 ^ k0;
            uint32_t n1 = lo1;
            uint32_t n2 = hi0 ^ c3 ^ k1;
            uint32_t n3 = lo0;
            c0 = n0; c1 = n1; c2 = n2; c3 = n3;
            k0 += W0;
            k1 += W1;
        }
        return PhiloxBlock{{c0, c1, c2, c3}};
    }

    // ------------------------------------------------------------------
    // PCG32 (PCG-XSH-RR, 64-bit state; O'Neill, "PCG: A Family of Simple Fast
    // Space-Efficient Statistically Good Algorithms for Random Number Generation",
    // 2014): the product's second RNG policy. One stream per sample: seeded by a
    // splitmix64 hash (Steele, Lea, Flood, OOPSLA 2014) of (seed, key), key = the
    // sample index plus the shard offset, positioned by LCG jump-ahead (Brown 1994).
    // ------------------------------------------------------------------
    enum RngPolicy : uint32_t { RngPhilox = 0, RngPcg32 = 1 };

    inline uint64_t Mix64(uint64_t z)
    {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }

    struct Pcg32
    {
        static constexpr uint64_t Multiplier = 6364136223846793005ull;
        uint64_t state = 0, inc = 1;
        uint32_t Next()
        {
            const uint64_t old = state;
            state = old * Multiplier + inc;
            const uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
            const uint32_t rot = static_cast<uint32_t>(old >> 59u);
            return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
        }
        void Seed(uint64_t initstate, uint64_t initseq)
        {
            state = 0;
            inc = (initseq << 1u) | 1u;
            Next();
            state += initstate;
            Next();
        }
        void Advance(uint64_t delta)
        {
            uint64_t accMult = 1, accPlus = 0, curMult = Multiplier, curPlus = inc;
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
        static Pcg32 ForKey(uint64_t key)
        {
            Pcg32 g;
            g.Seed(Mix64(RandomSeed ^ Mix64(key)), Mix64(key ^ 0x9E3779B97F4A7C15ull));
            return g;
        }
    };

    struct Random
    {
        uint64_t subsequence;
        uint64_t position;
        uint32_t policy = RngPhilox;

        uint32_t Word(uint64_t pos) const
        {
            if (policy == RngPcg32)
            {
                Pcg32 g = Pcg32::ForKey(subsequence);
                g.Advance(pos);
                return g.Next();
            }
            uint64_t block = pos >> 2;
            PhiloxBlock b = Philox4x32_10(
                static_cast<uint32_t>(block), static_cast<uint32_t>(block >> 32),
                static_cast<uint32_t>(subsequence), static_cast<uint32_t>(subsequence >> 32),
                static_cast<uint32_t>(RandomSeed), static_cast<uint32_t>(RandomSeed >> 32));
            return b.v[pos & 3];
        }
        static float ToUniform(uint32_t u)
        {
            const float inv2pow32 = 2.3283064e-10f;
            return static_cast<float>(u) * inv2pow32 + (inv2pow32 / 2.0f);
        }
        // PCG32 uniforms: the top 24 bits, centred: (w >> 8) 2^-24 + 2^-25, in (0, 1]
        static float ToUniformPcg(uint32_t u) { return static_cast<float>(u >> 8) * 0x1p-24f + 0x1p-25f; }
        float Uniform(uint64_t pos) const { return policy == RngPcg32 ? ToUniformPcg(Word(pos)) : ToUniform(Word(pos)); }
        float NextFloat() { return Uniform(position++); }
        float4 NextFloat4()
        {
            float4 r{Uniform(position), Uniform(position + 1), Uniform(position + 2), Uniform(position + 3)};
            position += 4;
            return r;
        }
        float2 NextFloat2() { float4 v = NextFloat4(); return make_float2(v.x, v.y); }
        float3 NextFloat3() { float4 v = NextFloat4(); return make_float3(v.x, v.y, v.z); }
    };

    // ------------------------------------------------------------------
    // Scene records (Triangle.hpp:8-58, Renderer.cpp:144-213, Material.hpp:73-87)
    // ------------------------------------------------------------------
    enum Model : uint32_t { ModelNormal = 0, ModelDiffuse, ModelMirror, ModelPhong, ModelGgx, ModelEmissive, ModelCount };

    struct MaterialRecord // 20 words; identical layout to gpt_material in the product C-ABI
    {
        uint32_t model;
        float color[3];
        float specular[3];
        float shininess;     // normalised texel in [0, 1]
        float rma[3];
        float emission[3];
        float normal[3];     // tangent-space normal-map texel in [0, 1]
        float ior;
        float transmission;
        float pad;
    };
    static_assert(sizeof(MaterialRecord) == 80, "material record layout");

    struct TriangleIntersection { float3 edge1, edge2, v0; uint32_t model; };
    struct TriangleShading
    {
        float4 normals[3];
        float4 tangents[3];
        float3 geometricNormal;
        uint32_t material;
        float2 uvs[3];
    };
    struct LightTriangle
    {
        float3 edge1, edge2, v0;
        uint32_t index;
        float3 geometricNormal;
        float area;
        float3 emission;
    };
    struct Bin { float q, p; uint32_t alias, value; };

    struct Scene
    {
        uint32_t triangleCount = 0;
        std::vector<float3> positions;          // 3 per triangle
        std::vector<TriangleIntersection> isect; // original order
        std::vector<TriangleShading> shading;    // original order
        std::vector<MaterialRecord> materials;
        std::vector<uint32_t> materialCounts;    // per model, Renderer.cpp:90
        // reference BVH (HostBvh.cpp, DeviceBvh.cpp:7-19)
        struct Node { float3 bmin, bmax; uint32_t left, right, first, count; };
        std::vector<Node> nodes;
        std::vector<uint32_t> order;             // BVH position -> original triangle index
        std::vector<TriangleIntersection> bvhIsect; // BVH order
        uint32_t bvhDepth = 0;
        // lights (LightSampler.cpp:5-40) and alias table (AliasTable.hpp:22-84)
        std::vector<LightTriangle> lights;
        std::vector<Bin> bins;
        std::vector<Bin> binsPower;  // the product's power-weighted table
    };

    // ------------------------------------------------------------------
    // Alias table, AliasTable.hpp:22-84 (sequential Vose with LIFO stacks)
    // ------------------------------------------------------------------
    inline std::vector<Bin> BuildAliasTable(const std::vector<float>& weights, const std::vector<uint32_t>& values)
    {
        float sum = static_cast<float>(std::accumulate(weights.begin(), weights.end(), 0.0));
        std::vector<Bin> bins(weights.size());
        for (uint32_t i = 0; i < weights.size(); i++)
            bins[i] = Bin{0.0f, weights[i] / sum, 0u, values[i]};
        struct Outcome { float pHat; uint32_t index; };
        std::vector<Outcome> under, over;
        for (uint32_t i = 0; i < bins.size(); i++)
        {
            float pHat = bins[i].p * bins.size();
            if (pHat < 1)
                under.push_back(Outcome{pHat, i});
            else
                over.push_back(Outcome{pHat, i});
        }
        while (!under.empty() && !over.empty())
        {
            Outcome un = under.back(), ov = over.back();
            under.pop_back();
            over.pop_back();
            bins[un.index].q = un.pHat;
            bins[un.index].alias = ov.index;
            float pExcess = un.pHat + ov.pHat - 1;
            if (pExcess < 1)
                under.push_back(Outcome{pExcess, ov.index});
            else
                over.push_back(Outcome{pExcess, ov.index});
        }
        while (!over.empty())
        {
            Outcome ov = over.back();
            over.pop_back();
            bins[ov.index].q = 1;
            bins[ov.index].alias = InvalidIndex;
        }
        while (!under.empty())
        {
            Outcome un = under.back();
            under.pop_back();
            bins[un.index].q = 1;
            bins[un.index].alias = InvalidIndex;
        }
        return bins;
    }

    // AliasTableView.hpp:32-60 (returns the outcome index and its pmf)
    inline void SampleAlias(const std::vector<Bin>& bins, float u, uint32_t* outIndex, float* outPmf)
    {
        const uint32_t size = static_cast<uint32_t>(bins.size());
        const float scaledU = u * static_cast<float>(size);
        const uint32_t binIndex = std::min(static_cast<uint32_t>(scaledU), size - 1u);
        const float up = std::fmin(scaledU - static_cast<float>(binIndex), OneMinusEpsilon);
        const Bin& bin = bins[binIndex];
        if (up < bin.q)
        {
            *outIndex = binIndex;
            *outPmf = bin.p;
            return;
        }
        *outIndex = bin.alias;
        *outPmf = bins[bin.alias].p;
    }

    // ------------------------------------------------------------------
    // Power-weighted alias table of the product (no counterpart in the reference).
    // ------------------------------------------------------------------
    // Exclusive prefix sum in the product's device order (its block scan over 1024-element
    // blocks): Hillis-Steele inclusive scan within each 32-lane warp (a lane adds the value
    // of the lane o below it, o = 1, 2, 4, 8, 16), the same over the 32 warp totals, then
    // exclusive = (lane value + warp offset) - x; block totals scanned recursively the same
    // way and added to every later block.
    template <typename T>
    inline void DeviceOrderExclusiveScan(const T* in, T* out, size_t n)
    {
        if (n == 0) return;
        const size_t blocks = (n + 1023) / 1024;
        std::vector<T> sums(blocks);
        std::vector<T> x(1024), v(1024), prev(1024);
        for (size_t blk = 0; blk < blocks; blk++)
        {
            for (size_t t = 0; t < 1024; t++)
            {
                const size_t i = blk * 1024 + t;
                x[t] = i < n ? in[i] : T(0);
                v[t] = x[t];
            }
            for (size_t o = 1; o < 32; o <<= 1)
            {
                prev = v;
                for (size_t t = 0; t < 1024; t++)
                    if ((t & 31) >= o) v[t] = prev[t] + prev[t - o];
            }
            T ws[32], wprev[32];
            for (size_t w = 0; w < 32; w++) ws[w] = v[w * 32 + 31];
            for (size_t o = 1; o < 32; o <<= 1)
            {
                std::copy(ws, ws + 32, wprev);
                for (size_t l = o; l < 32; l++) ws[l] = wprev[l] + wprev[l - o];
            }
            T last = T(0);
            for (size_t t = 0; t < 1024; t++)
            {
                const size_t w = t >> 5;
                const T warpOffset = w > 0 ? ws[w - 1] : T(0);
                const T inclusive = v[t] + warpOffset;
                const size_t i = blk * 1024 + t;
                if (i < n) out[i] = inclusive - x[t];
                last = inclusive;
            }
            sums[blk] = last;
        }
        if (blocks == 1) return;
        DeviceOrderExclusiveScan(sums.data(), sums.data(), blocks);
        for (size_t blk = 1; blk < blocks; blk++)
            for (size_t t = 0; t < 1024; t++)
            {
                const size_t i = blk * 1024 + t;
                if (i < n) out[i] = out[i] + sums[blk];
            }
    }

    // The product's parallel sweep (scene-upload alias_*_kernel): classify by pHat = w n / W,
    // prefix sums of deficits (lights) and excesses (heavies) in input order with zeros for the other
    // class, running maxima over both, then the merge of the keys D_i (lights) and E_(j+1) (heavies,
    // first on ties), here run sequentially. Area weights replace power weights whose sum is not positive.
    inline std::vector<Bin> BuildPowerAliasTable(const std::vector<double>& power, const std::vector<double>& area)
    {
        const size_t n = power.size();
        std::vector<Bin> bins(n);
        if (n == 0) return bins;
        std::vector<double> prefix(n), areaPrefix(n);
        DeviceOrderExclusiveScan(power.data(), prefix.data(), n);
        DeviceOrderExclusiveScan(area.data(), areaPrefix.data(), n);
        const double totalPower = prefix[n - 1] + power[n - 1];
        const bool usePower = totalPower > 0.0 && totalPower < 1e300;
        const std::vector<double>& w = usePower ? power : area;
        const double total = usePower ? totalPower : areaPrefix[n - 1] + area[n - 1];
        std::vector<double> pHat(n), deficit(n), excess(n), dp(n), ep(n);
        std::vector<uint32_t> lightIdx, heavyIdx;
        for (size_t k = 0; k < n; k++)
        {
            const double ph = w[k] * static_cast<double>(n) / total;
            const bool light = ph < 1.0;
            pHat[k] = ph;
            deficit[k] = light ? 1.0 - ph : 0.0;
            excess[k] = light ? 0.0 : ph - 1.0;
            (light ? lightIdx : heavyIdx).push_back(static_cast<uint32_t>(k));
            bins[k] = Bin{1.0f, static_cast<float>(w[k] / total), InvalidIndex, static_cast<uint32_t>(k)};
        }
        DeviceOrderExclusiveScan(deficit.data(), dp.data(), n);
        DeviceOrderExclusiveScan(excess.data(), ep.data(), n);
        for (size_t k = 1; k < n; k++)
        {
            dp[k] = std::fmax(dp[k], dp[k - 1]);
            ep[k] = std::fmax(ep[k], ep[k - 1]);
        }
        const size_t a = lightIdx.size(), b = heavyIdx.size();
        const double deficitTotal = dp[n - 1] + deficit[n - 1];
        const double excessTotal = ep[n - 1] + excess[n - 1];
        auto D = [&](size_t i) { return i < a ? dp[lightIdx[i]] : deficitTotal; };
        auto E = [&](size_t j) { return j < b ? ep[heavyIdx[j]] : excessTotal; };
        size_t i = 0, j = 0;
        for (size_t k = 0; k < n; k++)
        {
            if (i < a && (j >= b || D(i) < E(j + 1)))
            {
                const uint32_t item = lightIdx[i];
                if (j < b)
                {
                    bins[item].q = static_cast<float>(pHat[item]);
                    bins[item].alias = heavyIdx[j];
                }
                i++;
            }
            else
            {
                const uint32_t item = heavyIdx[j];
                if (j + 1 < b)
                {
                    const double residual = E(j + 1) - D(i) + 1.0;
                    bins[item].q = static_cast<float>(residual < 0.0 ? 0.0 : (residual > 1.0 ? 1.0 : residual));
                    bins[item].alias = heavyIdx[j + 1];
                }
                j++;
            }
        }
        return bins;
    }

    // ------------------------------------------------------------------
    // Reference BVH: HostBvh.cpp:22-100 and DeviceBvh.cpp:7-19
    // ------------------------------------------------------------------
    struct BvhBuilder
    {
        const Scene& scene;
        std::vector<uint32_t>& order;
        std::vector<Scene::Node>& nodes;
        uint32_t maxDepth = 0, minTriangles = 0, depthReached = 0;

        struct HostNode { std::unique_ptr<HostNode> left, right; uint32_t first = 0, count = 0; float3 bmin, bmax; };

        static uint32_t EstimateMaxTrianglesPerLeaf(size_t n)
        {
            if (n < 5'000) return 4;
            if (n < 50'000) return 6;
            if (n < 500'000) return 8;
            if (n < 2'000'000) return 12;
            if (n < 10'000'000) return 16;
            return 24;
        }
        static uint32_t EstimateMaxDepth(size_t n)
        {
            return std::min(64u, static_cast<uint32_t>(std::max(1.0, std::ceil(2 * std::log2(n)))));
        }

        std::unique_ptr<HostNode> BuildRecurse(uint32_t first, uint32_t count, uint32_t depth)
        {
            depthReached = std::max(depthReached, depth);
            auto node = std::make_unique<HostNode>();
            node->first = first;
            node->count = count;
            float3 bmin = make_float3(FLT_MAX), bmax = make_float3(-FLT_MAX);
            for (uint32_t i = first; i < first + count; i++)
                for (int k = 0; k < 3; k++)
                {
                    const float3& p = scene.positions[order[i] * 3 + k];
                    bmin = make_float3(std::min(bmin.x, p.x), std::min(bmin.y, p.y), std::min(bmin.z, p.z));
                    bmax = make_float3(std::max(bmax.x, p.x), std::max(bmax.y, p.y), std::max(bmax.z, p.z));
                }
            if (count == 0)
            {
                node->bmin = make_float3(FLT_MAX);
                node->bmax = make_float3(-FLT_MAX);
            }
            else
            {
                // PadBounds, HostBvh.cpp:37-48
                const float3 extent = bmax - bmin;
                const float largestExtent = std::fmax(extent.x, std::fmax(extent.y, extent.z));
                const float padding = std::fmax(1e-5f * largestExtent, 1e-5f);
                node->bmin = bmin - make_float3(padding, padding, padding);
                node->bmax = bmax + make_float3(padding, padding, padding);
            }
            if (depth >= maxDepth || count <= minTriangles)
                return node;
            uint32_t axis = 0;
            float extentX = bmax.x - bmin.x, extentY = bmax.y - bmin.y, extentZ = bmax.z - bmin.z;
            if (extentY > extentX && extentY > extentZ)
                axis = 1;
            else if (extentZ > extentX && extentZ > extentY)
                axis = 2;
            uint32_t mid = first + (count / 2);
            const std::vector<float3>& pos = scene.positions;
            std::nth_element(order.begin() + first, order.begin() + mid, order.begin() + first + count,
                [axis, &pos](uint32_t a, uint32_t b)
                {
                    float3 centerA = (pos[a * 3 + 0] + pos[a * 3 + 1] + pos[a * 3 + 2]) / 3.0f;
                    float3 centerB = (pos[b * 3 + 0] + pos[b * 3 + 1] + pos[b * 3 + 2]) / 3.0f;
                    float ca = axis == 0 ? centerA.x : (axis == 1 ? centerA.y : centerA.z);
                    float cb = axis == 0 ? centerB.x : (axis == 1 ? centerB.y : centerB.z);
                    return ca < cb;
                });
            node->left = BuildRecurse(first, mid - first, depth + 1);
            node->right = BuildRecurse(mid, count - (mid - first), depth + 1);
            return node;
        }

        uint32_t Flatten(const HostNode& node)
        {
            uint32_t index = static_cast<uint32_t>(nodes.size());
            nodes.push_back(Scene::Node{node.bmin, node.bmax, InvalidIndex, InvalidIndex, node.first, node.count});
            if (node.left && node.right)
            {
                uint32_t l = Flatten(*node.left);
                nodes[index].left = l;
                uint32_t r = Flatten(*node.right);
                nodes[index].right = r;
            }
            return index;
        }
    };

    // ------------------------------------------------------------------
    // Traversal: Intersect.cu:11-61 (slab test, Moller-Trumbore) and :63-179
    // ------------------------------------------------------------------
    struct Ray { float3 origin, direction; float tMin, tMax; };
    struct Hit { uint32_t triangle; float u, v; uint32_t model; };

    inline bool AabbIntersect(const Scene::Node& n, const Ray& ray, float3 invDirection)
    {
        const float3 tNear = (n.bmin - ray.origin) * invDirection;
        const float3 tFar = (n.bmax - ray.origin) * invDirection;
        const float3 low = fminf3(tNear, tFar);
        const float3 high = fmaxf3(tNear, tFar);
        const float t0 = std::fmax(ray.tMin, MaxComponent(low));
        const float t1 = std::fmin(ray.tMax, MinComponent(high));
        return t0 <= t1;
    }

    // Returns the Moller-Trumbore t, u, v if the barycentric and determinant tests
    // pass (Intersect.cu:25-59); the caller applies the t-range test (:60).
    inline bool IntersectTriangleUvt(const TriangleIntersection& tri, const Ray& ray, float& t, float& u, float& v)
    {
        const float3 p = cross(ray.direction, tri.edge2);
        const float det = dot(tri.edge1, p);
        const float epsilon = 1e-7f;
        if (std::fabs(det) < epsilon)
            return false;
        const float invDet = 1.0f / det;
        const float3 s = ray.origin - tri.v0;
        u = dot(s, p) * invDet;
        if (u < 0.0f || u > 1.0f)
            return false;
        const float3 q = cross(s, tri.edge1);
        v = dot(ray.direction, q) * invDet;
        if (v < 0.0f || u + v > 1.0f)
            return false;
        t = dot(tri.edge2, q) * invDet;
        return true;
    }

    inline bool TraceClosest(const Scene& scene, Ray& ray, Hit& hit)
    {
        hit = Hit{InvalidIndex, 0.0f, 0.0f, ModelCount};
        const float3 invDirection = make_float3(1.0f) / ray.direction;
        uint32_t stack[80];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0)
        {
            const Scene::Node& node = scene.nodes[stack[--sp]];
            if (!AabbIntersect(node, ray, invDirection))
                continue;
            if (node.left == InvalidIndex && node.right == InvalidIndex)
            {
                for (uint32_t i = 0; i < node.count; i++)
                {
                    const TriangleIntersection& tri = scene.bvhIsect[node.first + i];
                    float t, u, v;
                    if (!IntersectTriangleUvt(tri, ray, t, u, v))
                        continue;
                    if (!(t >= ray.tMin))
                        continue;
                    const uint32_t original = scene.order[node.first + i];
                    bool better = t < ray.tMax ||
                                  (t == ray.tMax && hit.triangle != InvalidIndex && original < hit.triangle);
                    if (better)
                    {
                        ray.tMax = t;
                        hit = Hit{original, u, v, tri.model};
                    }
                }
            }
            else
            {
                stack[sp++] = node.left;
                stack[sp++] = node.right;
            }
        }
        return hit.triangle != InvalidIndex;
    }

    inline bool TraceAny(const Scene& scene, const Ray& ray)
    {
        const float3 invDirection = make_float3(1.0f) / ray.direction;
        uint32_t stack[80];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0)
        {
            const Scene::Node& node = scene.nodes[stack[--sp]];
            if (!AabbIntersect(node, ray, invDirection))
                continue;
            if (node.left == InvalidIndex && node.right == InvalidIndex)
            {
                for (uint32_t i = 0; i < node.count; i++)
                {
                    float t, u, v;
                    if (IntersectTriangleUvt(scene.bvhIsect[node.first + i], ray, t, u, v) && t >= ray.tMin && t < ray.tMax)
                        return true;
                }
            }
            else
            {
                stack[sp++] = node.left;
                stack[sp++] = node.right;
            }
        }
        return false;
    }

    // ------------------------------------------------------------------
    // Path state and camera (PathData.hpp:8-35, PathGeneration.cu:15-54)
    // ------------------------------------------------------------------
    struct Camera { float3 origin, lowerLeftCorner, horizontal, vertical; };
    struct PixelGrid { uint32_t width, height, samplesPerPixel, samplesPerPixelAxis; };

    struct PathState
    {
        uint64_t sample;
        uint32_t depth;
        float3 throughput;
        float currentMediumIor;
        bool lastScatterWasDelta;
        Random random;
        float3 radiance;  // accumulated contributions of this path, in arrival order
        Ray ray;
        const std::vector<Bin>* bins;  // the light-selection table of the render (area or power weights)
    };

    inline void ComputePathSample(const PixelGrid& grid, uint64_t sampleIndex, float2 jitter, uint32_t* pixel, float2* uv)
    {
        const uint64_t spp = grid.samplesPerPixel;
        const uint32_t pixelIndex = static_cast<uint32_t>(sampleIndex / spp);
        const uint32_t sampleGridIndex = static_cast<uint32_t>(sampleIndex - (sampleIndex / spp) * spp);
        const uint32_t x = pixelIndex - (pixelIndex / grid.width) * grid.width;
        const uint32_t y = pixelIndex / grid.width;
        const uint32_t sampleGridX = sampleGridIndex - (sampleGridIndex / grid.samplesPerPixelAxis) * grid.samplesPerPixelAxis;
        const uint32_t sampleGridY = sampleGridIndex / grid.samplesPerPixelAxis;
        const float u = (x + (sampleGridX + jitter.x) / grid.samplesPerPixelAxis) / grid.width;
        const float v = (y + (sampleGridY + jitter.y) / grid.samplesPerPixelAxis) / grid.height;
        *pixel = pixelIndex;
        *uv = make_float2(u, v);
    }

    inline Ray GenerateCameraRay(const Camera& camera, float2 uv)
    {
        Ray ray;
        ray.direction = normalize(camera.lowerLeftCorner + uv.x * camera.horizontal + uv.y * camera.vertical - camera.origin);
        ray.origin = camera.origin;
        ray.tMin = MinT;
        ray.tMax = MaxT;
        return ray;
    }

    // PathGeneration.cu:56-102 for one sample: Philox stream, jitter, camera ray
    inline void GeneratePath(const Camera& camera, const PixelGrid& grid, uint64_t sampleIndex, PathState& ps, uint64_t rngOffset,
                             uint32_t rngPolicy, const std::vector<Bin>* bins)
    {
        ps.sample = sampleIndex;
        ps.random = Random{sampleIndex + rngOffset, 0, rngPolicy};
        ps.bins = bins;
        const float2 jitter = ps.random.NextFloat2();
        uint32_t pixel;
        float2 uv;
        ComputePathSample(grid, sampleIndex, jitter, &pixel, &uv);
        ps.depth = 0;
        ps.throughput = make_float3(1.0f, 1.0f, 1.0f);
        ps.currentMediumIor = DefaultIor;
        ps.lastScatterWasDelta = true;
        ps.radiance = make_float3(0.0f);
        ps.ray = GenerateCameraRay(camera, uv);
    }

    // ------------------------------------------------------------------
    // Material evaluation, MaterialEval.cu
    // ------------------------------------------------------------------
    struct ResolvedHit
    {
        uint32_t index;
        float3 position, geometricNormal, normal;
        float4 tangent;
        float2 uv;
        uint32_t material;
    };

    inline float3 FixGeometricNormal(float3 n, float3 d) // :25-30
    {
        if (dot(n, d) > 0.0f)
            return -n;
        return n;
    }

    inline ResolvedHit LoadResolvedHit(const Scene& scene, const Ray& ray, const Hit& hitData) // :54-87
    {
        const TriangleShading& tri = scene.shading[hitData.triangle];
        float b0 = 1.0f - hitData.u - hitData.v;
        float b1 = hitData.u;
        float b2 = hitData.v;
        ResolvedHit hit;
        hit.index = hitData.triangle;
        hit.position = ray.origin + ray.direction * ray.tMax;
        hit.geometricNormal = FixGeometricNormal(tri.geometricNormal, ray.direction);
        hit.normal = b0 * make_float3(tri.normals[0]) + b1 * make_float3(tri.normals[1]) + b2 * make_float3(tri.normals[2]);
        hit.tangent = b0 * tri.tangents[0] + b1 * tri.tangents[1] + b2 * tri.tangents[2];
        hit.uv = b0 * tri.uvs[0] + b1 * tri.uvs[1] + b2 * tri.uvs[2];
        hit.material = tri.material;
        return hit;
    }

    inline float3 Texel3(const float* v) { return make_float3(v[0], v[1], v[2]); }

    inline Frame GetShadingFrame(const ResolvedHit& hit, const MaterialRecord& m) // :89-115
    {
        float3 baseTangent = make_float3(hit.tangent.x, hit.tangent.y, hit.tangent.z);
        float tangentSign = hit.tangent.w < 0.0f ? -1.0f : 1.0f;
        Frame baseFrame = BuildFrame(hit.normal, baseTangent, tangentSign);
        float3 tangentSpaceNormal = normalize(Texel3(m.normal) * 2.0f - 1.0f);
        float3 shadingNormal = tangentSpaceNormal.x * baseFrame.tangent + tangentSpaceNormal.y * baseFrame.bitangent +
                               tangentSpaceNormal.z * baseFrame.normal;
        return BuildFrame(shadingNormal, baseTangent, tangentSign);
    }

    inline float Luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; } // :117-120

    struct PathContinuation { bool terminated; uint32_t depth; float3 throughput; };

    inline PathContinuation ComputePathContinuation(const PathState& path, uint32_t limit, float3 w, float rr) // :129-146
    {
        uint32_t nextDepth = path.depth + 1;
        if (nextDepth >= limit)
            return {true, nextDepth, make_float3(0.0f)};
        float3 nextThroughput = path.throughput * w;
        if (nextDepth < RussianRouletteStartDepth)
            return {false, nextDepth, nextThroughput};
        float survival = clampf(MaxComponent(nextThroughput), 0.0f, 1.0f);
        if (rr > survival)
            return {true, nextDepth, make_float3(0.0f)};
        return {false, nextDepth, nextThroughput / survival};
    }

    inline Ray SpawnScatteredRay(const Ray& ray, float3 nextDirection, float3 geometricNormal) // :148-156
    {
        Ray r;
        r.origin = ray.origin + ray.direction * ray.tMax + geometricNormal * 1e-4f;
        r.direction = nextDirection;
        r.tMin = MinT;
        r.tMax = MaxT;
        return r;
    }

    struct ResolvedLightHit
    {
        uint32_t index;
        float3 position, geometricNormal, wi;
        float distanceSquared;
        float3 emission;
        float pdf;
    };

    inline ResolvedLightHit SampleLightTriangle(const Scene& scene, const std::vector<Bin>& bins, float lightSelectionSample, float2 xi,
                                                float3 hitPoint) // :171-192
    {
        uint32_t lightIndex;
        float pmf;
        SampleAlias(bins, lightSelectionSample, &lightIndex, &pmf);
        const LightTriangle& light = scene.lights[lightIndex];
        float sqrtXi0 = std::sqrt(xi.x);
        const float b1 = sqrtXi0 * (1.0f - xi.y);
        const float b2 = sqrtXi0 * xi.y;
        float3 position = light.v0 + b1 * light.edge1 + b2 * light.edge2;
        float3 toLight = position - hitPoint;
        float distanceSquared = dot(toLight, toLight);
        float3 wi = normalize(toLight);
        float3 gn = FixGeometricNormal(light.geometricNormal, wi);
        return {light.index, position, gn, wi, distanceSquared, light.emission, pmf / light.area};
    }

    struct ShadowRay { bool valid; float3 radiance; Ray ray; };
    enum Outcome { Terminated = 0, Continued = 1 };

    inline float3 SampleCosineWeightedHemisphere(float2 u) // :222-229
    {
        float phi = 2.0f * PiF * u.x;
        float cosTheta = std::sqrt(u.y);
        float sinTheta = std::sqrt(1.0f - u.y);
        float s, c;
        dm_sincos(phi, &s, &c);
        return make_float3(sinTheta * c, sinTheta * s, cosTheta);
    }

    inline ShadowRay MakeShadowRay(float3 hitPosition, float3 geometricNormal, const ResolvedLightHit& lightHit, float3 radiance) // :261-267
    {
        float3 shadowOrigin = hitPosition + geometricNormal * 1e-4f;
        float3 shadowRayVector = lightHit.position - shadowOrigin;
        float dist = length(shadowRayVector);
        float3 direction = shadowRayVector / dist;
        return ShadowRay{true, radiance, Ray{shadowOrigin, direction, MinT, dist - 1e-4f}};
    }

    inline ShadowRay EvaluateDiffuseDirect(const PathState& path, float3 hitPosition, float3 gn, const Frame& frame, float3 rs, float3 albedo, const Scene& scene) // :231-268
    {
        const ResolvedLightHit lightHit = SampleLightTriangle(scene, *path.bins, rs.x, make_float2(rs.y, rs.z), hitPosition);
        if (lightHit.distanceSquared < 1e-6f) return ShadowRay{false, {}, {}};
        float cosThetaI = std::fmax(dot(frame.normal, lightHit.wi), 0.0f);
        float geometricCosThetaI = std::fmax(dot(gn, lightHit.wi), 0.0f);
        if (cosThetaI <= 0.0f || geometricCosThetaI <= 0.0f) return ShadowRay{false, {}, {}};
        float cosThetaLight = std::fmax(dot(lightHit.geometricNormal, make_float3(0.0f) - lightHit.wi), 0.0f);
        if (cosThetaLight <= 0.0f) return ShadowRay{false, {}, {}};
        float3 brdf = albedo / PiF;
        float geometryTerm = cosThetaI * cosThetaLight / lightHit.distanceSquared;
        float3 radiance = lightHit.emission * path.throughput * brdf * geometryTerm / lightHit.pdf;
        return MakeShadowRay(hitPosition, gn, lightHit, radiance);
    }

    inline Outcome Continue(PathState& path, const Ray& ray, float3 dir, float3 gn, const PathContinuation& c, bool delta)
    {
        Ray next = SpawnScatteredRay(ray, dir, gn);
        path.depth = c.depth;
        path.throughput = c.throughput;
        path.lastScatterWasDelta = delta;
        path.ray = next;
        return Continued;
    }

    inline Outcome EvaluateDiffuseIndirect(PathState& path, const Ray& ray, uint32_t limit, float3 gn, const Frame& frame, float3 rs, float3 albedo) // :270-309
    {
        const float2 directionSample = make_float2(rs.x, rs.y);
        const float rrSample = rs.z;
        const float3 omegaI = frame.FromLocal(SampleCosineWeightedHemisphere(directionSample));
        float cosThetaI = std::fmax(dot(frame.normal, omegaI), 0.0f);
        float geometricCosThetaI = std::fmax(dot(gn, omegaI), 0.0f);
        if (cosThetaI <= 0.0f || geometricCosThetaI <= 0.0f) return Terminated;
        const PathContinuation c = ComputePathContinuation(path, limit, albedo, rrSample);
        if (c.terminated) return Terminated;
        return Continue(path, ray, omegaI, gn, c, false);
    }

    inline float3 SamplePhongLobe(float3 reflected, float exponent, float2 u) // :394-403
    {
        float phi = 2.0f * PiF * u.x;
        float cosTheta = dm_pow(u.y, 1.0f / (exponent + 1.0f));
        float sinTheta = std::sqrt(1.0f - cosTheta * cosTheta);
        float s, c;
        dm_sincos(phi, &s, &c);
        float3 sampled = make_float3(sinTheta * c, sinTheta * s, cosTheta);
        return BuildFrame(reflected).FromLocal(sampled);
    }

    inline float LoadShininess(const MaterialRecord& m) // :405-408
    {
        return m.shininess * (MaxShininess - MinShininess) + MinShininess;
    }

    inline ShadowRay EvaluatePhongDirect(const PathState& path, const Ray& ray, float3 hitPosition, float3 gn, const Frame& frame, float3 rs,
                                         float3 albedo, float3 specular, float shininess, const Scene& scene) // :410-455
    {
        const ResolvedLightHit lightHit = SampleLightTriangle(scene, *path.bins, rs.x, make_float2(rs.y, rs.z), hitPosition);
        if (lightHit.distanceSquared < 1e-6f) return ShadowRay{false, {}, {}};
        float cosThetaI = std::fmax(dot(frame.normal, lightHit.wi), 0.0f);
        float geometricCosThetaI = std::fmax(dot(gn, lightHit.wi), 0.0f);
        if (cosThetaI <= 0.0f || geometricCosThetaI <= 0.0f) return ShadowRay{false, {}, {}};
        float cosThetaLight = std::fmax(dot(lightHit.geometricNormal, make_float3(0.0f) - lightHit.wi), 0.0f);
        if (cosThetaLight <= 0.0f) return ShadowRay{false, {}, {}};
        float3 reflectionDirection = normalize(reflect(ray.direction, frame.normal));
        float cosThetaR = std::fmax(dot(reflectionDirection, lightHit.wi), 0.0f);
        float3 diffuseBrdf = albedo / PiF;
        float3 specularBrdf = specular * (shininess + 2.0f) * InvTwoPi * dm_pow(cosThetaR, shininess);
        float3 brdf = diffuseBrdf + specularBrdf;
        float geometryTerm = cosThetaI * cosThetaLight / lightHit.distanceSquared;
        float3 radiance = lightHit.emission * path.throughput * brdf * geometryTerm / lightHit.pdf;
        return MakeShadowRay(hitPosition, gn, lightHit, radiance);
    }

    inline Outcome EvaluatePhongIndirect(PathState& path, const Ray& ray, uint32_t limit, float3 gn, const Frame& frame, float4 rs,
                                         float3 albedo, float3 specular, float shininess) // :457-542
    {
        const float2 directionSample = make_float2(rs.x, rs.y);
        const float lobeSample = rs.z;
        const float rrSample = rs.w;
        float diffuseWeight = Luminance(albedo);
        float specularWeight = Luminance(specular);
        float weightSum = diffuseWeight + specularWeight;
        if (weightSum <= 0.0f) return Terminated;
        float diffuseSelectionProbability = diffuseWeight / weightSum;
        float specularSelectionProbability = 1.0f - diffuseSelectionProbability;
        float3 reflectionDirection = normalize(reflect(ray.direction, frame.normal));
        float3 omegaI;
        if (lobeSample < diffuseSelectionProbability)
            omegaI = frame.FromLocal(SampleCosineWeightedHemisphere(directionSample));
        else
            omegaI = SamplePhongLobe(reflectionDirection, shininess, directionSample);
        float cosThetaI = std::fmax(dot(frame.normal, omegaI), 0.0f);
        float geometricCosThetaI = std::fmax(dot(gn, omegaI), 0.0f);
        if (cosThetaI <= 0.0f || geometricCosThetaI <= 0.0f) return Terminated;
        float cosThetaR = std::fmax(dot(reflectionDirection, omegaI), 0.0f);
        float phongLobeOverTwoPi = InvTwoPi * dm_pow(cosThetaR, shininess);
        float diffusePdf = cosThetaI * InvPi;
        float specularPdf = (shininess + 1.0f) * phongLobeOverTwoPi;
        float pdf = diffuseSelectionProbability * diffusePdf + specularSelectionProbability * specularPdf;
        if (pdf <= 0.0f) return Terminated;
        float3 diffuseBrdf = albedo * InvPi;
        float3 specularBrdf = specular * (shininess + 2.0f) * phongLobeOverTwoPi;
        const PathContinuation c = ComputePathContinuation(path, limit, (diffuseBrdf + specularBrdf) * (cosThetaI / pdf), rrSample);
        if (c.terminated) return Terminated;
        return Continue(path, ray, omegaI, gn, c, false);
    }

    // GGX helpers, MaterialEval.cu:587-650
    inline float2 SampleUniformDiskPolar(float2 u)
    {
        float r = std::sqrt(u.x);
        float theta = 2.0f * PiF * u.y;
        float s, c;
        dm_sincos(theta, &s, &c);
        return make_float2(r * c, r * s);
    }

    inline float3 TrowbridgeSampleWm(float3 w, float2 alpha, float2 u)
    {
        float3 wh = normalize(make_float3(alpha.x * w.x, alpha.y * w.y, w.z));
        if (wh.z < 0)
            wh = -wh;
        float3 tangent = (wh.z < 0.999f) ? normalize(cross(wh, make_float3(0.0f, 0.0f, 1.0f))) : make_float3(1.0f, 0.0f, 0.0f);
        float3 bitangent = cross(wh, tangent);
        float2 diskSample = SampleUniformDiskPolar(u);
        float h = std::sqrt(1.0f - diskSample.x * diskSample.x);
        diskSample.y = lerpf(h, diskSample.y, (1 + wh.z) * 0.5f);
        float pz = std::sqrt(std::fmax(0.0f, 1.0f - dot(diskSample, diskSample)));
        float3 nh = diskSample.x * tangent + diskSample.y * bitangent + pz * wh;
        return normalize(make_float3(alpha.x * nh.x, alpha.y * nh.y, std::fmax(1e-6f, nh.z)));
    }

    inline float Lambda(float3 w, float alpha)
    {
        float tan2Theta = Tan2Theta(w);
        if (tan2Theta == INFINITY)
            return 0.0f;
        float alpha2 = Sqr(CosPhi(w) * alpha) + Sqr(SinPhi(w) * alpha);
        return (std::sqrt(1.0f + alpha2 * tan2Theta) - 1.0f) * 0.5f;
    }

    inline float G1(float3 w, float alpha) { return 1.0f / (1.0f + Lambda(w, alpha)); }
    inline float G(float3 wo, float3 wi, float alpha) { return 1 / (1 + Lambda(wo, alpha) + Lambda(wi, alpha)); }

    inline float D(float3 wm, float alpha)
    {
        float tan2Theta = Tan2Theta(wm);
        if (tan2Theta == INFINITY)
            return 0.0f;
        float cos4Theta = Sqr(Cos2Theta(wm));
        if (cos4Theta < 1e-16f) return 0.0f;
        float e = tan2Theta * (Sqr(CosPhi(wm) / alpha) + Sqr(SinPhi(wm) / alpha));
        return 1 / (PiF * Sqr(alpha) * cos4Theta * Sqr(1 + e));
    }

    inline float D(float3 w, float3 wm, float alpha)
    {
        return G1(w, alpha) / AbsCosTheta(w) * D(wm, alpha) * std::fabs(dot(w, wm));
    }

    inline float3 FresnelSchlick(float3 f0, float cosThetaH)
    {
        return f0 + (1.0f - f0) * dm_pow5(1.0f - cosThetaH);
    }

    inline ShadowRay EvaluateGgxDirect(const PathState& path, const Ray& ray, float3 hitPosition, float3 gn, const Frame& frame, float3 rs,
                                       float3 baseColor, float alpha, float metallic, float ior, const Scene& scene) // :652-718
    {
        const ResolvedLightHit lightHit = SampleLightTriangle(scene, *path.bins, rs.x, make_float2(rs.y, rs.z), hitPosition);
        if (lightHit.distanceSquared < 1e-6f || lightHit.pdf <= 0.0f) return ShadowRay{false, {}, {}};
        float geometricCosThetaI = dot(gn, lightHit.wi);
        if (geometricCosThetaI <= 0.0f) return ShadowRay{false, {}, {}};
        float cosThetaLight = std::fmax(dot(lightHit.geometricNormal, make_float3(0.0f) - lightHit.wi), 0.0f);
        if (cosThetaLight <= 0.0f) return ShadowRay{false, {}, {}};
        float3 wo = frame.ToLocal(make_float3(0.0f) - ray.direction);
        float3 wi = frame.ToLocal(lightHit.wi);
        float cosThetaI = CosTheta(wi);
        float cosThetaO = CosTheta(wo);
        if (cosThetaI <= 0.0f || cosThetaO <= 0.0f) return ShadowRay{false, {}, {}};
        float3 wm = normalize(wo + wi);
        if (CosTheta(wm) <= 0.0f) return ShadowRay{false, {}, {}};
        float woDotWm = dot(wo, wm);
        float wiDotWm = dot(wi, wm);
        if (woDotWm <= 1e-6f || wiDotWm <= 1e-6f) return ShadowRay{false, {}, {}};
        float dielectricF0 = Sqr((path.currentMediumIor - ior) / (path.currentMediumIor + ior));
        float3 f0 = lerp3(make_float3(dielectricF0), baseColor, metallic);
        float3 diffuseColor = baseColor * (1.0f - metallic);
        float3 fresnel = FresnelSchlick(f0, clampf(woDotWm, 0.0f, 1.0f));
        float3 diffuseBsdf = (1.0f - fresnel) * diffuseColor * InvPi;
        float3 ggxBsdf = fresnel * D(wm, alpha) * G(wo, wi, alpha) / (4.0f * cosThetaI * cosThetaO);
        float3 bsdf = diffuseBsdf + ggxBsdf;
        float geometryTerm = cosThetaI * cosThetaLight / lightHit.distanceSquared;
        float3 radiance = lightHit.emission * path.throughput * bsdf * geometryTerm / lightHit.pdf;
        return MakeShadowRay(hitPosition, gn, lightHit, radiance);
    }

    inline Outcome EvaluateGgxIndirect(PathState& path, const Ray& ray, uint32_t limit, float3 gn, const Frame& frame, float4 rs,
                                       float3 baseColor, float alpha, float metallic, float ior) // :720-836
    {
        const float2 directionSample = make_float2(rs.x, rs.y);
        const float lobeSample = rs.z;
        const float rrSample = rs.w;
        float3 wo = frame.ToLocal(make_float3(0.0f) - ray.direction);
        if (wo.z <= 0.0f) return Terminated;
        float dielectricF0 = Sqr((path.currentMediumIor - ior) / (path.currentMediumIor + ior));
        float3 f0 = lerp3(make_float3(dielectricF0), baseColor, metallic);
        float3 diffuseColor = baseColor * (1.0f - metallic);
        float diffuseWeight = Luminance(diffuseColor);
        float specularWeight = Luminance(f0);
        float weightSum = diffuseWeight + specularWeight;
        if (weightSum <= 1e-6f) return Terminated;
        float diffuseSelectionProbability = diffuseWeight / weightSum;
        float specularSelectionProbability = specularWeight / weightSum;
        float3 wi;
        if (lobeSample < diffuseSelectionProbability)
            wi = SampleCosineWeightedHemisphere(directionSample);
        else
        {
            float3 sampledWm = TrowbridgeSampleWm(wo, make_float2(alpha, alpha), directionSample);
            wi = reflect(-wo, sampledWm);
        }
        float cosThetaI = CosTheta(wi);
        float cosThetaO = CosTheta(wo);
        if (cosThetaI <= 0.0f) return Terminated;
        float3 wm = normalize(wi + wo);
        if (CosTheta(wm) <= 0.0f) return Terminated;
        float woDotWm = dot(wo, wm);
        if (woDotWm <= 1e-6f) return Terminated;
        float3 fresnel = FresnelSchlick(f0, clampf(woDotWm, 0.0f, 1.0f));
        float3 diffuseBsdf = (1.0f - fresnel) * diffuseColor * InvPi;
        float3 ggxBsdf = fresnel * D(wm, alpha) * G(wo, wi, alpha) / (4.0f * cosThetaI * cosThetaO);
        float diffusePdf = cosThetaI * InvPi;
        float ggxPdf = D(wo, wm, alpha) / (4.0f * woDotWm);
        float pdf = diffuseSelectionProbability * diffusePdf + specularSelectionProbability * ggxPdf;
        if (pdf <= 1e-8f) return Terminated;
        float3 worldWi = frame.FromLocal(wi);
        if (dot(worldWi, gn) <= 0.0f) return Terminated;
        const PathContinuation c = ComputePathContinuation(path, limit, (diffuseBsdf + ggxBsdf) * (cosThetaI / pdf), rrSample);
        if (c.terminated) return Terminated;
        return Continue(path, ray, worldWi, gn, c, false);
    }

    // Shadow radiance clamp, Intersect.cu:125-134
    inline float3 ClampRadiance(float3 radiance, float maxLength)
    {
        float lengthSquared = dot(radiance, radiance);
        float maxLengthSquared = maxLength * maxLength;
        if (lengthSquared > maxLengthSquared)
            radiance = radiance * (maxLength * dm_rsqrt(lengthSquared));
        return radiance;
    }

    // Shades one hit; returns the continuation outcome and fills the NEE shadow ray.
    // Dispatch mirrors the per-model kernels at MaterialEval.cu:194-912.
    inline Outcome Shade(const Scene& scene, PathState& path, const Hit& h, uint32_t limit, bool nee, ShadowRay& shadow)
    {
        shadow.valid = false;
        const Ray ray = path.ray;
        Ray hitRay = ray;
        switch (h.model)
        {
            case ModelNormal: // :194-220
            {
                const ResolvedHit hit = LoadResolvedHit(scene, hitRay, h);
                float3 normal = hit.normal;
                path.radiance = path.radiance + (path.throughput * normal * 0.5f + 0.5f);
                return Terminated;
            }
            case ModelDiffuse: // :311-350
            {
                const ResolvedHit hit = LoadResolvedHit(scene, hitRay, h);
                const MaterialRecord& m = scene.materials[hit.material];
                const float3 albedo = Texel3(m.color);
                const Frame frame = GetShadingFrame(hit, m);
                const float3 indirect = path.random.NextFloat3();
                if (nee)
                {
                    const float3 direct = path.random.NextFloat3();
                    shadow = EvaluateDiffuseDirect(path, hit.position, hit.geometricNormal, frame, direct, albedo, scene);
                }
                return EvaluateDiffuseIndirect(path, hitRay, limit, hit.geometricNormal, frame, indirect, albedo);
            }
            case ModelMirror: // :352-392
            {
                const ResolvedHit hit = LoadResolvedHit(scene, hitRay, h);
                const MaterialRecord& m = scene.materials[hit.material];
                const float3 reflectance = Texel3(m.specular);
                const Frame frame = GetShadingFrame(hit, m);
                const float rrSample = path.random.NextFloat();
                const float3 omegaI = reflect(hitRay.direction, frame.normal);
                const PathContinuation c = ComputePathContinuation(path, limit, reflectance, rrSample);
                if (c.terminated) return Terminated;
                return Continue(path, hitRay, omegaI, hit.geometricNormal, c, true);
            }
            case ModelPhong: // :544-585
            {
                const ResolvedHit hit = LoadResolvedHit(scene, hitRay, h);
                const MaterialRecord& m = scene.materials[hit.material];
                const float3 albedo = Texel3(m.color);
                const float3 specular = Texel3(m.specular);
                const float shininess = LoadShininess(m);
                const Frame frame = GetShadingFrame(hit, m);
                const float4 indirect = path.random.NextFloat4();
                if (nee)
                {
                    const float3 direct = make_float3(indirect.x, indirect.y, indirect.z);
                    shadow = EvaluatePhongDirect(path, hitRay, hit.position, hit.geometricNormal, frame, direct, albedo, specular, shininess, scene);
                }
                return EvaluatePhongIndirect(path, hitRay, limit, hit.geometricNormal, frame, indirect, albedo, specular, shininess);
            }
            case ModelGgx: // :838-880
            {
                const ResolvedHit hit = LoadResolvedHit(scene, hitRay, h);
                const MaterialRecord& m = scene.materials[hit.material];
                const float3 baseColor = Texel3(m.color);
                const float3 rma = Texel3(m.rma);
                float alpha = std::fmax(rma.x * rma.x, 0.001f);
                float metallic = rma.y;
                const Frame frame = GetShadingFrame(hit, m);
                const float4 indirect = path.random.NextFloat4();
                if (nee)
                {
                    const float3 direct = path.random.NextFloat3();
                    shadow = EvaluateGgxDirect(path, hitRay, hit.position, hit.geometricNormal, frame, direct, baseColor, alpha, metallic, m.ior, scene);
                }
                return EvaluateGgxIndirect(path, hitRay, limit, hit.geometricNormal, frame, indirect, baseColor, alpha, metallic, m.ior);
            }
            case ModelEmissive: // :882-912
            default:
            {
                if (nee && !path.lastScatterWasDelta)
                    return Terminated;
                const uint32_t material = scene.shading[h.triangle].material;
                const float3 emission = Texel3(scene.materials[material].emission);
                path.radiance = path.radiance + path.throughput * emission;
                return Terminated;
            }
        }
    }

    // ------------------------------------------------------------------
    // Thread pool helper
    // ------------------------------------------------------------------
    inline void ParallelFor(size_t n, int threads, const std::function<void(size_t, size_t)>& fn)
    {
        if (threads <= 1 || n < 4096)
        {
            fn(0, n);
            return;
        }
        size_t chunks = static_cast<size_t>(threads) * 8;
        std::atomic<size_t> next{0};
        size_t chunk = (n + chunks - 1) / chunks;
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; t++)
            pool.emplace_back([&]()
            {
                for (;;)
                {
                    size_t c = next.fetch_add(1);
                    size_t b = c * chunk;
                    if (b >= n) break;
                    fn(b, std::min(n, b + chunk));
                }
            });
        for (auto& th : pool) th.join();
    }

    // ------------------------------------------------------------------
    // Scene preparation: Renderer.cpp:144-213 (triangle records),
    // LightSampler.cpp:5-40 (lights, area weights), HostBvh/DeviceBvh (BVH).
    // ------------------------------------------------------------------
    inline Scene* BuildScene(uint32_t triangleCount, const float* positions, const float* normals, const float* tangents,
                             const float* uvs, const uint32_t* materialIds, uint32_t materialCount, const MaterialRecord* materials)
    {
        auto scene = std::make_unique<Scene>();
        scene->triangleCount = triangleCount;
        scene->materials.assign(materials, materials + materialCount);
        scene->materialCounts.assign(ModelCount, 0);
        for (uint32_t m = 0; m < materialCount; m++)
            scene->materialCounts[std::min<uint32_t>(materials[m].model, ModelCount - 1)]++;
        scene->positions.resize(static_cast<size_t>(triangleCount) * 3);
        scene->isect.resize(triangleCount);
        scene->shading.resize(triangleCount);
        for (uint32_t t = 0; t < triangleCount; t++)
        {
            float3 p[3];
            for (int k = 0; k < 3; k++)
            {
                const float* pp = positions + (static_cast<size_t>(t) * 3 + k) * 3;
                p[k] = make_float3(pp[0], pp[1], pp[2]);
                scene->positions[static_cast<size_t>(t) * 3 + k] = p[k];
                const float* nn = normals + (static_cast<size_t>(t) * 3 + k) * 3;
                const float* tt = tangents + (static_cast<size_t>(t) * 3 + k) * 4;
                const float* uu = uvs + (static_cast<size_t>(t) * 3 + k) * 2;
                scene->shading[t].normals[k] = make_float4(nn[0], nn[1], nn[2], 0.0f);
                scene->shading[t].tangents[k] = make_float4(tt[0], tt[1], tt[2], tt[3]);
                scene->shading[t].uvs[k] = make_float2(uu[0], uu[1]);
            }
            TriangleIntersection& ti = scene->isect[t];
            ti.edge1 = p[1] - p[0];
            ti.edge2 = p[2] - p[0];
            ti.v0 = p[0];
            uint32_t mat = materialIds[t];
            ti.model = std::min<uint32_t>(scene->materials[mat].model, ModelCount - 1);
            scene->shading[t].material = mat;
            scene->shading[t].geometricNormal = normalize(cross(ti.edge1, ti.edge2));
        }
        // lights in input order (LightSampler.cpp:12-27)
        std::vector<float> weights;
        std::vector<uint32_t> values;
        for (uint32_t t = 0; t < triangleCount; t++)
        {
            if (scene->isect[t].model != ModelEmissive) continue;
            const TriangleIntersection& ti = scene->isect[t];
            float area = 0.5f * length(cross(ti.edge1, ti.edge2));
            weights.push_back(area);
            values.push_back(static_cast<uint32_t>(scene->lights.size()));
            LightTriangle lt;
            lt.edge1 = ti.edge1;
            lt.edge2 = ti.edge2;
            lt.v0 = ti.v0;
            lt.index = t;
            lt.geometricNormal = scene->shading[t].geometricNormal;
            lt.area = area;
            lt.emission = Texel3(scene->materials[scene->shading[t].material].emission);
            scene->lights.push_back(lt);
        }
        if (!weights.empty())
        {
            scene->bins = BuildAliasTable(weights, values);
            // power weights: area x luminance of the emission constant (Rec. 709, as MaterialEval.cu's
            // Luminance), in FP64
            std::vector<double> power(weights.size()), area(weights.size());
            for (size_t k = 0; k < weights.size(); k++)
            {
                const float* e = scene->materials[scene->shading[scene->lights[k].index].material].emission;
                const double lum = 0.2126 * static_cast<double>(e[0]) + 0.7152 * static_cast<double>(e[1]) + 0.0722 * static_cast<double>(e[2]);
                area[k] = static_cast<double>(weights[k]);
                power[k] = lum * area[k];
            }
            scene->binsPower = BuildPowerAliasTable(power, area);
        }
        // reference BVH
        scene->order.resize(triangleCount);
        std::iota(scene->order.begin(), scene->order.end(), 0u);
        BvhBuilder b{*scene, scene->order, scene->nodes};
        b.maxDepth = BvhBuilder::EstimateMaxDepth(triangleCount);
        b.minTriangles = BvhBuilder::EstimateMaxTrianglesPerLeaf(triangleCount);
        auto root = b.BuildRecurse(0, triangleCount, 0);
        b.Flatten(*root);
        scene->bvhDepth = b.depthReached;
        scene->bvhIsect.resize(triangleCount);
        for (uint32_t i = 0; i < triangleCount; i++)
            scene->bvhIsect[i] = scene->isect[scene->order[i]];
        return scene.release();
    }

    struct RenderSettings
    {
        uint32_t width, height, spp, depth, nee, poolSize;
        uint64_t maxSamples;   // 0 = the whole frame
        int threads;
        int accumulation;      // 0 = FP32 sequential, 1 = FP32 Kahan (sample order), 2 = FP64
        uint64_t rngOffset;    // added to the sample index to form the Philox subsequence
        uint32_t rngPolicy;    // RngPhilox (the reference's) or RngPcg32
        uint32_t lightMode;    // 0 = area weights (the reference's), 1 = power weights
    };

    // Renderer.cpp:468-647 replayed on the CPU, iteration by iteration, with the
    // same regeneration rule (:573-619). Outputs per-sample radiance (capture),
    // per-pixel accumulation, the RGBA8 framebuffer (Image.cu:34-54) and a
    // per-iteration log of queue sizes.
    inline int Render(const Scene& scene, const Camera& camera, const RenderSettings& s, float* sampleRadiance, float* accumulation,
                      uint32_t* framebuffer, uint32_t* queueLog, uint32_t queueLogCapacity, uint32_t* iterations)
    {
        PixelGrid grid;
        grid.width = s.width;
        grid.height = s.height;
        grid.samplesPerPixelAxis = static_cast<uint32_t>(std::sqrt(static_cast<double>(s.spp)));
        grid.samplesPerPixel = grid.samplesPerPixelAxis * grid.samplesPerPixelAxis;
        uint64_t totalSamples = static_cast<uint64_t>(grid.samplesPerPixel) * s.width * s.height;
        if (s.maxSamples != 0 && s.maxSamples < totalSamples)
            totalSamples = s.maxSamples;
        const uint32_t generateCount = static_cast<uint32_t>(std::min<uint64_t>(totalSamples, s.poolSize));
        // The reference's light sampler reads bin 0 of an empty table when NEE meets a scene without
        // emitters (AliasTableView.hpp:32-60); here NEE is off for such scenes (nothing to connect to).
        const bool nee = s.nee != 0 && !scene.lights.empty();
        const std::vector<Bin>* bins = s.lightMode == 1 ? &scene.binsPower : &scene.bins;

        std::vector<PathState> active(generateCount);
        ParallelFor(generateCount, s.threads, [&](size_t b, size_t e)
        {
            for (size_t i = b; i < e; i++) GeneratePath(camera, grid, i, active[i], s.rngOffset, s.rngPolicy, bins);
        });
        uint64_t launched = generateCount;
        uint32_t iter = 0;
        std::vector<Hit> hits;
        std::vector<uint8_t> outcome;
        std::vector<ShadowRay> shadows;
        std::vector<uint8_t> hitFlag;
        while (!active.empty())
        {
            const size_t n = active.size();
            hits.resize(n);
            hitFlag.resize(n);
            outcome.resize(n);
            shadows.resize(n);
            // intersect (Intersect.cu:63-123), shade (MaterialEval.cu), shadow (Intersect.cu:136-179)
            ParallelFor(n, s.threads, [&](size_t b, size_t e)
            {
                for (size_t i = b; i < e; i++)
                {
                    PathState& ps = active[i];
                    Ray ray = ps.ray;
                    Hit h;
                    bool found = TraceClosest(scene, ray, h);
                    hitFlag[i] = found ? 1 : 0;
                    hits[i] = h;
                    shadows[i].valid = false;
                    if (!found)
                    {
                        outcome[i] = Terminated;
                        continue;
                    }
                    ps.ray.tMax = ray.tMax;
                    outcome[i] = static_cast<uint8_t>(Shade(scene, ps, h, s.depth, nee, shadows[i]));
                    if (shadows[i].valid && !TraceAny(scene, shadows[i].ray))
                        ps.radiance = ps.radiance + ClampRadiance(shadows[i].radiance, 20.0f);
                }
            });
            uint32_t modelCounts[ModelCount] = {0, 0, 0, 0, 0, 0};
            uint32_t shadowCount = 0, regenCount = 0;
            for (size_t i = 0; i < n; i++)
            {
                if (hitFlag[i]) modelCounts[hits[i].model]++;
                if (shadows[i].valid) shadowCount++;
                if (outcome[i] == Terminated) regenCount++;
            }
            if (queueLog != nullptr && iter < queueLogCapacity)
            {
                uint32_t* row = queueLog + static_cast<size_t>(iter) * 9;
                row[0] = static_cast<uint32_t>(n);
                for (uint32_t m = 0; m < ModelCount; m++) row[1 + m] = modelCounts[m];
                row[7] = shadowCount;
                row[8] = regenCount;
            }
            // finalize terminated paths, keep continued ones, regenerate (Renderer.cpp:573-619)
            std::vector<PathState> next;
            next.reserve(n);
            for (size_t i = 0; i < n; i++)
            {
                if (outcome[i] == Terminated)
                {
                    float* dst = sampleRadiance + active[i].sample * 3;
                    dst[0] = active[i].radiance.x;
                    dst[1] = active[i].radiance.y;
                    dst[2] = active[i].radiance.z;
                }
                else
                    next.push_back(active[i]);
            }
            const uint64_t remaining = totalSamples - launched;
            const uint32_t regenerate = static_cast<uint32_t>(std::min<uint64_t>(regenCount, remaining));
            size_t base = next.size();
            next.resize(base + regenerate);
            ParallelFor(regenerate, s.threads, [&](size_t b, size_t e)
            {
                for (size_t i = b; i < e; i++) GeneratePath(camera, grid, launched + i, next[base + i], s.rngOffset, s.rngPolicy, bins);
            });
            launched += regenerate;
            active.swap(next);
            iter++;
        }
        if (iterations) *iterations = iter;

        // accumulation in sample order, then PostprocessKernel (Image.cu:34-54)
        const size_t pixels = static_cast<size_t>(s.width) * s.height;
        const float invSpp = 1.0f / static_cast<float>(grid.samplesPerPixel);
        const uint64_t spp = grid.samplesPerPixel;
        ParallelFor(pixels, s.threads, [&](size_t b, size_t e)
        {
            for (size_t p = b; p < e; p++)
            {
                float acc[3];
                for (int c = 0; c < 3; c++)
                {
                    if (s.accumulation == 2)
                    {
                        double sum = 0.0;
                        for (uint64_t k = 0; k < spp; k++)
                        {
                            uint64_t si = p * spp + k;
                            if (si < totalSamples) sum += static_cast<double>(sampleRadiance[si * 3 + c]);
                        }
                        acc[c] = static_cast<float>(sum);
                    }
                    else if (s.accumulation == 1)
                    {
                        float sum = 0.0f, comp = 0.0f;
                        for (uint64_t k = 0; k < spp; k++)
                        {
                            uint64_t si = p * spp + k;
                            if (si >= totalSamples) break;
                            float y = sampleRadiance[si * 3 + c] - comp;
                            float t = sum + y;
                            comp = (t - sum) - y;
                            sum = t;
                        }
                        acc[c] = sum;
                    }
                    else
                    {
                        float sum = 0.0f;
                        for (uint64_t k = 0; k < spp; k++)
                        {
                            uint64_t si = p * spp + k;
                            if (si < totalSamples) sum += sampleRadiance[si * 3 + c];
                        }
                        acc[c] = sum;
                    }
                }
                if (accumulation)
                {
                    accumulation[p * 4 + 0] = acc[0];
                    accumulation[p * 4 + 1] = acc[1];
                    accumulation[p * 4 + 2] = acc[2];
                    accumulation[p * 4 + 3] = 0.0f;
                }
                if (framebuffer)
                {
                    uint8_t rgb[3];
                    for (int c = 0; c < 3; c++)
                    {
                        float hdr = acc[c] * invSpp;
                        float ldr = hdr / (hdr + 1.0f);
                        float g = dm_pow(ldr, 1.0f / 2.2f);
                        rgb[c] = static_cast<uint8_t>(clampf(g * 255.0f, 0.0f, 255.0f));
                    }
                    framebuffer[p] = static_cast<uint32_t>(rgb[0]) | (static_cast<uint32_t>(rgb[1]) << 8) |
                                     (static_cast<uint32_t>(rgb[2]) << 16) | (255u << 24);
                }
            }
        });
        return 0;
    }
}

// ----------------------------------------------------------------------
// C entry points for the Python test harness (ctypes)
// ----------------------------------------------------------------------
extern "C"
{
    void* oracle_scene_create(uint32_t triangleCount, const float* positions, const float* normals, const float* tangents,
                              const float* uvs, const uint32_t* materialIds, uint32_t materialCount, const void* materials)
    {
        return oracle::BuildScene(triangleCount, positions, normals, tangents, uvs, materialIds, materialCount,
                                  static_cast<const oracle::MaterialRecord*>(materials));
    }

    void oracle_scene_destroy(void* scene) { delete static_cast<oracle::Scene*>(scene); }

    // Reference BVH as flattened: nodes [n][10] floats-or-words (min3, max3, left, right, first, count),
    // and the BVH-position -> original-index order.
    uint32_t oracle_scene_bvh_node_count(void* scene) { return static_cast<uint32_t>(static_cast<oracle::Scene*>(scene)->nodes.size()); }
    uint32_t oracle_scene_bvh_depth(void* scene) { return static_cast<oracle::Scene*>(scene)->bvhDepth; }
    void oracle_scene_bvh_export(void* scene, void* nodesOut, uint32_t* orderOut)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        std::memcpy(nodesOut, s->nodes.data(), s->nodes.size() * sizeof(oracle::Scene::Node));
        std::memcpy(orderOut, s->order.data(), s->order.size() * sizeof(uint32_t));
    }
    uint32_t oracle_scene_light_count(void* scene) { return static_cast<uint32_t>(static_cast<oracle::Scene*>(scene)->lights.size()); }
    void oracle_scene_alias_export(void* scene, void* binsOut)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        std::memcpy(binsOut, s->bins.data(), s->bins.size() * sizeof(oracle::Bin));
    }
    void oracle_scene_alias_power_export(void* scene, void* binsOut)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        std::memcpy(binsOut, s->binsPower.data(), s->binsPower.size() * sizeof(oracle::Bin));
    }

    // The product's power-weighted alias table from FP64 power and area weights. bins [n][4] words.
    void oracle_power_alias_build(const double* power, const double* area, uint32_t n, void* binsOut)
    {
        std::vector<double> p(power, power + n), a(area, area + n);
        auto bins = oracle::BuildPowerAliasTable(p, a);
        std::memcpy(binsOut, bins.data(), bins.size() * sizeof(oracle::Bin));
    }

    // Exclusive FP64 prefix sum in the product's device order.
    void oracle_device_order_scan(const double* in, uint32_t n, double* out) { oracle::DeviceOrderExclusiveScan(in, out, n); }

    // Raw PCG32 stream of a sample key: count words from position, and their uniforms.
    void oracle_pcg_words(uint64_t key, uint64_t position, uint32_t count, uint32_t* wordsOut, float* uniformsOut)
    {
        oracle::Random r{key, position, oracle::RngPcg32};
        for (uint32_t i = 0; i < count; i++)
        {
            uint32_t w = r.Word(position + i);
            if (wordsOut) wordsOut[i] = w;
            if (uniformsOut) uniformsOut[i] = oracle::Random::ToUniformPcg(w);
        }
    }

    // PCG32 with an explicit (initstate, initseq) seeding, for the generator's published sequence.
    void oracle_pcg_seeded_words(uint64_t initstate, uint64_t initseq, uint32_t count, uint32_t* wordsOut)
    {
        oracle::Pcg32 g;
        g.Seed(initstate, initseq);
        for (uint32_t i = 0; i < count; i++) wordsOut[i] = g.Next();
    }

    // Closest hit for a ray batch: rays [n][8] = origin3, dir3, tMin, tMax.
    // Output: triangle (original index or 0xFFFFFFFF), u, v, t.
    void oracle_trace_closest(void* scene, const float* rays, uint32_t n, uint32_t* triOut, float* uvtOut, int threads)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        oracle::ParallelFor(n, threads, [&](size_t b, size_t e)
        {
            for (size_t i = b; i < e; i++)
            {
                const float* r = rays + i * 8;
                oracle::Ray ray{{r[0], r[1], r[2]}, {r[3], r[4], r[5]}, r[6], r[7]};
                oracle::Hit h;
                bool found = oracle::TraceClosest(*s, ray, h);
                triOut[i] = found ? h.triangle : oracle::InvalidIndex;
                uvtOut[i * 3 + 0] = found ? h.u : 0.0f;
                uvtOut[i * 3 + 1] = found ? h.v : 0.0f;
                uvtOut[i * 3 + 2] = found ? ray.tMax : 0.0f;
            }
        });
    }

    void oracle_trace_any(void* scene, const float* rays, uint32_t n, uint8_t* occludedOut, int threads)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        oracle::ParallelFor(n, threads, [&](size_t b, size_t e)
        {
            for (size_t i = b; i < e; i++)
            {
                const float* r = rays + i * 8;
                oracle::Ray ray{{r[0], r[1], r[2]}, {r[3], r[4], r[5]}, r[6], r[7]};
                occludedOut[i] = oracle::TraceAny(*s, ray) ? 1 : 0;
            }
        });
    }

    // Sequential Vose alias table (AliasTable.hpp:22-84). bins [n][4] words (q, p, alias, value).
    void oracle_alias_build(const float* weights, uint32_t n, void* binsOut)
    {
        std::vector<float> w(weights, weights + n);
        std::vector<uint32_t> v(n);
        std::iota(v.begin(), v.end(), 0u);
        auto bins = oracle::BuildAliasTable(w, v);
        std::memcpy(binsOut, bins.data(), bins.size() * sizeof(oracle::Bin));
    }

    void oracle_alias_sample(const void* bins, uint32_t nBins, const float* u, uint32_t n, uint32_t* indexOut, float* pmfOut)
    {
        const auto* b = static_cast<const oracle::Bin*>(bins);
        std::vector<oracle::Bin> table(b, b + nBins);
        for (uint32_t i = 0; i < n; i++)
            oracle::SampleAlias(table, u[i], &indexOut[i], &pmfOut[i]);
    }

    // Raw Philox stream words and uniforms: count words starting at position.
    void oracle_philox_words(uint64_t subsequence, uint64_t position, uint32_t count, uint32_t* wordsOut, float* uniformsOut)
    {
        oracle::Random r{subsequence, position};
        for (uint32_t i = 0; i < count; i++)
        {
            uint32_t w = r.Word(position + i);
            if (wordsOut) wordsOut[i] = w;
            if (uniformsOut) uniformsOut[i] = oracle::Random::ToUniform(w);
        }
    }

    void oracle_sincos(const float* x, uint32_t n, float* s, float* c)
    {
        for (uint32_t i = 0; i < n; i++) oracle::dm_sincos(x[i], &s[i], &c[i]);
    }

    void oracle_pow(const float* x, const float* y, uint32_t n, float* out)
    {
        for (uint32_t i = 0; i < n; i++) out[i] = oracle::dm_pow(x[i], y[i]);
    }

    // camera: origin3, lowerLeft3, horizontal3, vertical3 (DeviceCamera.hpp:5-11)
    int oracle_render(void* scene, const float* camera, uint32_t width, uint32_t height, uint32_t spp, uint32_t depth, uint32_t nee,
                      uint32_t poolSize, uint64_t maxSamples, int threads, int accumulationMode, float* sampleRadiance,
                      float* accumulation, uint32_t* framebuffer, uint32_t* queueLog, uint32_t queueLogCapacity, uint32_t* iterations,
                      uint64_t rngOffset, uint32_t rngPolicy, uint32_t lightMode)
    {
        auto* s = static_cast<oracle::Scene*>(scene);
        oracle::Camera cam{{camera[0], camera[1], camera[2]}, {camera[3], camera[4], camera[5]},
                           {camera[6], camera[7], camera[8]}, {camera[9], camera[10], camera[11]}};
        oracle::RenderSettings rs{width, height, spp, depth, nee, poolSize, maxSamples, threads, accumulationMode, rngOffset,
                                  rngPolicy, lightMode};
        return oracle::Render(*s, cam, rs, sampleRadiance, accumulation, framebuffer, queueLog, queueLogCapacity, iterations);
    }

    // MakeDeviceCamera (Renderer.cpp:237-257): fovY radians, aspect, position3, quaternion (w, x, y, z).
    void oracle_make_camera(float fovY, float aspect, const float* position, const float* quat, float* cameraOut)
    {
        float w = quat[0], x = quat[1], y = quat[2], z = quat[3];
        // glm::quat * vec3 rotation, expanded: v + 2w(q x v) + 2 q x (q x v)
        auto rotate = [&](oracle::float3 v)
        {
            oracle::float3 q = oracle::make_float3(x, y, z);
            oracle::float3 uv = oracle::cross(q, v);
            oracle::float3 uuv = oracle::cross(q, uv);
            return v + ((uv * w) + uuv) * 2.0f;
        };
        oracle::float3 forward = rotate(oracle::make_float3(0.0f, 0.0f, -1.0f));
        oracle::float3 right = rotate(oracle::make_float3(1.0f, 0.0f, 0.0f));
        oracle::float3 up = rotate(oracle::make_float3(0.0f, 1.0f, 0.0f));
        float halfH = std::tan(fovY * 0.5f);
        float halfW = halfH * aspect;
        oracle::float3 origin = oracle::make_float3(position[0], position[1], position[2]);
        oracle::float3 horizontal = 2.0f * halfW * right;
        oracle::float3 vertical = 2.0f * halfH * up;
        oracle::float3 llc = origin + forward - halfW * right - halfH * up;
        float out[12] = {origin.x, origin.y, origin.z, llc.x, llc.y, llc.z, horizontal.x, horizontal.y, horizontal.z, vertical.x, vertical.y, vertical.z};
        std::memcpy(cameraOut, out, sizeof(out));
    }
}
