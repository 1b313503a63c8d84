// Scene-upload kernels: triangle shading records, the emitter list and the light alias table.
//
// The reference builds these records on the host (Renderer.cpp:116-213, LightSampler.cpp:5-40,
// AliasTable.hpp:22-84), where every float operator rounds once and normalize() is
// v * (1 / sqrtf(dot(v, v))) (helper_math.h:78). This file is therefore compiled with
// -fmad=false and the IEEE math of pt_math.cuh in every build of the library, so the records,
// light areas and alias bins are the host's bits whichever arithmetic the wavefront kernels use.
#include "kernels.h"
#include "pt_math.cuh"

namespace pt
{
    __device__ __forceinline__ uint32_t scan_lane_id() { return threadIdx.x & 31u; }

    // ------------------------------------------------------------------ scene: lights and alias table on the device
    // LightSampler::BuildSync (LightSampler.cpp:5-40): emissive triangles in input order.
    __global__ void light_flag_kernel(const float4* shading, const MaterialDev* materials, uint32_t n, uint32_t* flags)
    {
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        {
            const uint32_t mat = __float_as_uint(shading[static_cast<size_t>(t) * 9 + 6].w);
            flags[t] = materials[mat].model == kModelEmissive ? 1u : 0u;
        }
    }

    // Light records, the area weight of each emitter (the reference's, LightSampler.cpp:16-19) and its
    // power weight for the production sampler: area x luminance of the emission constant (Rec. 709
    // weights, as Luminance in MaterialEval.cu), in FP64. An emitter whose emission comes from an image
    // texture gets area x 1: its mean texel is not known here, and any positive weight keeps NEE unbiased.
    __global__ void light_record_kernel(const float* positions, const float4* shading, const MaterialDev* materials,
                                        const MaterialTextures* textures, uint32_t n, const uint32_t* flags, const uint32_t* index,
                                        float4* lights, double* weights, double* powerWeights)
    {
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        {
            if (!flags[t]) continue;
            const float* p = positions + static_cast<size_t>(t) * 9;
            const float3 p0 = make_float3(p[0], p[1], p[2]);
            const float3 e1 = make_float3(p[3], p[4], p[5]) - p0;
            const float3 e2 = make_float3(p[6], p[7], p[8]) - p0;
            const float area = 0.5f * length(cross(e1, e2));
            const float4 g = shading[static_cast<size_t>(t) * 9 + 6];
            const uint32_t mat = __float_as_uint(g.w);
            const uint32_t li = index[t];
            float4* L = lights + static_cast<size_t>(li) * 7;
            L[0] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(t));
            L[1] = make_float4(e1.x, e1.y, e1.z, area);
            L[2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
            L[3] = make_float4(g.x, g.y, g.z, 0.0f);
            L[4] = make_float4(materials[mat].emission[0], materials[mat].emission[1], materials[mat].emission[2], 0.0f);
            // uv0, uv1 - uv0, uv2 - uv0 (LightSampler.cpp:28-30) and the material for its emission texture
            const float4 u01 = shading[static_cast<size_t>(t) * 9 + 7], u2 = shading[static_cast<size_t>(t) * 9 + 8];
            L[5] = make_float4(u01.x, u01.y, u01.z - u01.x, u01.w - u01.y);
            L[6] = make_float4(u2.x - u01.x, u2.y - u01.y, __uint_as_float(mat), 0.0f);
            weights[li] = static_cast<double>(area);
            const float* e = materials[mat].emission;
            const bool textured = textures != nullptr && textures[mat].tex[4] != 0;
            const double lum = textured ? 1.0
                                        : 0.2126 * static_cast<double>(e[0]) + 0.7152 * static_cast<double>(e[1]) +
                                              0.0722 * static_cast<double>(e[2]);
            powerWeights[li] = lum * static_cast<double>(area);
        }
    }

    // Triangle records of the shading pass (Renderer.cpp:159-213): normals, tangents, geometric
    // normal normalize(cross(e1, e2)), material, uvs; 144 bytes per triangle.
    __global__ void shading_record_kernel(const float* positions, const float* normals, const float* tangents, const float* uvs,
                                          const uint32_t* materialIds, uint32_t n, float4* shading)
    {
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        {
            const float* p = positions + static_cast<size_t>(t) * 9;
            const float* nn = normals + static_cast<size_t>(t) * 9;
            const float* tt = tangents + static_cast<size_t>(t) * 12;
            const float* uu = uvs + static_cast<size_t>(t) * 6;
            const float3 p0 = make_float3(p[0], p[1], p[2]);
            const float3 e1 = make_float3(p[3], p[4], p[5]) - p0;
            const float3 e2 = make_float3(p[6], p[7], p[8]) - p0;
            const float3 gn = normalize(cross(e1, e2));
            float4* S = shading + static_cast<size_t>(t) * 9;
            S[0] = make_float4(nn[0], nn[1], nn[2], 0.0f);
            S[1] = make_float4(nn[3], nn[4], nn[5], 0.0f);
            S[2] = make_float4(nn[6], nn[7], nn[8], 0.0f);
            S[3] = make_float4(tt[0], tt[1], tt[2], tt[3]);
            S[4] = make_float4(tt[4], tt[5], tt[6], tt[7]);
            S[5] = make_float4(tt[8], tt[9], tt[10], tt[11]);
            S[6] = make_float4(gn.x, gn.y, gn.z, __uint_as_float(materialIds[t]));
            S[7] = make_float4(uu[0], uu[1], uu[2], uu[3]);
            S[8] = make_float4(uu[4], uu[5], 0.0f, 0.0f);
        }
    }

    // Exclusive scan, one block of 1024 threads per 1024 elements; block totals out.
    template <typename T>
    __global__ void scan_block_kernel(const T* in, T* out, T* blockSums, uint32_t n)
    {
        __shared__ T warpSums[32];
        const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
        const T x = i < n ? in[i] : T(0);
        T v = x;
        const uint32_t lane = scan_lane_id(), warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1)
        {
            const T y = __shfl_up_sync(0xFFFFFFFFu, v, o);
            if (lane >= static_cast<uint32_t>(o)) v = v + y;
        }
        if (lane == 31) warpSums[warp] = v;
        __syncthreads();
        if (warp == 0)
        {
            T w = warpSums[lane];
            for (int o = 1; o < 32; o <<= 1)
            {
                const T y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= static_cast<uint32_t>(o)) w = w + y;
            }
            warpSums[lane] = w;
        }
        __syncthreads();
        const T warpOffset = warp > 0 ? warpSums[warp - 1] : T(0);
        const T inclusive = v + warpOffset;
        if (i < n) out[i] = inclusive - x;
        if (threadIdx.x == 1023u && blockSums) blockSums[blockIdx.x] = inclusive;
    }

    template <typename T>
    __global__ void scan_add_kernel(T* data, const T* blockOffsets, uint32_t n)
    {
        const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
        if (i < n && blockIdx.x > 0) data[i] = data[i] + blockOffsets[blockIdx.x];
    }

    __global__ void scan_total_kernel(const uint32_t* flags, const uint32_t* excl, uint32_t n, uint32_t* total)
    {
        *total = n ? excl[n - 1] + flags[n - 1] : 0u;
    }

    // AliasTable<uint32_t>::BuildSync (AliasTable.hpp:22-84): p_i = w_i / sum (sum accumulated in
    // FP64 by the device prefix sum, rounded to float), pHat = p * n, then the reference's
    // sequential pairing of the last light (under) and last heavy (over) outcome. The pairing is
    // inherently ordered, so one thread runs it; under/over stacks live in the scratch arrays.
    __global__ void alias_build_kernel(const double* weights, const double* prefix, uint32_t n, uint4* bins,
                                       uint32_t* stackIndex, float* stackValue)
    {
        if (blockIdx.x != 0 || threadIdx.x != 0 || n == 0) return;
        const float sum = static_cast<float>(prefix[n - 1] + weights[n - 1]);
        uint32_t* underIdx = stackIndex;
        uint32_t* overIdx = stackIndex + n;
        float* underVal = stackValue;
        float* overVal = stackValue + n;
        uint32_t nu = 0, no = 0;
        for (uint32_t i = 0; i < n; i++)
        {
            const float p = static_cast<float>(weights[i]) / sum;
            bins[i] = make_uint4(__float_as_uint(0.0f), __float_as_uint(p), 0u, i);
            const float pHat = p * static_cast<float>(n);
            if (pHat < 1)
            {
                underIdx[nu] = i;
                underVal[nu] = pHat;
                nu++;
            }
            else
            {
                overIdx[no] = i;
                overVal[no] = pHat;
                no++;
            }
        }
        while (nu > 0 && no > 0)
        {
            nu--;
            no--;
            const uint32_t ui = underIdx[nu], oi = overIdx[no];
            const float uv = underVal[nu], ov = overVal[no];
            bins[ui].x = __float_as_uint(uv);
            bins[ui].z = oi;
            const float excess = uv + ov - 1;
            if (excess < 1)
            {
                underIdx[nu] = oi;
                underVal[nu] = excess;
                nu++;
            }
            else
            {
                overIdx[no] = oi;
                overVal[no] = excess;
                no++;
            }
        }
        while (no > 0)
        {
            no--;
            bins[overIdx[no]].x = __float_as_uint(1.0f);
            bins[overIdx[no]].z = kInvalid;
        }
        while (nu > 0)
        {
            nu--;
            bins[underIdx[nu]].x = __float_as_uint(1.0f);
            bins[underIdx[nu]].z = kInvalid;
        }
    }

    // ------------------------------------------------------------------ parallel alias table (power weights)
    // The sequential sweep of an alias table (Walker, "An efficient method for generating discrete random
    // variables with general distributions", ACM TOMS 1977; the sweeping form of Huebschle-Schneider and
    // Sanders, "Parallel Weighted Random Sampling", ESA 2019) visits light items (pHat = w n / W < 1) and
    // heavy items (pHat >= 1) in input order. At state (i lights done, j heavies done) heavy j donates;
    // with D_i = sum of (1 - pHat) over the first i lights and E_j = sum of (pHat - 1) over the first j
    // heavies, heavy j's residual is E_(j+1) - D_i + 1, and the next step fills light i's bucket (alias
    // heavy j) if D_i < E_(j+1), else closes heavy j's bucket (q = its residual, alias heavy j+1). The
    // step order is therefore the merge of the sorted keys D_i (lights) and E_(j+1) (heavies; first on
    // ties), so the state after k steps is found by a binary search over the prefix sums (merge path) and
    // threads fill disjoint ranges of steps independently. Every q comes from the FP64 prefix sums, never
    // from a running subtraction. The prefix sums run over all n items in input order, with zeros for the
    // other class: D_i is the exclusive sum at the position of the i-th light, E_j at the j-th heavy. A
    // running maximum over each prefix array keeps the keys sorted (a tree-ordered FP64 sum of non-negative
    // terms is not monotone by construction), which makes every thread's split the sequential merge's state.
    struct AliasSplit
    {
        uint32_t lights, heavies;
        double deficitTotal, excessTotal;
    };

    // pHat of every item (power weights, or area weights when no emitter has positive power), its class,
    // its deficit or excess in input order; the bins get their pmf and value (leftover form: q 1, no alias).
    __global__ void alias_classify_kernel(const double* weights, const double* prefix, const double* fallback, const double* fallbackPrefix,
                                          uint32_t n, double* pHat, uint32_t* lightFlag, double* deficit, double* excess, uint4* bins)
    {
        const double totalPower = prefix[n - 1] + weights[n - 1];
        const bool power = totalPower > 0.0 && totalPower < 1e300;
        const double* w = power ? weights : fallback;
        const double total = power ? totalPower : fallbackPrefix[n - 1] + fallback[n - 1];
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        {
            const double ph = w[k] * static_cast<double>(n) / total;
            const bool light = ph < 1.0;
            pHat[k] = ph;
            lightFlag[k] = light ? 1u : 0u;
            deficit[k] = light ? 1.0 - ph : 0.0;
            excess[k] = light ? 0.0 : ph - 1.0;
            bins[k] = make_uint4(__float_as_uint(1.0f), __float_as_uint(static_cast<float>(w[k] / total)), kInvalid, k);
        }
    }

    // Lights and heavies in input order (lightPos = exclusive scan of lightFlag).
    __global__ void alias_partition_kernel(const uint32_t* lightFlag, const uint32_t* lightPos, uint32_t n, uint32_t* lightIdx, uint32_t* heavyIdx)
    {
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        {
            const uint32_t lp = lightPos[k];
            if (lightFlag[k]) lightIdx[lp] = k;
            else heavyIdx[k - lp] = k;
        }
    }

    __global__ void alias_totals_kernel(const uint32_t* lightFlag, const uint32_t* lightPos, const double* deficit, const double* deficitPrefix,
                                        const double* excess, const double* excessPrefix, uint32_t n, AliasSplit* split)
    {
        AliasSplit a;
        a.lights = lightPos[n - 1] + lightFlag[n - 1];
        a.heavies = n - a.lights;
        a.deficitTotal = deficitPrefix[n - 1] + deficit[n - 1];
        a.excessTotal = excessPrefix[n - 1] + excess[n - 1];
        *split = a;
    }

    constexpr uint32_t kSweepSteps = 32;  // buckets closed per thread

    __global__ void alias_sweep_kernel(const double* pHat, const uint32_t* lightIdx, const double* deficitPrefix, const uint32_t* heavyIdx,
                                       const double* excessPrefix, const AliasSplit* splitPtr, uint32_t n, uint4* bins)
    {
        const AliasSplit sp = *splitPtr;
        const uint32_t a = sp.lights, b = sp.heavies;
        // D_i (i <= a) and E_j (j <= b)
        auto D = [&](uint32_t i) { return i < a ? deficitPrefix[lightIdx[i]] : sp.deficitTotal; };
        auto E = [&](uint32_t j) { return j < b ? excessPrefix[heavyIdx[j]] : sp.excessTotal; };
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; static_cast<uint64_t>(t) * kSweepSteps < n; t += gridDim.x * blockDim.x)
        {
            const uint32_t k0 = t * kSweepSteps;
            const uint32_t k1 = n - k0 > kSweepSteps ? k0 + kSweepSteps : n;
            // lights among the first k0 steps: the largest i for which light i-1 precedes heavy k0 - i
            uint32_t lo = k0 > b ? k0 - b : 0u, hi = k0 < a ? k0 : a;
            while (lo < hi)
            {
                const uint32_t mid = (lo + hi + 1u) >> 1;
                const uint32_t j = k0 - mid;
                if (j >= b || D(mid - 1u) < E(j + 1u)) lo = mid;
                else hi = mid - 1u;
            }
            uint32_t i = lo, j = k0 - lo;
            for (uint32_t k = k0; k < k1; k++)
            {
                if (i < a && (j >= b || D(i) < E(j + 1u)))
                {
                    // light i: its own share q = pHat, the rest from heavy j (none left: leftover, q 1)
                    const uint32_t item = lightIdx[i];
                    if (j < b)
                    {
                        bins[item].x = __float_as_uint(static_cast<float>(pHat[item]));
                        bins[item].z = heavyIdx[j];
                    }
                    i++;
                }
                else
                {
                    // heavy j closes: its residual, topped up by heavy j+1 (the last heavy is a leftover, q 1)
                    const uint32_t item = heavyIdx[j];
                    if (j + 1u < b)
                    {
                        const double residual = E(j + 1u) - D(i) + 1.0;
                        const float q = static_cast<float>(residual < 0.0 ? 0.0 : (residual > 1.0 ? 1.0 : residual));
                        bins[item].x = __float_as_uint(q);
                        bins[item].z = heavyIdx[j + 1u];
                    }
                    j++;
                }
            }
        }
    }

    cudaError_t launch_shading_records(const float* positions, const float* normals, const float* tangents, const float* uvs,
                                       const uint32_t* materialIds, uint32_t n, float4* shading, cudaStream_t s)
    {
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        shading_record_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(positions, normals, tangents, uvs, materialIds, n, shading);
        return cudaGetLastError();
    }

    // Running maximum in place (inclusive), one block of 1024 threads per 1024 elements. Maximum is exact,
    // so the result does not depend on the order of the tree.
    __global__ void running_max_block_kernel(double* data, double* blockMax, uint32_t n)
    {
        __shared__ double warpMax[32];
        const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
        double v = i < n ? data[i] : -INFINITY;
        const uint32_t lane = scan_lane_id(), warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1)
        {
            const double y = __shfl_up_sync(0xFFFFFFFFu, v, o);
            if (lane >= static_cast<uint32_t>(o)) v = fmax(v, y);
        }
        if (lane == 31) warpMax[warp] = v;
        __syncthreads();
        if (warp == 0)
        {
            double w = warpMax[lane];
            for (int o = 1; o < 32; o <<= 1)
            {
                const double y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= static_cast<uint32_t>(o)) w = fmax(w, y);
            }
            warpMax[lane] = w;
        }
        __syncthreads();
        if (warp > 0) v = fmax(v, warpMax[warp - 1]);
        if (i < n) data[i] = v;
        if (threadIdx.x == 1023u && blockMax) blockMax[blockIdx.x] = v;
    }

    __global__ void running_max_apply_kernel(double* data, const double* blockMax, uint32_t n)
    {
        const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
        if (i < n && blockIdx.x > 0) data[i] = fmax(data[i], blockMax[blockIdx.x - 1]);
    }

    static cudaError_t running_max(double* data, uint32_t n, double* scratch, cudaStream_t s)
    {
        if (n == 0) return cudaSuccess;
        const uint32_t blocks = (n + 1023) / 1024;
        running_max_block_kernel<<<blocks, 1024, 0, s>>>(data, blocks > 1 ? scratch : nullptr, n);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess || blocks == 1) return e;
        e = running_max(scratch, blocks, scratch + blocks, s);
        if (e != cudaSuccess) return e;
        running_max_apply_kernel<<<blocks, 1024, 0, s>>>(data, scratch, n);
        return cudaGetLastError();
    }

    template <typename T>
    static cudaError_t exclusive_scan(const T* in, T* out, uint32_t n, T* scratch, cudaStream_t s)
    {
        // scratch: >= ceil(n/1024) + ceil(n/1024^2) + ... + 3 elements
        if (n == 0) return cudaSuccess;
        const uint32_t blocks = (n + 1023) / 1024;
        T* sums = scratch;
        scan_block_kernel<T><<<blocks, 1024, 0, s>>>(in, out, blocks > 1 ? sums : nullptr, n);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess || blocks == 1) return e;
        e = exclusive_scan<T>(sums, sums, blocks, scratch + blocks, s);
        if (e != cudaSuccess) return e;
        scan_add_kernel<T><<<blocks, 1024, 0, s>>>(out, sums, n);
        return cudaGetLastError();
    }

    cudaError_t launch_light_build(const float4* shading, const MaterialDev* materials, uint32_t n,
                                   uint32_t* flags, uint32_t* index, uint32_t* scanScratch, uint32_t* lightCountDev, cudaStream_t s)
    {
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        light_flag_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(shading, materials, n, flags);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        e = exclusive_scan<uint32_t>(flags, index, n, scanScratch, s);
        if (e != cudaSuccess) return e;
        scan_total_kernel<<<1, 1, 0, s>>>(flags, index, n, lightCountDev);
        return cudaGetLastError();
    }

    cudaError_t launch_light_records(const float* positions, const float4* shading, const MaterialDev* materials,
                                     const MaterialTextures* textures, uint32_t n, const uint32_t* flags, const uint32_t* index,
                                     float4* lights, double* weights, double* powerWeights, cudaStream_t s)
    {
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        light_record_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(positions, shading, materials, textures, n, flags, index, lights, weights,
                                                                powerWeights);
        return cudaGetLastError();
    }

    cudaError_t launch_alias_build(const double* weights, uint32_t n, double* prefix, double* scanScratch, uint4* bins,
                                   uint32_t* stackIndex, float* stackValue, cudaStream_t s)
    {
        if (n == 0) return cudaSuccess;
        cudaError_t e = exclusive_scan<double>(weights, prefix, n, scanScratch, s);
        if (e != cudaSuccess) return e;
        alias_build_kernel<<<1, 32, 0, s>>>(weights, prefix, n, bins, stackIndex, stackValue);
        return cudaGetLastError();
    }

    // Power-weighted alias table, built in parallel (alias_sweep_kernel); falls back to the area weights when
    // no emitter has positive power. Scratch of alias_power_scratch_bytes(n) bytes, 16-byte aligned.
    size_t alias_power_scratch_bytes(uint32_t n)
    {
        const size_t m = (static_cast<size_t>(n) + 1) & ~static_cast<size_t>(1);  // even, so the u32 arrays keep 8-byte alignment
        return m * 8 * 7 + m * 4 * 4 + scan_scratch_elements(n) * 8 + sizeof(AliasSplit) + 16;
    }

    cudaError_t launch_alias_build_power(const double* weights, const double* areaWeights, uint32_t n, void* scratch, uint4* bins,
                                         cudaStream_t s)
    {
        if (n == 0) return cudaSuccess;
        const size_t m = (static_cast<size_t>(n) + 1) & ~static_cast<size_t>(1);
        double* prefix = static_cast<double*>(scratch);
        double* areaPrefix = prefix + m;
        double* pHat = areaPrefix + m;
        double* deficit = pHat + m;
        double* excess = deficit + m;
        double* deficitPrefix = excess + m;
        double* excessPrefix = deficitPrefix + m;
        uint32_t* lightFlag = reinterpret_cast<uint32_t*>(excessPrefix + m);
        uint32_t* lightPos = lightFlag + m;
        uint32_t* lightIdx = lightPos + m;
        uint32_t* heavyIdx = lightIdx + m;
        double* scan = reinterpret_cast<double*>(heavyIdx + m);
        AliasSplit* split = reinterpret_cast<AliasSplit*>(scan + scan_scratch_elements(n));
        const uint32_t blocks = (n + 255) / 256 < 16384 ? (n + 255) / 256 : 16384;
        cudaError_t e;
        if ((e = exclusive_scan<double>(weights, prefix, n, scan, s)) != cudaSuccess) return e;
        if ((e = exclusive_scan<double>(areaWeights, areaPrefix, n, scan, s)) != cudaSuccess) return e;
        alias_classify_kernel<<<blocks, 256, 0, s>>>(weights, prefix, areaWeights, areaPrefix, n, pHat, lightFlag, deficit, excess, bins);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = exclusive_scan<uint32_t>(lightFlag, lightPos, n, reinterpret_cast<uint32_t*>(scan), s)) != cudaSuccess) return e;
        if ((e = exclusive_scan<double>(deficit, deficitPrefix, n, scan, s)) != cudaSuccess) return e;
        if ((e = exclusive_scan<double>(excess, excessPrefix, n, scan, s)) != cudaSuccess) return e;
        // the tree-ordered sums of non-negative terms can step down by an ulp; the merge needs sorted keys
        if ((e = running_max(deficitPrefix, n, scan, s)) != cudaSuccess) return e;
        if ((e = running_max(excessPrefix, n, scan, s)) != cudaSuccess) return e;
        alias_partition_kernel<<<blocks, 256, 0, s>>>(lightFlag, lightPos, n, lightIdx, heavyIdx);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        alias_totals_kernel<<<1, 1, 0, s>>>(lightFlag, lightPos, deficit, deficitPrefix, excess, excessPrefix, n, split);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const uint32_t threads = (n + kSweepSteps - 1) / kSweepSteps;
        const uint32_t sweepBlocks = (threads + 127) / 128 < 16384 ? (threads + 127) / 128 : 16384;
        alias_sweep_kernel<<<sweepBlocks, 128, 0, s>>>(pHat, lightIdx, deficitPrefix, heavyIdx, excessPrefix, split, n, bins);
        return cudaGetLastError();
    }

    size_t scan_scratch_elements(uint32_t n)
    {
        size_t total = 3;
        uint32_t m = n;
        while (m > 1)
        {
            m = (m + 1023) / 1024;
            total += m;
        }
        return total;
    }
}
