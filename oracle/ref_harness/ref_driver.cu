// ORACLE — test infrastructure only: driver of the reference's own GPU kernels.
//
// The reference's kernel translation units (Core/Source/Graphics/Cuda/PathTracing/Kernels/
// Intersect.cu, Iteration.cu, PathGeneration.cu, MaterialEval.cu) and its BVH builder
// (Core/Source/Graphics/Cuda/Bvh/HostBvh.cpp) are compiled unmodified from the reference tree by
// oracle/ref_harness/Makefile. The reference's host classes around them need C++23, spdlog and
// entt, which are absent, so this driver (C++17, written for this harness) stands in for them:
//  * it builds the reference's POD views (RayQueueView, MaterialEvalQueueView, ShadowRayQueueView,
//    RegenQueueView, PathPoolView, IntersectionBvhView, LightSamplerView) over plain cudaMalloc'd
//    structure-of-arrays buffers;
//  * it restates BuildTriangles (Renderer.cpp:159-213), LightSampler::BuildSync
//    (LightSampler.cpp:5-40), AliasTable::BuildSync (AliasTable.hpp:22-84), the DFS flattening of
//    DeviceBvh::BuildFlattenSync (DeviceBvh.cpp:7-52), the 1x1 material textures of
//    Manager::ImportMaterial / Texture::Create2D (Manager.cpp:321-380, Texture.cpp:65-189) and the
//    PostprocessKernel tone map (Image.cu:22-54, which needs C++20 and is not compiled);
//  * it replays Renderer::RenderFrame's launch sequence (Renderer.cpp:468-647) through the
//    reference's launchers (Kernels/Launchers.hpp).
// It is used by tests/ to pin the oracle against the reference, and by bench.py to time the
// reference's own build on the same GPU. It is never part of the product.
#include <Core/Graphics/Cuda/Bvh/HostBvh.hpp>
#include <Core/Graphics/Cuda/PathTracing/Kernels/Launchers.hpp>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

using namespace Core::Graphics::Cuda;

namespace
{
    struct RefMaterial  // 48 bytes, see oracle/ref_harness.py
    {
        uint32_t model;          // GlobalShadingModel
        uint32_t colorU8;        // r | g << 8 | b << 16, sRGB texel
        uint32_t specularU8;     // sRGB texel
        uint32_t shininessU8;    // linear texel
        uint32_t rmaU8;          // linear texel
        uint32_t normalU8;       // linear texel
        float emission[3];       // float32 texel
        float ior;
        float transmission;
        uint32_t pad;
    };
    static_assert(sizeof(RefMaterial) == 48, "RefMaterial layout");

    template <typename T>
    T* dalloc(size_t n)
    {
        T* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
        return p;
    }

    struct Texture
    {
        cudaArray_t array = nullptr;
        cudaTextureObject_t object = 0;
    };

    // Texture::Create2D descriptors (Texture.cpp:65-87): clamp, linear filter, normalised coordinates.
    bool make_u8_texture(Texture& t, const uint8_t* rgba, int channels, bool srgb)
    {
        cudaChannelFormatDesc desc = channels == 1 ? cudaCreateChannelDesc<uchar1>() : cudaCreateChannelDesc<uchar4>();
        if (cudaMallocArray(&t.array, &desc, 1, 1) != cudaSuccess) return false;
        if (cudaMemcpy2DToArray(t.array, 0, 0, rgba, channels, channels, 1, cudaMemcpyHostToDevice) != cudaSuccess) return false;
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = t.array;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.normalizedCoords = 1;
        td.sRGB = srgb ? 1 : 0;
        td.readMode = cudaReadModeNormalizedFloat;
        return cudaCreateTextureObject(&t.object, &res, &td, nullptr) == cudaSuccess;
    }

    // Image texture with Texture::Create2D's descriptors; channels 1 or 4 (3-channel data is
    // expanded by the caller), format 0 = u8 sRGB, 1 = u8 linear, 2 = f32.
    bool make_image_texture(Texture& t, const void* data, int w, int h, int channels, int format)
    {
        const bool u8 = format != 2;
        cudaChannelFormatDesc desc = u8 ? (channels == 1 ? cudaCreateChannelDesc<uchar1>() : cudaCreateChannelDesc<uchar4>())
                                        : (channels == 1 ? cudaCreateChannelDesc<float1>() : cudaCreateChannelDesc<float4>());
        if (cudaMallocArray(&t.array, &desc, w, h) != cudaSuccess) return false;
        const size_t pitch = static_cast<size_t>(w) * channels * (u8 ? 1 : 4);
        if (cudaMemcpy2DToArray(t.array, 0, 0, data, pitch, pitch, h, cudaMemcpyHostToDevice) != cudaSuccess) return false;
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = t.array;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.normalizedCoords = 1;
        td.sRGB = format == 0 ? 1 : 0;
        td.readMode = u8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        return cudaCreateTextureObject(&t.object, &res, &td, nullptr) == cudaSuccess;
    }

    struct ImageDesc  // 24 bytes, see oracle/ref_harness.py
    {
        uint32_t width, height, channels, format;
        const void* data;  // channels 1 or 4
    };

    bool make_f32_texture(Texture& t, const float* rgba)
    {
        cudaChannelFormatDesc desc = cudaCreateChannelDesc<float4>();
        if (cudaMallocArray(&t.array, &desc, 1, 1) != cudaSuccess) return false;
        if (cudaMemcpy2DToArray(t.array, 0, 0, rgba, 16, 16, 1, cudaMemcpyHostToDevice) != cudaSuccess) return false;
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = t.array;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModeLinear;
        td.normalizedCoords = 1;
        td.sRGB = 0;
        td.readMode = cudaReadModeElementType;
        return cudaCreateTextureObject(&t.object, &res, &td, nullptr) == cudaSuccess;
    }

    struct Queues
    {
        uint32_t capacity = 0;
        std::vector<void*> allocations;
        uint32_t* counters = nullptr;  // [0,1] ray queues, [2..7] material queues, [8] shadow, [9] regen
        RayQueueView rays[2];
        MaterialEvalQueueViewsProvider materials;
        ShadowRayQueueView shadow;
        RegenQueueView regen;
        Pixel* pixels = nullptr;
        Random* randoms = nullptr;

        // Allocations are made one statement at a time (function-argument evaluation order is
        // unspecified), so allocations[] holds each queue's arrays in constructor order.
        void* f(size_t bytesPerEntry)
        {
            void* p = nullptr;
            if (cudaMalloc(&p, bytesPerEntry * (capacity ? capacity : 1)) != cudaSuccess) p = nullptr;
            allocations.push_back(p);
            return p;
        }
        RayQueueView make_ray_queue(uint32_t* size)
        {
            void* v[15];
            for (int k = 0; k < 15; k++) v[k] = f(k == 6 ? sizeof(bool) : 4);
            return RayQueueView(size, capacity, (uint32_t*)v[0], (uint32_t*)v[1], (float*)v[2], (float*)v[3], (float*)v[4], (float*)v[5],
                                (bool*)v[6], (float*)v[7], (float*)v[8], (float*)v[9], (float*)v[10], (float*)v[11], (float*)v[12],
                                (float*)v[13], (float*)v[14]);
        }
        MaterialEvalQueueView make_material_queue(uint32_t* size)
        {
            void* v[18];
            for (int k = 0; k < 18; k++) v[k] = f(k == 6 ? sizeof(bool) : 4);
            return MaterialEvalQueueView(size, capacity, (uint32_t*)v[0], (uint32_t*)v[1], (float*)v[2], (float*)v[3], (float*)v[4],
                                         (float*)v[5], (bool*)v[6], (float*)v[7], (float*)v[8], (float*)v[9], (float*)v[10],
                                         (float*)v[11], (float*)v[12], (float*)v[13], (float*)v[14], (uint32_t*)v[15], (float*)v[16],
                                         (float*)v[17]);
        }
        bool allocate(uint32_t cap)
        {
            capacity = cap;
            counters = static_cast<uint32_t*>(f(0));
            cudaFree(counters);
            allocations.pop_back();
            if (cudaMalloc(&counters, 64) != cudaSuccess) return false;
            allocations.push_back(counters);
            rays[0] = make_ray_queue(counters + 0);
            rays[1] = make_ray_queue(counters + 1);
            for (int m = 0; m < 6; m++) materials.At(m) = make_material_queue(counters + 2 + m);
            void* v[12];
            for (int k = 0; k < 12; k++) v[k] = f(4);
            shadow = ShadowRayQueueView(counters + 8, cap, (uint32_t*)v[0], (float*)v[1], (float*)v[2], (float*)v[3], (float*)v[4],
                                        (float*)v[5], (float*)v[6], (float*)v[7], (float*)v[8], (float*)v[9], (float*)v[10],
                                        (float*)v[11]);
            regen = RegenQueueView(counters + 9, cap, static_cast<uint32_t*>(f(4)));
            pixels = static_cast<Pixel*>(f(sizeof(Pixel)));
            randoms = static_cast<Random*>(f(sizeof(Random)));
            for (void* p : allocations)
                if (!p) return false;
            return cudaMemset(counters, 0, 64) == cudaSuccess;
        }
        ~Queues()
        {
            for (void* p : allocations) cudaFree(p);
        }
        PathPoolView pool() const
        {
            return PathPoolView{Runtime::DeviceBuffer1DView<Pixel>(pixels, capacity), Runtime::DeviceBuffer1DView<Random>(randoms, capacity)};
        }
    };

    // MaterialEvalQueueView fields read back for the ray-batch mode (the SoA arrays are private;
    // the constructor's argument order fixes which allocation holds which field).
    struct Scene
    {
        uint32_t triangleCount = 0, nodeCount = 0, depth = 0, lightCount = 0, materialCount = 0;
        DeviceBvhNode* nodes = nullptr;
        TriangleIntersection* isect = nullptr;
        TriangleShading* shading = nullptr;
        Material* materials = nullptr;
        LightTriangle* lights = nullptr;
        Bin<uint32_t>* bins = nullptr;
        std::vector<uint32_t> order;              // BVH position -> input index
        std::vector<Texture> textures;
        std::vector<Material> hostMaterials;
        uint32_t materialCounts[6] = {};
        Queues* queues = nullptr;
        ~Scene()
        {
            delete queues;
            cudaFree(nodes);
            cudaFree(isect);
            cudaFree(shading);
            cudaFree(materials);
            cudaFree(lights);
            cudaFree(bins);
            for (Texture& t : textures)
            {
                if (t.object) cudaDestroyTextureObject(t.object);
                if (t.array) cudaFreeArray(t.array);
            }
        }
    };

    // DeviceBvh.cpp:7-19 (DFS pre-order)
    uint32_t Flatten(const HostBvhNode& node, std::vector<DeviceBvhNode>& nodes)
    {
        uint32_t index = static_cast<uint32_t>(nodes.size());
        nodes.emplace_back(node.bounds, PathTracerDefaults::InvalidIndex, PathTracerDefaults::InvalidIndex, node.first, node.count);
        if (node.left && node.right)
        {
            nodes[index].left = Flatten(*node.left, nodes);
            nodes[index].right = Flatten(*node.right, nodes);
        }
        return index;
    }

    // AliasTable.hpp:22-84 restated (the class needs C++23).
    std::vector<Bin<uint32_t>> BuildAlias(const std::vector<float>& weights, const std::vector<uint32_t>& values)
    {
        float sum = static_cast<float>(std::accumulate(weights.begin(), weights.end(), 0.0));
        std::vector<Bin<uint32_t>> bins(weights.size());
        for (uint32_t i = 0; i < weights.size(); i++)
            bins[i] = Bin<uint32_t>{0.0f, weights[i] / sum, 0u, values[i]};
        struct Outcome { float pHat; uint32_t index; };
        std::vector<Outcome> under, over;
        for (uint32_t i = 0; i < bins.size(); i++)
        {
            float pHat = bins[i].p * bins.size();
            if (pHat < 1) under.push_back(Outcome{pHat, i});
            else over.push_back(Outcome{pHat, i});
        }
        while (!under.empty() && !over.empty())
        {
            Outcome un = under.back(), ov = over.back();
            under.pop_back();
            over.pop_back();
            bins[un.index].q = un.pHat;
            bins[un.index].alias = ov.index;
            float pExcess = un.pHat + ov.pHat - 1;
            if (pExcess < 1) under.push_back(Outcome{pExcess, ov.index});
            else over.push_back(Outcome{pExcess, ov.index});
        }
        while (!over.empty())
        {
            Outcome ov = over.back();
            over.pop_back();
            bins[ov.index].q = 1;
            bins[ov.index].alias = PathTracerDefaults::InvalidIndex;
        }
        while (!under.empty())
        {
            Outcome un = under.back();
            under.pop_back();
            bins[un.index].q = 1;
            bins[un.index].alias = PathTracerDefaults::InvalidIndex;
        }
        return bins;
    }

    __global__ void sample_material_kernel(const Material* materials, uint32_t n, float* out)
    {
        uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n) return;
        const Material m = materials[i];
        const float2 uv = make_float2(0.5f, 0.5f);
        float* o = out + static_cast<size_t>(i) * 20;
        float4 c = m.color.Sample(uv), s = m.specular.Sample(uv), r = m.rma.Sample(uv), e = m.emission.Sample(uv), nm = m.normal.Sample(uv);
        float sh = m.shininess.Sample(uv.x, uv.y);
        o[1] = c.x; o[2] = c.y; o[3] = c.z;
        o[4] = s.x; o[5] = s.y; o[6] = s.z;
        o[7] = sh;
        o[8] = r.x; o[9] = r.y; o[10] = r.z;
        o[11] = e.x; o[12] = e.y; o[13] = e.z;
        o[14] = nm.x; o[15] = nm.y; o[16] = nm.z;
        o[17] = m.ior;
        o[18] = m.transmission;
        o[19] = 0.0f;
    }

    void unpack_rgb(uint32_t v, uint8_t* out4)
    {
        out4[0] = v & 0xFF;
        out4[1] = (v >> 8) & 0xFF;
        out4[2] = (v >> 16) & 0xFF;
        out4[3] = 255;
    }
}

extern "C"
{
    void ref_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

    void* ref_scene_create(uint32_t n, const float* positions, const float* normals, const float* tangents, const float* uvs,
                           const uint32_t* materialIds, uint32_t materialCount, const void* materialsIn, int* status,
                           uint32_t imageCount, const void* imagesIn, const int32_t* materialImages)
    {
        const ImageDesc* images = static_cast<const ImageDesc*>(imagesIn);
        *status = 1;
        auto* scene = new Scene();
        const RefMaterial* mats = static_cast<const RefMaterial*>(materialsIn);
        scene->triangleCount = n;
        scene->materialCount = materialCount;
        // materials as 1x1 textures (Manager.cpp:321-380)
        for (uint32_t m = 0; m < materialCount; m++)
        {
            const RefMaterial& rm = mats[m];
            Texture color, spec, shin, rma, emis, norm;
            uint8_t px[4];
            unpack_rgb(rm.colorU8, px);
            bool ok = make_u8_texture(color, px, 4, true);
            unpack_rgb(rm.specularU8, px);
            ok = ok && make_u8_texture(spec, px, 4, true);
            uint8_t sh = static_cast<uint8_t>(rm.shininessU8 & 0xFF);
            ok = ok && make_u8_texture(shin, &sh, 1, false);
            unpack_rgb(rm.rmaU8, px);
            ok = ok && make_u8_texture(rma, px, 4, false);
            float e[4] = {rm.emission[0], rm.emission[1], rm.emission[2], 1.0f};
            ok = ok && make_f32_texture(emis, e);
            unpack_rgb(rm.normalU8, px);
            ok = ok && make_u8_texture(norm, px, 4, false);
            // image textures replace the slot's 1x1 texel (Manager.cpp:337-355: file texture or pixel texture)
            Texture* slots[6] = {&color, &spec, &shin, &rma, &emis, &norm};
            if (materialImages)
                for (int k = 0; k < 6; k++)
                {
                    const int32_t img = materialImages[static_cast<size_t>(m) * 6 + k];
                    if (img < 0 || static_cast<uint32_t>(img) >= imageCount) continue;
                    Texture tex;
                    const ImageDesc& d = images[img];
                    ok = ok && make_image_texture(tex, d.data, static_cast<int>(d.width), static_cast<int>(d.height),
                                                  static_cast<int>(d.channels), static_cast<int>(d.format));
                    scene->textures.push_back(*slots[k]);  // keep the replaced 1x1 texture for cleanup
                    *slots[k] = tex;
                }
            for (Texture* t : {&color, &spec, &shin, &rma, &emis, &norm}) scene->textures.push_back(*t);
            if (!ok)
            {
                delete scene;
                return nullptr;
            }
            scene->hostMaterials.push_back(Material{TextureView<float4>(color.object), TextureView<float4>(spec.object),
                                                    TextureView<float>(shin.object), TextureView<float4>(rma.object),
                                                    TextureView<float4>(emis.object), TextureView<float4>(norm.object), rm.ior,
                                                    rm.transmission});
            scene->materialCounts[std::min<uint32_t>(rm.model, 5)]++;
        }
        // BuildTriangles (Renderer.cpp:159-213) on already world-space data; the input index rides in
        // normals[0].w, which the kernels never read, to recover the BVH permutation.
        std::vector<Triangle> triangles(n);
        for (uint32_t t = 0; t < n; t++)
        {
            float3 p[3];
            for (int k = 0; k < 3; k++)
            {
                const float* pp = positions + (static_cast<size_t>(t) * 3 + k) * 3;
                const float* nn = normals + (static_cast<size_t>(t) * 3 + k) * 3;
                const float* tt = tangents + (static_cast<size_t>(t) * 3 + k) * 4;
                const float* uu = uvs + (static_cast<size_t>(t) * 3 + k) * 2;
                p[k] = make_float3(pp[0], pp[1], pp[2]);
                triangles[t].shading.normals[k] = make_float4(nn[0], nn[1], nn[2], 0.0f);
                triangles[t].shading.tangents[k] = make_float4(tt[0], tt[1], tt[2], tt[3]);
                triangles[t].shading.uvs[k] = make_float2(uu[0], uu[1]);
                triangles[t].positions[k] = p[k];
            }
            uint32_t tag = t;
            std::memcpy(&triangles[t].shading.normals[0].w, &tag, 4);
            TriangleIntersection ti;
            ti.edge1 = make_float4(p[1] - p[0], 1.0f);
            ti.edge2 = make_float4(p[2] - p[0], 1.0f);
            ti.v0 = p[0];
            const uint32_t mat = materialIds[t];
            ti.shadingModel = static_cast<GlobalShadingModel>(std::min<uint32_t>(mats[mat].model, 5));
            triangles[t].intersection = ti;
            triangles[t].shading.material = mat;
            triangles[t].shading.geometricNormal = normalize(cross(make_float3(ti.edge1), make_float3(ti.edge2)));
        }
        // LightSampler::BuildSync (LightSampler.cpp:5-40), before the BVH reorders the triangles
        std::vector<LightTriangle> lights;
        std::vector<float> weights;
        std::vector<uint32_t> indices;
        for (uint32_t i = 0; i < n; i++)
        {
            if (triangles[i].intersection.shadingModel != GlobalShadingModel::Emissive) continue;
            float area = 0.5f * length(cross(make_float3(triangles[i].intersection.edge1), make_float3(triangles[i].intersection.edge2)));
            weights.push_back(area);
            indices.push_back(static_cast<uint32_t>(lights.size()));
            LightTriangle lt{triangles[i].intersection.edge1, triangles[i].intersection.edge2, triangles[i].intersection.v0, i,
                             triangles[i].shading.geometricNormal, area, triangles[i].shading.uvs[0],
                             triangles[i].shading.uvs[1] - triangles[i].shading.uvs[0],
                             triangles[i].shading.uvs[2] - triangles[i].shading.uvs[0],
                             scene->hostMaterials[triangles[i].shading.material].emission};
            lights.push_back(lt);
        }
        std::vector<Bin<uint32_t>> bins = weights.empty() ? std::vector<Bin<uint32_t>>{} : BuildAlias(weights, indices);
        scene->lightCount = static_cast<uint32_t>(lights.size());
        // HostBvh (compiled from the reference) + DFS flatten
        HostBvh bvh(std::move(triangles));
        std::vector<DeviceBvhNode> nodes;
        nodes.reserve(bvh.GetNodeCount());
        Flatten(bvh.GetRoot(), nodes);
        scene->nodeCount = static_cast<uint32_t>(nodes.size());
        scene->depth = bvh.GetDepth();
        const std::vector<Triangle>& ordered = bvh.GetTriangles();
        std::vector<TriangleIntersection> isect(n);
        std::vector<TriangleShading> shading(n);
        scene->order.resize(n);
        for (uint32_t i = 0; i < n; i++)
        {
            isect[i] = ordered[i].intersection;
            shading[i] = ordered[i].shading;
            uint32_t tag;
            std::memcpy(&tag, &shading[i].normals[0].w, 4);
            scene->order[i] = tag;
            shading[i].normals[0].w = 0.0f;
        }
        scene->nodes = dalloc<DeviceBvhNode>(nodes.size());
        scene->isect = dalloc<TriangleIntersection>(n);
        scene->shading = dalloc<TriangleShading>(n);
        scene->materials = dalloc<Material>(materialCount);
        scene->lights = dalloc<LightTriangle>(lights.size());
        scene->bins = dalloc<Bin<uint32_t>>(bins.size());
        bool ok = scene->nodes && scene->isect && scene->shading && scene->materials && scene->lights && scene->bins;
        ok = ok && cudaMemcpy(scene->nodes, nodes.data(), nodes.size() * sizeof(DeviceBvhNode), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(scene->isect, isect.data(), n * sizeof(TriangleIntersection), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(scene->shading, shading.data(), n * sizeof(TriangleShading), cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaMemcpy(scene->materials, scene->hostMaterials.data(), materialCount * sizeof(Material), cudaMemcpyHostToDevice) == cudaSuccess;
        if (!lights.empty())
        {
            ok = ok && cudaMemcpy(scene->lights, lights.data(), lights.size() * sizeof(LightTriangle), cudaMemcpyHostToDevice) == cudaSuccess;
            ok = ok && cudaMemcpy(scene->bins, bins.data(), bins.size() * sizeof(Bin<uint32_t>), cudaMemcpyHostToDevice) == cudaSuccess;
        }
        if (!ok)
        {
            delete scene;
            return nullptr;
        }
        *status = 0;
        return scene;
    }

    int ref_scene_info(void* sp, uint32_t* nodes, uint32_t* depth, uint32_t* lights)
    {
        auto* s = static_cast<Scene*>(sp);
        *nodes = s->nodeCount;
        *depth = s->depth;
        *lights = s->lightCount;
        return 0;
    }

    // The decoded texel values the reference kernels see for each material, in the 20-word
    // material record layout of the oracle and the product (model word left 0).
    int ref_scene_decoded_materials(void* sp, float* out)
    {
        auto* s = static_cast<Scene*>(sp);
        float* d = dalloc<float>(static_cast<size_t>(s->materialCount) * 20);
        if (!d) return 1;
        sample_material_kernel<<<(s->materialCount + 63) / 64, 64>>>(s->materials, s->materialCount, d);
        cudaError_t e = cudaMemcpy(out, d, static_cast<size_t>(s->materialCount) * 80, cudaMemcpyDeviceToHost);
        cudaFree(d);
        return e == cudaSuccess ? 0 : 2;
    }

    static bool ensure_queues(Scene* s, uint32_t capacity)
    {
        if (s->queues && s->queues->capacity >= capacity) return true;
        delete s->queues;
        s->queues = new Queues();
        return s->queues->allocate(capacity);
    }

    // Renderer::RenderFrame (Renderer.cpp:468-647) replayed through the reference's launchers.
    // accum: [w*h][4]; queueLog rows: rays, 6 material queues, shadow, regen.
    int ref_render(void* sp, const float* cam, uint32_t width, uint32_t height, uint32_t spp, uint32_t depthLimit, uint32_t nee,
                   uint32_t poolSize, float* accumOut, uint32_t* framebufferOut, uint32_t* queueLog, uint32_t logCapacity,
                   uint32_t* iterationsOut, float* frameMsOut)
    {
        auto* s = static_cast<Scene*>(sp);
        if (!ensure_queues(s, poolSize)) return 1;
        Queues& q = *s->queues;
        cudaStream_t stream;
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        DeviceCamera camera;
        camera.origin = make_float3(cam[0], cam[1], cam[2]);
        camera.lowerLeftCorner = make_float3(cam[3], cam[4], cam[5]);
        camera.horizontal = make_float3(cam[6], cam[7], cam[8]);
        camera.vertical = make_float3(cam[9], cam[10], cam[11]);
        PixelGrid grid;
        grid.width = width;
        grid.height = height;
        grid.samplesPerPixelAxis = static_cast<uint32_t>(std::sqrt(spp));
        grid.samplesPerPixel = grid.samplesPerPixelAxis * grid.samplesPerPixelAxis;
        const uint64_t totalSamples = static_cast<uint64_t>(grid.samplesPerPixel) * width * height;
        const uint32_t generateCount = static_cast<uint32_t>(std::min<uint64_t>(totalSamples, poolSize));
        float4* accum = dalloc<float4>(static_cast<size_t>(width) * height);
        if (!accum) return 2;
        IntersectionBvhView bvh(Runtime::DeviceBuffer1DView<DeviceBvhNode>(s->nodes, s->nodeCount),
                                Runtime::DeviceBuffer1DView<TriangleIntersection>(s->isect, s->triangleCount));
        Runtime::DeviceBuffer1DView<TriangleShading> shadingView(s->shading, s->triangleCount);
        Runtime::DeviceBuffer1DView<Material> materialView(s->materials, s->materialCount);
        LightSamplerView lightSampler(Runtime::DeviceBuffer1DView<LightTriangle>(s->lights, s->lightCount),
                                      AliasTableView<uint32_t>(Runtime::DeviceBuffer1DView<Bin<uint32_t>>(s->bins, s->lightCount)));
        Runtime::DeviceBuffer1DView<float4> accumView(accum, width * height);
        using Evaluator = void (*)(bool, cudaStream_t, PathPoolView, MaterialEvalQueueView, Runtime::DeviceBuffer1DView<TriangleShading>,
                                   Runtime::DeviceBuffer1DView<Material>, uint32_t, LightSamplerView, ShadowRayQueueView, RegenQueueView,
                                   Runtime::DeviceBuffer1DView<float4>, RayQueueView);
        const Evaluator evaluators[6] = {&Kernels::EvaluateNormalMaterial, &Kernels::EvaluateDiffuseMaterial, &Kernels::EvaluateMirrorMaterial,
                                         &Kernels::EvaluatePhongMaterial, &Kernels::EvaluateGgxMaterial, &Kernels::EvaluateEmissiveMaterial};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaMemsetAsync(q.counters, 0, 64, stream);
        cudaEventRecord(e0, stream);
        cudaMemsetAsync(accum, 0, sizeof(float4) * width * height, stream);
        uint32_t nextQueue = 0, currentQueue = 1;
        Kernels::InitializePaths(stream, generateCount, camera, grid, q.pool(), q.rays[nextQueue]);
        Kernels::PrepareIteration(stream, q.rays[currentQueue], q.rays[nextQueue], q.shadow, q.regen, q.materials, generateCount);
        currentQueue = nextQueue;
        nextQueue = currentQueue ^ 1;
        uint32_t rayCount = generateCount;
        uint64_t launched = generateCount;
        uint32_t iter = 0;
        uint32_t hostCounters[16];
        for (;;)
        {
            Kernels::IntersectRaysWithScene(stream, rayCount, q.rays[currentQueue], bvh, s->depth, q.materials, q.regen);
            cudaStreamSynchronize(stream);
            for (uint32_t i = 0; i < 6; i++)
            {
                if (s->materialCounts[i] == 0) continue;
                evaluators[i](nee != 0, stream, q.pool(), q.materials.At(i), shadingView, materialView, depthLimit, lightSampler, q.shadow,
                              q.regen, accumView, q.rays[nextQueue]);
            }
            if (nee) Kernels::IntersectShadowRaysWithScene(stream, q.shadow, bvh, s->depth, q.pool(), accumView);
            const uint32_t remaining = static_cast<uint32_t>(std::min<uint64_t>(totalSamples - launched, poolSize));
            Kernels::RegeneratePaths(stream, remaining, q.regen, launched, camera, grid, q.pool(), q.rays[nextQueue]);
            cudaMemcpyAsync(hostCounters, q.counters, 64, cudaMemcpyDeviceToHost, stream);
            cudaStreamSynchronize(stream);
            const uint32_t regenSize = hostCounters[9];
            if (queueLog && iter < logCapacity)
            {
                uint32_t* row = queueLog + static_cast<size_t>(iter) * 9;
                row[0] = rayCount;
                for (int m = 0; m < 6; m++) row[1 + m] = hostCounters[2 + m];
                row[7] = hostCounters[8];
                row[8] = regenSize;
            }
            iter++;
            const uint32_t regenerate = std::min(regenSize, remaining);
            const uint32_t nextRayCount = rayCount - regenSize + regenerate;
            if (nextRayCount == 0) break;
            Kernels::PrepareIteration(stream, q.rays[currentQueue], q.rays[nextQueue], q.shadow, q.regen, q.materials, nextRayCount);
            currentQueue = nextQueue;
            nextQueue = currentQueue ^ 1;
            rayCount = nextRayCount;
            launched += regenerate;
        }
        cudaEventRecord(e1, stream);
        cudaStreamSynchronize(stream);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (frameMsOut) *frameMsOut = ms;
        if (iterationsOut) *iterationsOut = iter;
        cudaError_t err = cudaGetLastError();
        std::vector<float4> host(static_cast<size_t>(width) * height);
        if (err == cudaSuccess) err = cudaMemcpy(host.data(), accum, host.size() * sizeof(float4), cudaMemcpyDeviceToHost);
        if (accumOut) std::memcpy(accumOut, host.data(), host.size() * sizeof(float4));
        if (framebufferOut)
        {
            // PostprocessKernel (Image.cu:34-54) on the host: x/spp, Reinhard, pow(x, 1/2.2), u8 truncation.
            const float invSpp = 1.0f / static_cast<float>(grid.samplesPerPixel);
            for (size_t p = 0; p < host.size(); p++)
            {
                const float v[3] = {host[p].x, host[p].y, host[p].z};
                uint32_t px = 255u << 24;
                for (int c = 0; c < 3; c++)
                {
                    float h = v[c] * invSpp;
                    float l = h / (h + 1.0f);
                    float g = std::pow(l, 1.0f / 2.2f);
                    float x = std::fmax(0.0f, std::fmin(g * 255.0f, 255.0f));
                    px |= static_cast<uint32_t>(static_cast<unsigned char>(x)) << (8 * c);
                }
                framebufferOut[p] = px;
            }
        }
        cudaFree(accum);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(stream);
        return err == cudaSuccess ? 0 : 3;
    }

    // IntersectRaysWithScene (Intersect.cu:63-123) over a host ray batch [n][8]: hits are read back
    // from the per-model MaterialEvalQueue arrays (path index = ray index), misses from the regen queue.
    int ref_trace_closest(void* sp, const float* rays, uint32_t n, uint32_t* triOut, float* uvtOut)
    {
        auto* s = static_cast<Scene*>(sp);
        const uint32_t chunk = 1u << 20;
        if (!ensure_queues(s, chunk)) return 1;
        Queues& q = *s->queues;
        IntersectionBvhView bvh(Runtime::DeviceBuffer1DView<DeviceBvhNode>(s->nodes, s->nodeCount),
                                Runtime::DeviceBuffer1DView<TriangleIntersection>(s->isect, s->triangleCount));
        // the queue allocations in constructor order: ray queue 0 = allocations[1..15]
        auto field = [&](int base, int k) { return q.allocations[base + k]; };
        const int ray0 = 1, mat0 = 1 + 2 * 15;
        for (uint32_t begin = 0; begin < n; begin += chunk)
        {
            const uint32_t m = std::min(chunk, n - begin);
            std::vector<uint32_t> idx(m), zero(m, 0);
            std::vector<float> one(m, 1.0f), comp(m);
            std::vector<uint8_t> delta(m, 1);
            std::iota(idx.begin(), idx.end(), 0u);
            cudaMemcpy(field(ray0, 0), idx.data(), m * 4, cudaMemcpyHostToDevice);      // paths
            cudaMemcpy(field(ray0, 1), zero.data(), m * 4, cudaMemcpyHostToDevice);     // depths
            for (int k = 2; k <= 5; k++) cudaMemcpy(field(ray0, k), one.data(), m * 4, cudaMemcpyHostToDevice);  // throughput, ior
            cudaMemcpy(field(ray0, 6), delta.data(), m, cudaMemcpyHostToDevice);
            for (int c = 0; c < 8; c++)
            {
                for (uint32_t i = 0; i < m; i++) comp[i] = rays[static_cast<size_t>(begin + i) * 8 + c];
                cudaMemcpy(field(ray0, 7 + c), comp.data(), m * 4, cudaMemcpyHostToDevice);
            }
            cudaMemset(q.counters, 0, 64);
            cudaMemcpy(q.counters, &m, 4, cudaMemcpyHostToDevice);  // ray queue size (PrepareIteration's SetSize)
            Kernels::IntersectRaysWithScene(nullptr, m, q.rays[0], bvh, s->depth, q.materials, q.regen);
            if (cudaDeviceSynchronize() != cudaSuccess) return 2;
            uint32_t counters[16];
            cudaMemcpy(counters, q.counters, 64, cudaMemcpyDeviceToHost);
            for (uint32_t i = 0; i < m; i++)
            {
                triOut[begin + i] = PathTracerDefaults::InvalidIndex;
                uvtOut[(static_cast<size_t>(begin) + i) * 3 + 0] = 0.0f;
                uvtOut[(static_cast<size_t>(begin) + i) * 3 + 1] = 0.0f;
                uvtOut[(static_cast<size_t>(begin) + i) * 3 + 2] = 0.0f;
            }
            for (int model = 0; model < 6; model++)
            {
                const uint32_t size = counters[2 + model];
                if (!size) continue;
                const int base = mat0 + model * 18;
                std::vector<uint32_t> paths(size), tris(size);
                std::vector<float> us(size), vs(size), tmax(size);
                cudaMemcpy(paths.data(), field(base, 0), size * 4, cudaMemcpyDeviceToHost);
                cudaMemcpy(tmax.data(), field(base, 14), size * 4, cudaMemcpyDeviceToHost);
                cudaMemcpy(tris.data(), field(base, 15), size * 4, cudaMemcpyDeviceToHost);
                cudaMemcpy(us.data(), field(base, 16), size * 4, cudaMemcpyDeviceToHost);
                cudaMemcpy(vs.data(), field(base, 17), size * 4, cudaMemcpyDeviceToHost);
                for (uint32_t k = 0; k < size; k++)
                {
                    const size_t r = static_cast<size_t>(begin) + paths[k];
                    triOut[r] = s->order[tris[k]];
                    uvtOut[r * 3 + 0] = us[k];
                    uvtOut[r * 3 + 1] = vs[k];
                    uvtOut[r * 3 + 2] = tmax[k];
                }
            }
        }
        return 0;
    }
}
