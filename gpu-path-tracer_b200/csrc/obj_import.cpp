// Headless OBJ/MTL scene ingest: a Wavefront OBJ file becomes the world-space triangle arrays and
// constant material table of gpt_scene_desc, the way the reference turns an OBJ into the input
// of its renderer:
//   LoadObj (Core/Source/Import/ObjLoader.cpp:67-234): triangulated faces grouped per shape and
//     per material id (ascending, faces without a material first), vertex normals and uvs
//     required, normals normalised, MTL keys Kd Ks Ns Pr Pm Ke Ni Tf d and the extension keys
//     `surface` (unlit normal diffuse lambert mirror phong microfacet ggx emissive) and `flip_textures`;
//   GenerateTangentSpace (Core/Source/Utils/Math/TangentSpace.cpp:66-89): per-vertex tangents with a
//     handedness sign by Mikkelsen's method, per submesh (tangent_space.cpp, gpt_generate_tangents);
//   Manager::ImportMaterial (Core/Source/Assets/Manager.cpp:311-412): constants become the texels of
//     1x1 textures (sRGB u8 colour and specular, linear u8 shininess (Ns-1)/999, float emission,
//     default normal texel); like the reference, the RMA texel is the default (255, 0, 255) when no
//     map_RMA texture is given;
//   BuildTriangles (Core/Source/Graphics/Cuda/PathTracing/Renderer.cpp:116-213): an optional affine
//     world transform, normals by the inverse transpose, tangents re-orthogonalised to the normal.
//   Texture maps (ObjLoader.cpp:197-225, Manager.cpp:311-385): map_Kd (albedo, sRGB), map_Ks (specular,
//     sRGB), map_Ns (shininess, linear, first channel), map_RMA (linear), map_Ke (emission, linear), norm
//     or else map_Bump/bump (normal map, linear), flipped vertically when the material says
//     flip_textures true; paths relative to the MTL file. PNG and binary PPM/PGM files are decoded
//     (image_io.cpp); the reference reads any format its image library knows, and other formats are
//     rejected here with an error naming the file.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gpt_b200.h"
#include "image_io.hpp"

struct gpt_obj_scene
{
    std::vector<float> positions, normals, tangents, uvs;
    std::vector<uint32_t> materialIds;
    std::vector<gpt_material> materials;
    std::vector<std::string> materialNames;
    std::vector<std::vector<uint8_t>> textureData;
    std::vector<gpt_texture_desc> textures;
    std::vector<int32_t> materialTextures;  // [materials][GPT_TEX_SLOTS], -1 = the constant
    std::string error;
};

namespace
{
    struct V3 { float x, y, z; };

    struct MtlEntry
    {
        std::string name;
        uint32_t model = GPT_MODEL_DIFFUSE;  // Unlit maps to Diffuse (Material.hpp:122-146)
        float kd[3] = {0, 0, 0}, ks[3] = {0, 0, 0}, ke[3] = {0, 0, 0};
        float ns = 1.0f, ni = 1.0f, tf = 0.0f, pr = 0.0f, pm = 0.0f;
        std::string maps[GPT_TEX_SLOTS];  // texture file per slot (color, specular, shininess, rma, emission, normal)
        std::string bump;                 // map_Bump / bump: the normal map when there is no norm
        bool flip = false;
        std::filesystem::path dir;        // the MTL file's folder
    };

    uint8_t lround_u8(float v)
    {
        long r = std::lround(v);
        return static_cast<uint8_t>(std::min(255L, std::max(0L, r)));
    }

    // LinearNormalizedFloatToSrgbU8 (Manager.cpp:65-79)
    uint8_t srgb_u8(float x)
    {
        if (!std::isfinite(x)) x = 0.0f;
        x = std::clamp(x, 0.0f, 1.0f);
        float s = x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
        return lround_u8(s * 255.0f);
    }

    // sRGB texel decode of an sRGB texture
    float srgb_decode(uint8_t u)
    {
        double c = u / 255.0;
        double l = c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
        return static_cast<float>(l);
    }

    uint8_t linear_u8(float x)  // NormalizedFloatToU8 (Manager.cpp:48-54)
    {
        if (!std::isfinite(x)) x = 0.0f;
        return lround_u8(std::clamp(x, 0.0f, 1.0f) * 255.0f);
    }

    gpt_material encode(const MtlEntry& m)
    {
        gpt_material g{};
        g.model = m.model;
        for (int k = 0; k < 3; k++)
        {
            g.color[k] = srgb_decode(srgb_u8(m.kd[k]));
            g.specular[k] = srgb_decode(srgb_u8(m.ks[k]));
            g.emission[k] = m.ke[k];
        }
        float ns = std::isfinite(m.ns) ? m.ns : 1.0f;
        ns = std::clamp(ns, 1.0f, 1000.0f);
        g.shininess = static_cast<float>(linear_u8((ns - 1.0f) / (1000.0f - 1.0f))) / 255.0f;
        g.rma[0] = 1.0f;  // default RMA texel (255, 0, 255): Manager.cpp:369-372 uses it for constants
        g.rma[1] = 0.0f;
        g.rma[2] = 1.0f;
        g.normal[0] = 128.0f / 255.0f;
        g.normal[1] = 128.0f / 255.0f;
        g.normal[2] = 1.0f;
        g.ior = m.ni;
        g.transmission = m.tf;
        return g;
    }

    bool parse_mtl(const std::filesystem::path& file, std::vector<MtlEntry>& out)
    {
        std::ifstream in(file);
        if (!in) return false;
        std::string line;
        MtlEntry* cur = nullptr;
        static const std::pair<const char*, uint32_t> models[] = {
            {"unlit", GPT_MODEL_DIFFUSE}, {"normal", GPT_MODEL_NORMAL}, {"diffuse", GPT_MODEL_DIFFUSE}, {"lambert", GPT_MODEL_DIFFUSE},
            {"mirror", GPT_MODEL_MIRROR}, {"phong", GPT_MODEL_PHONG}, {"microfacet", GPT_MODEL_GGX}, {"ggx", GPT_MODEL_GGX},
            {"emissive", GPT_MODEL_EMISSIVE}};
        while (std::getline(in, line))
        {
            std::istringstream ss(line);
            std::string key;
            if (!(ss >> key) || key[0] == '#') continue;
            if (key == "newmtl")
            {
                out.emplace_back();
                ss >> out.back().name;
                out.back().dir = file.parent_path();
                cur = &out.back();
                continue;
            }
            if (!cur) continue;
            auto read3 = [&](float* v) { ss >> v[0]; if (!(ss >> v[1] >> v[2])) v[1] = v[2] = v[0]; };
            if (key == "Kd") read3(cur->kd);
            else if (key == "Ks") read3(cur->ks);
            else if (key == "Ke") read3(cur->ke);
            else if (key == "Ns") ss >> cur->ns;
            else if (key == "Ni") ss >> cur->ni;
            else if (key == "Pr") ss >> cur->pr;
            else if (key == "Pm") ss >> cur->pm;
            else if (key == "Tf") { float t[3]; read3(t); cur->tf = t[0]; }
            else if (key == "surface")
            {
                std::string v;
                ss >> v;
                for (const auto& [name, model] : models)
                    if (v == name) cur->model = model;
            }
            else if (key == "flip_textures")
            {
                std::string v;
                ss >> v;
                cur->flip = v == "true";
            }
            else
            {
                // texture statements: options (-bm 1.0 ...) first, the file name last
                static const std::pair<const char*, int> maps[] = {{"map_Kd", GPT_TEX_COLOR}, {"map_Ks", GPT_TEX_SPECULAR},
                                                                   {"map_Ns", GPT_TEX_SHININESS}, {"map_RMA", GPT_TEX_RMA},
                                                                   {"map_Ke", GPT_TEX_EMISSION}, {"norm", GPT_TEX_NORMAL},
                                                                   {"map_Bump", -1}, {"bump", -1}};
                for (const auto& [name, slot] : maps)
                {
                    if (key != name) continue;
                    std::string tok, last;
                    while (ss >> tok) last = tok;
                    if (slot >= 0) cur->maps[slot] = last;
                    else cur->bump = last;
                }
            }
        }
        return true;
    }

    int resolve_index(long i, size_t count)
    {
        if (i > 0) return static_cast<int>(i - 1);
        if (i < 0) return static_cast<int>(static_cast<long>(count) + i);
        return -1;
    }

    // glm::normalize: v * (1 / sqrt(dot(v, v)))
    V3 normalize3(V3 v)
    {
        const float d = v.x * v.x + v.y * v.y + v.z * v.z;
        if (!(d > 0.0f)) return v;
        const float inv = 1.0f / std::sqrt(d);
        return {v.x * inv, v.y * inv, v.z * inv};
    }
}

extern "C"
{
    int gpt_obj_load(const char* path, const float* transform, gpt_obj_scene** out)
    {
        if (!path || !out) return GPT_ERR_INVALID_ARGUMENT;
        *out = nullptr;
        std::ifstream in(path);
        if (!in) return GPT_ERR_INVALID_ARGUMENT;
        const std::filesystem::path dir = std::filesystem::path(path).parent_path();
        std::vector<V3> pos, nrm;
        std::vector<std::array<float, 2>> tex;
        std::vector<MtlEntry> mtl;
        std::map<std::string, int> mtlIndex;
        struct Corner { int v, t, n; };
        struct Face { std::array<Corner, 3> c; };
        // shapes -> material id -> faces (tinyobj shape grouping, std::map order of material ids)
        std::vector<std::map<int, std::vector<Face>>> shapes(1);
        int currentMaterial = -1;
        std::string line;
        while (std::getline(in, line))
        {
            std::istringstream ss(line);
            std::string key;
            if (!(ss >> key) || key[0] == '#') continue;
            if (key == "v") { V3 p; ss >> p.x >> p.y >> p.z; pos.push_back(p); }
            else if (key == "vn") { V3 n; ss >> n.x >> n.y >> n.z; nrm.push_back(n); }
            else if (key == "vt") { std::array<float, 2> t{0, 0}; ss >> t[0] >> t[1]; tex.push_back(t); }
            else if (key == "mtllib")
            {
                std::string f;
                while (ss >> f)
                {
                    std::vector<MtlEntry> entries;
                    if (parse_mtl(dir / f, entries))
                        for (auto& e : entries)
                        {
                            mtlIndex[e.name] = static_cast<int>(mtl.size());
                            mtl.push_back(e);
                        }
                }
            }
            else if (key == "usemtl")
            {
                std::string n;
                ss >> n;
                auto it = mtlIndex.find(n);
                currentMaterial = it == mtlIndex.end() ? -1 : it->second;
            }
            else if (key == "o" || key == "g")
            {
                if (!shapes.back().empty()) shapes.emplace_back();
            }
            else if (key == "f")
            {
                std::vector<Corner> poly;
                std::string tok;
                while (ss >> tok)
                {
                    long vi = 0, ti = 0, ni = 0;
                    int field = 0;
                    std::string part;
                    std::stringstream ts(tok);
                    while (std::getline(ts, part, '/'))
                    {
                        long val = part.empty() ? 0 : std::stol(part);
                        if (field == 0) vi = val;
                        else if (field == 1) ti = val;
                        else ni = val;
                        field++;
                    }
                    poly.push_back({resolve_index(vi, pos.size()), resolve_index(ti, tex.size()), resolve_index(ni, nrm.size())});
                }
                for (size_t k = 2; k < poly.size(); k++)  // fan triangulation
                    shapes.back()[currentMaterial].push_back(Face{{poly[0], poly[k - 1], poly[k]}});
            }
        }
        auto scene = std::make_unique<gpt_obj_scene>();
        // material table: the file's materials, then a default white diffuse for faces without one
        for (const MtlEntry& e : mtl)
        {
            scene->materials.push_back(encode(e));
            scene->materialNames.push_back(e.name);
        }
        MtlEntry defaultMaterial;
        defaultMaterial.name = "default";
        defaultMaterial.kd[0] = defaultMaterial.kd[1] = defaultMaterial.kd[2] = 1.0f;
        const uint32_t defaultIndex = static_cast<uint32_t>(scene->materials.size());
        bool usesDefault = false;
        float M[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};  // column-major
        if (transform) std::memcpy(M, transform, sizeof(M));
        // normal matrix = inverse transpose of the linear part
        const float a = M[0], b = M[4], c = M[8], d = M[1], e = M[5], f = M[9], g = M[2], h = M[6], i = M[10];
        const float det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
        if (!(std::fabs(det) > 0.0f)) return GPT_ERR_INVALID_ARGUMENT;
        const float inv[9] = {(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det,
                              (f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det,
                              (d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det};  // row-major inverse
        auto xformP = [&](V3 p) { return V3{M[0] * p.x + M[4] * p.y + M[8] * p.z + M[12], M[1] * p.x + M[5] * p.y + M[9] * p.z + M[13],
                                            M[2] * p.x + M[6] * p.y + M[10] * p.z + M[14]}; };
        auto xformL = [&](V3 p) { return V3{M[0] * p.x + M[4] * p.y + M[8] * p.z, M[1] * p.x + M[5] * p.y + M[9] * p.z,
                                            M[2] * p.x + M[6] * p.y + M[10] * p.z}; };
        auto xformN = [&](V3 n) { return V3{inv[0] * n.x + inv[3] * n.y + inv[6] * n.z, inv[1] * n.x + inv[4] * n.y + inv[7] * n.z,
                                            inv[2] * n.x + inv[5] * n.y + inv[8] * n.z}; };
        for (auto& shape : shapes)
            for (auto& [matId, faces] : shape)
            {
                // dedupe corners of this submesh and accumulate tangents per vertex
                struct Key { int v, t, n; bool operator==(const Key& o) const { return v == o.v && t == o.t && n == o.n; } };
                struct KeyHash { size_t operator()(const Key& k) const { return (size_t(k.v) * 73856093u) ^ (size_t(k.t) * 19349663u) ^ (size_t(k.n) * 83492791u); } };
                std::unordered_map<Key, uint32_t, KeyHash> index;
                std::vector<Key> verts;
                std::vector<std::array<uint32_t, 3>> tris;
                for (const Face& fc : faces)
                {
                    std::array<uint32_t, 3> t{};
                    for (int k = 0; k < 3; k++)
                    {
                        const Corner& cr = fc.c[k];
                        if (cr.v < 0 || cr.v >= static_cast<int>(pos.size())) return GPT_ERR_INVALID_ARGUMENT;
                        if (cr.n < 0 || cr.n >= static_cast<int>(nrm.size())) return GPT_ERR_INVALID_ARGUMENT;  // normals are required
                        if (cr.t < 0 || cr.t >= static_cast<int>(tex.size())) return GPT_ERR_INVALID_ARGUMENT;  // uvs are required
                        Key key{cr.v, cr.t, cr.n};
                        auto it = index.try_emplace(key, static_cast<uint32_t>(verts.size()));
                        if (it.second) verts.push_back(key);
                        t[k] = it.first->second;
                    }
                    tris.push_back(t);
                }
                // MikkTSpace tangents of the submesh in object space (the loader's normalised normals)
                std::vector<float> vp(verts.size() * 3), vn(verts.size() * 3), vt(verts.size() * 2), vtan(verts.size() * 4);
                for (size_t k = 0; k < verts.size(); k++)
                {
                    const V3 p = pos[verts[k].v], n = normalize3(nrm[verts[k].n]);
                    vp[3 * k] = p.x; vp[3 * k + 1] = p.y; vp[3 * k + 2] = p.z;
                    vn[3 * k] = n.x; vn[3 * k + 1] = n.y; vn[3 * k + 2] = n.z;
                    vt[2 * k] = tex[verts[k].t][0]; vt[2 * k + 1] = tex[verts[k].t][1];
                }
                std::vector<uint32_t> vi(tris.size() * 3);
                for (size_t k = 0; k < tris.size(); k++)
                    for (int c = 0; c < 3; c++) vi[3 * k + c] = tris[k][c];
                const int trc = gpt_generate_tangents(vp.data(), vn.data(), vt.data(), static_cast<uint32_t>(verts.size()), vi.data(),
                                                      static_cast<uint32_t>(tris.size()), vtan.data());
                if (trc != GPT_OK) return trc;
                const uint32_t material = matId >= 0 ? static_cast<uint32_t>(matId) : defaultIndex;
                if (matId < 0) usesDefault = true;
                for (const auto& t : tris)
                {
                    for (int k = 0; k < 3; k++)
                    {
                        const Key& vk = verts[t[k]];
                        const V3 wp = xformP(pos[vk.v]);
                        const V3 n = normalize3(nrm[vk.n]);
                        const V3 wn = normalize3(xformN(n));
                        const float* mt = &vtan[4 * static_cast<size_t>(t[k])];
                        const V3 tg{mt[0], mt[1], mt[2]};
                        const float sign = mt[3];
                        // ComputeWorldTangent (Renderer.cpp:116-142)
                        V3 wt = xformL(tg);
                        float l2 = wt.x * wt.x + wt.y * wt.y + wt.z * wt.z;
                        if (l2 > 1e-16f)
                        {
                            const float inv = 1.0f / std::sqrt(l2);
                            wt = V3{wt.x * inv, wt.y * inv, wt.z * inv};
                            const float dd = wn.x * wt.x + wn.y * wt.y + wn.z * wt.z;
                            wt = V3{wt.x - wn.x * dd, wt.y - wn.y * dd, wt.z - wn.z * dd};
                        }
                        l2 = wt.x * wt.x + wt.y * wt.y + wt.z * wt.z;
                        if (l2 > 1e-16f)
                        {
                            const float inv = 1.0f / std::sqrt(l2);
                            wt = V3{wt.x * inv, wt.y * inv, wt.z * inv};
                        }
                        else
                        {
                            const V3 axis = std::fabs(wn.z) < 0.999f ? V3{0, 0, 1} : V3{1, 0, 0};
                            wt = normalize3(V3{axis.y * wn.z - axis.z * wn.y, axis.z * wn.x - axis.x * wn.z, axis.x * wn.y - axis.y * wn.x});
                        }
                        scene->positions.insert(scene->positions.end(), {wp.x, wp.y, wp.z});
                        scene->normals.insert(scene->normals.end(), {wn.x, wn.y, wn.z});
                        scene->tangents.insert(scene->tangents.end(), {wt.x, wt.y, wt.z, sign});
                        scene->uvs.insert(scene->uvs.end(), {tex[vk.t][0], tex[vk.t][1]});
                    }
                    scene->materialIds.push_back(material);
                }
            }
        if (usesDefault)
        {
            scene->materials.push_back(encode(defaultMaterial));
            scene->materialNames.push_back(defaultMaterial.name);
        }
        if (scene->materialIds.empty()) return GPT_ERR_INVALID_ARGUMENT;
        // texture maps: one texture per (file, colour space, flip), shared by the materials naming it
        bool anyMap = false;
        for (const MtlEntry& e : mtl)
            for (int k = 0; k < GPT_TEX_SLOTS; k++) anyMap = anyMap || !e.maps[k].empty() || !e.bump.empty();
        if (anyMap)
        {
            scene->materialTextures.assign(scene->materials.size() * GPT_TEX_SLOTS, -1);
            std::map<std::string, int32_t> loaded;
            for (size_t m = 0; m < mtl.size(); m++)
                for (int k = 0; k < GPT_TEX_SLOTS; k++)
                {
                    std::string file = mtl[m].maps[k];
                    if (k == GPT_TEX_NORMAL && file.empty()) file = mtl[m].bump;
                    if (file.empty()) continue;
                    const bool srgb = k == GPT_TEX_COLOR || k == GPT_TEX_SPECULAR;
                    const bool scalar = k == GPT_TEX_SHININESS;
                    std::filesystem::path full = mtl[m].dir / file;
                    if (!std::filesystem::exists(full)) full = file;
                    const std::string key = full.string() + (srgb ? "|s" : "|l") + (scalar ? "|1" : "|n") + (mtl[m].flip ? "|f" : "|u");
                    auto it = loaded.find(key);
                    if (it == loaded.end())
                    {
                        pt::Image8 img;
                        std::string err;
                        if (!pt::LoadImage8(full.string(), img, err))
                        {
                            scene->error = err;
                            std::fprintf(stderr, "gpt_obj_load: %s\n", err.c_str());
                            return GPT_ERR_INVALID_ARGUMENT;
                        }
                        uint32_t ch = img.channels;
                        std::vector<uint8_t> data;
                        if (scalar && ch != 1)
                        {
                            // one-channel slot: the first channel (ChannelLayout::R)
                            data.resize(static_cast<size_t>(img.width) * img.height);
                            for (size_t i = 0; i < data.size(); i++) data[i] = img.pixels[i * ch];
                            ch = 1;
                        }
                        else if (!scalar && ch == 1)
                        {
                            // grey map in a colour slot: replicated to RGB
                            data.resize(static_cast<size_t>(img.width) * img.height * 3);
                            for (size_t i = 0; i < img.pixels.size(); i++) data[i * 3] = data[i * 3 + 1] = data[i * 3 + 2] = img.pixels[i];
                            ch = 3;
                        }
                        else
                            data = std::move(img.pixels);
                        if (mtl[m].flip)
                        {
                            const size_t row = static_cast<size_t>(img.width) * ch;
                            for (uint32_t y = 0; y < img.height / 2; y++)
                                std::swap_ranges(data.begin() + static_cast<long>(y * row), data.begin() + static_cast<long>((y + 1) * row),
                                                 data.begin() + static_cast<long>((img.height - 1 - y) * row));
                        }
                        scene->textureData.push_back(std::move(data));
                        gpt_texture_desc t{};
                        t.width = img.width;
                        t.height = img.height;
                        t.channels = ch;
                        t.format = srgb ? GPT_TEXEL_U8_SRGB : GPT_TEXEL_U8_LINEAR;
                        scene->textures.push_back(t);
                        it = loaded.emplace(key, static_cast<int32_t>(scene->textures.size() - 1)).first;
                    }
                    scene->materialTextures[m * GPT_TEX_SLOTS + k] = it->second;
                }
            for (size_t i = 0; i < scene->textures.size(); i++) scene->textures[i].data = scene->textureData[i].data();
        }
        *out = scene.release();
        return GPT_OK;
    }

    int gpt_obj_scene_desc(const gpt_obj_scene* s, gpt_scene_desc* desc)
    {
        if (!s || !desc) return GPT_ERR_INVALID_ARGUMENT;
        desc->triangle_count = static_cast<uint32_t>(s->materialIds.size());
        desc->positions = s->positions.data();
        desc->normals = s->normals.data();
        desc->tangents = s->tangents.data();
        desc->uvs = s->uvs.data();
        desc->material_ids = s->materialIds.data();
        desc->material_count = static_cast<uint32_t>(s->materials.size());
        desc->materials = s->materials.data();
        desc->texture_count = static_cast<uint32_t>(s->textures.size());
        desc->textures = s->textures.empty() ? nullptr : s->textures.data();
        desc->material_textures = s->textures.empty() ? nullptr : s->materialTextures.data();
        return GPT_OK;
    }

    int gpt_obj_material_name(const gpt_obj_scene* s, uint32_t index, char* buffer, size_t length)
    {
        if (!s || !buffer || length == 0 || index >= s->materialNames.size()) return GPT_ERR_INVALID_ARGUMENT;
        std::snprintf(buffer, length, "%s", s->materialNames[index].c_str());
        return GPT_OK;
    }

    void gpt_obj_free(gpt_obj_scene* s) { delete s; }
}
