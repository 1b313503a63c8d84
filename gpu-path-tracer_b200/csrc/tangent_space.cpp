// Per-vertex tangent frames of an indexed triangle mesh by Mikkelsen's method (M. S. Mikkelsen,
// "Simulation of Wrinkled Surfaces Revisited", MSc thesis, University of Copenhagen, 2008), the
// tangent space the reference generates for every imported mesh (GenerateTangentSpace,
// Core/Source/Utils/Math/TangentSpace.cpp:66-89, with the default 180-degree angular threshold).
//
//  1. Corners with identical position, normal and uv are welded into one vertex identity.
//  2. Triangles with two equal positions are degenerate and set aside.
//  3. Each remaining triangle gets its first-order uv derivatives: the directions of increasing u and
//     v in the triangle's plane (thesis eq. 18-19), signed by the uv orientation, and their
//     magnitudes; a triangle with no uv area or zero derivatives may join any group.
//  4. Triangles are linked across shared edges (opposite directions, paired in triangle order).
//  5. Around every welded vertex, the triangles reachable through shared edges with the same uv
//     orientation form a group; a group's tangent is the corner-angle weighted mean of its triangles'
//     derivative directions projected into the vertex normal's plane.
//  6. A degenerate triangle's corner takes the frame of the first good corner with its identity.
// The sign is +1 for orientation-preserving groups, -1 otherwise; a vertex takes the frame of the
// last triangle corner that names it, as the reference's callback stores it per vertex. Host code.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>

#include "../../include/gpt_b200.h"

namespace
{
    struct V3
    {
        float x, y, z;
    };
    V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
    V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
    V3 scale(float s, V3 v) { return V3{s * v.x, s * v.y, s * v.z}; }
    float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    float length(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
    bool nonzero(float f) { return std::fabs(f) > FLT_MIN; }
    bool nonzero(V3 v) { return nonzero(v.x) || nonzero(v.y) || nonzero(v.z); }
    V3 unit(V3 v) { return scale(1.0f / length(v), v); }
    bool same(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
    // component of v in the plane normal to n, made unit length when it is not zero
    V3 in_plane(V3 v, V3 n)
    {
        V3 r = sub(v, scale(dot(n, v), n));
        return nonzero(r) ? unit(r) : r;
    }

    struct Frame
    {
        V3 s{1.0f, 0.0f, 0.0f};
        bool orientPreserving = false;
        bool set = false;
    };

    struct Tri
    {
        uint32_t corner[3];   // welded identities
        V3 os{0, 0, 0}, ot{0, 0, 0};
        float magS = 0.0f, magT = 0.0f;
        bool orientPreserving = false, anyGroup = true;
        int neighbour[3] = {-1, -1, -1};  // across edge k: corner k -> corner k+1
        int group[3] = {-1, -1, -1};
        uint32_t source = 0;  // triangle index in the input
    };

    struct Group
    {
        uint32_t vertex;
        bool orientPreserving;
        std::vector<int> tris;
    };
}

extern "C" int gpt_generate_tangents(const float* positions, const float* normals, const float* uvs, uint32_t vertexCount,
                                     const uint32_t* indices, uint32_t triangleCount, float* tangents)
{
    if (!positions || !normals || !uvs || !indices || !tangents) return GPT_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < 3ull * triangleCount; i++)
        if (indices[i] >= vertexCount) return GPT_ERR_INVALID_ARGUMENT;
    auto P = [&](uint32_t v) { return V3{positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]}; };
    auto N = [&](uint32_t v) { return V3{normals[3 * v], normals[3 * v + 1], normals[3 * v + 2]}; };
    auto T = [&](uint32_t v) { return std::array<float, 2>{uvs[2 * v], uvs[2 * v + 1]}; };

    // 1. welded identity of every corner: the first corner (in corner order) with equal attributes
    const size_t corners = static_cast<size_t>(triangleCount) * 3;
    std::vector<uint32_t> weld(corners);
    {
        auto bits = [](float f)
        {
            if (f == 0.0f) f = 0.0f;  // +0 and -0 compare equal
            uint32_t b;
            std::memcpy(&b, &f, 4);
            return b;
        };
        std::map<std::array<uint32_t, 8>, uint32_t> first;
        for (size_t c = 0; c < corners; c++)
        {
            const uint32_t v = indices[c];
            const V3 p = P(v), n = N(v);
            const auto t = T(v);
            const std::array<uint32_t, 8> key{bits(p.x), bits(p.y), bits(p.z), bits(n.x), bits(n.y), bits(n.z), bits(t[0]), bits(t[1])};
            weld[c] = first.emplace(key, static_cast<uint32_t>(c)).first->second;
        }
    }
    auto cornerVertex = [&](uint32_t c) { return indices[c]; };

    // 2. good triangles in input order; degenerate ones after
    std::vector<Tri> tris;
    std::vector<uint32_t> degenerate;
    for (uint32_t t = 0; t < triangleCount; t++)
    {
        const V3 p0 = P(indices[3 * t]), p1 = P(indices[3 * t + 1]), p2 = P(indices[3 * t + 2]);
        if (same(p0, p1) || same(p0, p2) || same(p1, p2))
        {
            degenerate.push_back(t);
            continue;
        }
        Tri tr;
        tr.source = t;
        for (int k = 0; k < 3; k++) tr.corner[k] = weld[3 * t + k];
        tris.push_back(tr);
    }

    // 3. first-order derivatives
    for (Tri& tr : tris)
    {
        const uint32_t a = cornerVertex(tr.corner[0]), b = cornerVertex(tr.corner[1]), c = cornerVertex(tr.corner[2]);
        const V3 v1 = P(a), v2 = P(b), v3 = P(c);
        const auto t1 = T(a), t2 = T(b), t3 = T(c);
        const float t21x = t2[0] - t1[0], t21y = t2[1] - t1[1];
        const float t31x = t3[0] - t1[0], t31y = t3[1] - t1[1];
        const V3 d1 = sub(v2, v1), d2 = sub(v3, v1);
        const float area2 = t21x * t31y - t21y * t31x;
        const V3 os = sub(scale(t31y, d1), scale(t21y, d2));
        const V3 ot = add(scale(-t31x, d1), scale(t21x, d2));
        tr.orientPreserving = area2 > 0.0f;
        if (nonzero(area2))
        {
            const float absArea = std::fabs(area2);
            const float lenS = length(os), lenT = length(ot);
            const float sgn = tr.orientPreserving ? 1.0f : -1.0f;
            if (nonzero(lenS)) tr.os = scale(sgn / lenS, os);
            if (nonzero(lenT)) tr.ot = scale(sgn / lenT, ot);
            tr.magS = lenS / absArea;
            tr.magT = lenT / absArea;
            if (nonzero(tr.magS) && nonzero(tr.magT)) tr.anyGroup = false;
        }
    }

    // 4. neighbours: edges keyed by their unordered identities; entries in triangle order pair with the
    //    first later entry running the other way whose edge is still free
    {
        std::unordered_map<uint64_t, std::vector<std::pair<int, int>>> edges;
        edges.reserve(tris.size() * 3);
        for (int f = 0; f < static_cast<int>(tris.size()); f++)
            for (int k = 0; k < 3; k++)
            {
                const uint64_t i0 = tris[f].corner[k], i1 = tris[f].corner[(k + 1) % 3];
                const uint64_t key = (std::min(i0, i1) << 32) | std::max(i0, i1);
                edges[key].emplace_back(f, k);
            }
        for (auto& [key, list] : edges)
        {
            (void)key;
            for (size_t a = 0; a < list.size(); a++)
            {
                const auto [fa, ka] = list[a];
                if (tris[fa].neighbour[ka] != -1) continue;
                const uint32_t from = tris[fa].corner[ka], to = tris[fa].corner[(ka + 1) % 3];
                for (size_t b = a + 1; b < list.size(); b++)
                {
                    const auto [fb, kb] = list[b];
                    if (tris[fb].neighbour[kb] != -1) continue;
                    if (tris[fb].corner[kb] == to && tris[fb].corner[(kb + 1) % 3] == from)
                    {
                        tris[fa].neighbour[ka] = fb;
                        tris[fb].neighbour[kb] = fa;
                        break;
                    }
                }
            }
        }
    }

    // 5. groups around each welded vertex (flood fill through the two edges at the vertex)
    std::vector<Group> groups;
    auto cornerOf = [&](const Tri& tr, uint32_t vertex)
    {
        for (int k = 0; k < 3; k++)
            if (tr.corner[k] == vertex) return k;
        return -1;
    };
    std::vector<int> stack;
    for (int f = 0; f < static_cast<int>(tris.size()); f++)
        for (int k = 0; k < 3; k++)
        {
            if (tris[f].anyGroup || tris[f].group[k] != -1) continue;
            const int g = static_cast<int>(groups.size());
            groups.push_back(Group{tris[f].corner[k], tris[f].orientPreserving, {f}});
            tris[f].group[k] = g;
            // depth first, neighbour across the edge leaving the vertex before the one entering it
            stack.clear();
            stack.push_back(tris[f].neighbour[(k + 2) % 3]);
            stack.push_back(tris[f].neighbour[k]);
            while (!stack.empty())
            {
                const int t = stack.back();
                stack.pop_back();
                if (t < 0) continue;
                Tri& tr = tris[t];
                const int i = cornerOf(tr, groups[g].vertex);
                if (i < 0 || tr.group[i] != -1) continue;
                if (tr.anyGroup && tr.group[0] == -1 && tr.group[1] == -1 && tr.group[2] == -1)
                    tr.orientPreserving = groups[g].orientPreserving;  // the first group to reach it decides
                if (tr.orientPreserving != groups[g].orientPreserving) continue;
                groups[g].tris.push_back(t);
                tr.group[i] = g;
                stack.push_back(tr.neighbour[(i + 2) % 3]);
                stack.push_back(tr.neighbour[i]);
            }
        }

    // the frame of a set of triangles at a vertex: corner-angle weighted mean direction
    auto evaluate = [&](const std::vector<int>& members, uint32_t vertex)
    {
        V3 s{0, 0, 0};
        for (int f : members)
        {
            const Tri& tr = tris[f];
            if (tr.anyGroup) continue;
            const int i = cornerOf(tr, vertex);
            const V3 n = N(cornerVertex(tr.corner[i]));
            const V3 os = in_plane(tr.os, n);
            const V3 p0 = P(cornerVertex(tr.corner[(i + 2) % 3])), p1 = P(cornerVertex(tr.corner[i])), p2 = P(cornerVertex(tr.corner[(i + 1) % 3]));
            const V3 e1 = in_plane(sub(p0, p1), n), e2 = in_plane(sub(p2, p1), n);
            float c = dot(e1, e2);
            c = c > 1.0f ? 1.0f : (c < -1.0f ? -1.0f : c);
            const float angle = static_cast<float>(std::acos(static_cast<double>(c)));
            s = add(s, scale(angle, os));
        }
        return nonzero(s) ? unit(s) : s;
    };

    // per group, per member triangle: the members whose projected directions are not opposite to its own
    // (a 180-degree threshold: all of them unless exactly opposite) form its subgroup; equal subgroups share a frame
    std::vector<Frame> frames(corners);
    const float threshold = static_cast<float>(std::cos(static_cast<double>((180.0f * static_cast<float>(M_PI)) / 180.0f)));
    for (const Group& G : groups)
    {
        std::vector<std::pair<std::vector<int>, V3>> subgroups;
        for (int f : G.tris)
        {
            const Tri& tr = tris[f];
            const int i = cornerOf(tr, G.vertex);
            const V3 n = N(cornerVertex(tr.corner[i]));
            const V3 os = in_plane(tr.os, n), ot = in_plane(tr.ot, n);
            std::vector<int> members;
            for (int t : G.tris)
            {
                const Tri& other = tris[t];
                const V3 os2 = in_plane(other.os, n), ot2 = in_plane(other.ot, n);
                const bool any = tr.anyGroup || other.anyGroup;
                if (any || f == t || (dot(os, os2) > threshold && dot(ot, ot2) > threshold)) members.push_back(t);
            }
            std::sort(members.begin(), members.end());
            auto it = std::find_if(subgroups.begin(), subgroups.end(), [&](const auto& sg) { return sg.first == members; });
            if (it == subgroups.end())
            {
                subgroups.emplace_back(members, evaluate(members, G.vertex));
                it = subgroups.end() - 1;
            }
            Frame& out = frames[3 * static_cast<size_t>(tr.source) + i];
            out.s = it->second;
            out.orientPreserving = G.orientPreserving;
            out.set = true;
        }
    }

    // 6. degenerate triangles: the frame of the first good corner with the same identity
    if (!degenerate.empty())
    {
        std::unordered_map<uint32_t, size_t> firstGood;
        for (const Tri& tr : tris)
            for (int k = 0; k < 3; k++) firstGood.emplace(tr.corner[k], 3 * static_cast<size_t>(tr.source) + k);
        for (uint32_t t : degenerate)
            for (int k = 0; k < 3; k++)
            {
                auto it = firstGood.find(weld[3 * t + k]);
                if (it != firstGood.end()) frames[3 * static_cast<size_t>(t) + k] = frames[it->second];
            }
    }

    // per vertex: the last corner that names it
    for (uint32_t v = 0; v < vertexCount; v++)
    {
        tangents[4 * v] = 1.0f;
        tangents[4 * v + 1] = tangents[4 * v + 2] = 0.0f;
        tangents[4 * v + 3] = -1.0f;
    }
    for (size_t c = 0; c < corners; c++)
    {
        const Frame& fr = frames[c];
        float* o = tangents + 4 * static_cast<size_t>(indices[c]);
        o[0] = fr.s.x;
        o[1] = fr.s.y;
        o[2] = fr.s.z;
        o[3] = fr.orientPreserving ? 1.0f : -1.0f;
    }
    return GPT_OK;
}
