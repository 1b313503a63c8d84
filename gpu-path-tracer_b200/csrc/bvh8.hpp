// Host construction of the BVH8 (see bvh8.cpp).
#pragma once
#include <cstdint>
#include <vector>

#include "pt_internal.h"

namespace pt
{
    struct Bvh8
    {
        std::vector<Node8> nodes;
        std::vector<float4> tris;      // kTriangleVec4 per triangle, leaf order: (v0, orig), (e1, model), (e2, 0), 0
        std::vector<uint32_t> order;   // leaf position -> input triangle index
        uint32_t depth = 0;            // levels of the wide tree
        std::vector<Node2> nodes2;     // the binary tree the BVH8 is collapsed from, FP32 boxes (same leaf order)
        uint32_t depth2 = 0;           // levels of the binary tree
    };

    // positions: [n][3][3] world positions; models: shading model per triangle. withBinary: also
    // flatten the binary tree into FP32 Node2 records (nodes2, depth2).
    Bvh8 BuildBvh8(const float* positions, const uint32_t* models, uint32_t n, int threads, bool withBinary = false);

    struct Bvh8Check
    {
        uint64_t containmentViolations;  // quantised child boxes not containing their subtree (exact arithmetic)
        uint64_t trianglesNotExactlyOnce;
        uint64_t leafTriangles;
    };

    // Structural validation of a built BVH8 on the host.
    Bvh8Check CheckBvh8(const Bvh8& bvh, const float* positions, uint32_t n);
}
