// Device construction of the BVH8 (see bvh_device.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "runtime.hpp"

namespace pt
{
    struct DeviceBvh
    {
        DeviceBuffer nodes;        // Node8 records, root first
        DeviceBuffer tris;         // kTriangleVec4 float4 per triangle, leaf order
        uint32_t nodeCount = 0;
        uint32_t depth = 0;        // levels of the wide tree
        uint32_t binaryNodes = 0;  // nodes of the clustered binary tree
        uint32_t rounds = 0;       // clustering rounds
    };

    // positions: device [n][3][3] world positions; models: device shading model per triangle (input
    // order). Builds on stream s and returns once the result is complete.
    Status BuildBvh8Device(const float* positions, const uint32_t* models, uint32_t n, cudaStream_t s, DeviceBvh& out);
}
