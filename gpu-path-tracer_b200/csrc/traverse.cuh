// BVH8 traversal primitives: quantised 8-child box test and the Moller-Trumbore
// triangle test, shared by the closest-hit and any-hit kernels.
#pragma once
#include "pt_internal.h"
#include "pt_math.cuh"

namespace pt
{
    // Per-ray values the node tests need (the direction itself is only needed by triangle tests,
    // which take it separately).
    struct RayPre
    {
        float3 o, invd;
        float tmin;
        uint32_t oct;   // child visiting order: bit k set when the ray's k-th direction component is negative
                        // (near to far); the any-hit kernel flips all three bits (far to near)
    };

    PT_HD float safe_inv(float dk)
    {
        float inv = 1.0f / dk;
        if (!(fabsf(inv) <= 1e30f)) inv = copysignf(1e30f, dk);
        return inv;
    }

    PT_HD RayPre make_ray(float3 o, float3 d, float tmin)
    {
        RayPre r;
        r.o = o;
        r.tmin = tmin;
        r.invd = make_float3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
        r.oct = (r.invd.x < 0.0f ? 1u : 0u) | (r.invd.y < 0.0f ? 2u : 0u) | (r.invd.z < 0.0f ? 4u : 0u);
        return r;
    }

    // bit i of the result = bit (i ^ oct) of m: slot order -> traversal order (and back).
    PT_HD uint32_t permute_mask(uint32_t m, uint32_t oct)
    {
        if (oct & 1u) m = ((m & 0x55u) << 1) | ((m & 0xAAu) >> 1);
        if (oct & 2u) m = ((m & 0x33u) << 2) | ((m & 0xCCu) >> 2);
        if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m & 0xF0u) >> 4);
        return m;
    }

    PT_HD float byte_to_float(uint32_t lo, uint32_t hi, int s)
    {
        const uint32_t w = s < 4 ? lo : hi;
        return static_cast<float>((w >> (8 * (s & 3))) & 0xFFu);
    }

    PT_HD float fma_hd(float a, float b, float c)
    {
#ifdef __CUDA_ARCH__
        return __fmaf_rn(a, b, c);
#else
        return fmaf(a, b, c);
#endif
    }

    // Slab test of the 8 quantised children against [tmin, tmax]. The computed entry
    // distance is lowered and the exit distance raised by 2^-20 of the node's scale in ray
    // space, so the test is conservative for every child box (a box the exact arithmetic
    // would hit is never culled). Returns the hit mask in slot order. Empty slots hold inverted
    // boxes and are almost always culled; one that passes has a zero child reference (no work).
    PT_HD uint32_t intersect_children(uint4 w0, uint4 w1, uint4 w2, uint4 w3, const RayPre& r, float tmin, float tmax)
    {
        const float px = as_float(w0.x), py = as_float(w0.y), pz = as_float(w0.z);
        const float sx = as_float((w0.w & 0xFFu) << 23);
        const float sy = as_float(((w0.w >> 8) & 0xFFu) << 23);
        const float sz = as_float(((w0.w >> 16) & 0xFFu) << 23);
        const float ax = sx * r.invd.x, ay = sy * r.invd.y, az = sz * r.invd.z;
        const float dx = px - r.o.x, dy = py - r.o.y, dz = pz - r.o.z;
        const float bx = dx * r.invd.x, by = dy * r.invd.y, bz = dz * r.invd.z;
        const float kEps = 9.5367431640625e-07f;  // 2^-20
        const float ex = (fabsf(dx) + 256.0f * sx) * fabsf(r.invd.x) * kEps;
        const float ey = (fabsf(dy) + 256.0f * sy) * fabsf(r.invd.y) * kEps;
        const float ez = (fabsf(dz) + 256.0f * sz) * fabsf(r.invd.z) * kEps;
        const float bnx = bx - ex, bfx = bx + ex;
        const float bny = by - ey, bfy = by + ey;
        const float bnz = bz - ez, bfz = bz + ez;
        // qlo.x = w1.xy, qlo.y = w1.zw, qlo.z = w2.xy, qhi.x = w2.zw, qhi.y = w3.xy, qhi.z = w3.zw
        const bool nx = r.invd.x < 0.0f, ny = r.invd.y < 0.0f, nz = r.invd.z < 0.0f;
        const uint32_t nxl = nx ? w2.z : w1.x, nxh = nx ? w2.w : w1.y;
        const uint32_t fxl = nx ? w1.x : w2.z, fxh = nx ? w1.y : w2.w;
        const uint32_t nyl = ny ? w3.x : w1.z, nyh = ny ? w3.y : w1.w;
        const uint32_t fyl = ny ? w1.z : w3.x, fyh = ny ? w1.w : w3.y;
        const uint32_t nzl = nz ? w3.z : w2.x, nzh = nz ? w3.w : w2.y;
        const uint32_t fzl = nz ? w2.x : w3.z, fzh = nz ? w2.y : w3.w;
        uint32_t hit = 0;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
        for (int s = 0; s < 8; s++)
        {
            const float tnx = fma_hd(byte_to_float(nxl, nxh, s), ax, bnx);
            const float tny = fma_hd(byte_to_float(nyl, nyh, s), ay, bny);
            const float tnz = fma_hd(byte_to_float(nzl, nzh, s), az, bnz);
            const float tfx = fma_hd(byte_to_float(fxl, fxh, s), ax, bfx);
            const float tfy = fma_hd(byte_to_float(fyl, fyh, s), ay, bfy);
            const float tfz = fma_hd(byte_to_float(fzl, fzh, s), az, bfz);
            const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
            const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
            hit |= (tn <= tf ? 1u : 0u) << s;
        }
        return hit;
    }

    // Moller-Trumbore with the reference's determinant cull and inclusive edges
    // (Intersect.cu:25-61), one IEEE rounding per operator. Returns false on a miss;
    // on a barycentric hit returns true with t, u, v (the caller applies the t range).
    PT_HD bool intersect_triangle(float4 a, float4 b, float4 c, float3 o, float3 d, float& t, float& u, float& v)
    {
        const float3 v0 = make_float3(a.x, a.y, a.z);
        const float3 e1 = make_float3(b.x, b.y, b.z);
        const float3 e2 = make_float3(c.x, c.y, c.z);
        const float3 p = mt_cross(d, e2);
        const float det = mt_dot(e1, p);
        if (fabsf(det) < 1e-7f) return false;
        const float3 s = o - v0;
        const float sp = mt_dot_sp(s, p);
        // u = sp * (1/det) is negative when sp and det have opposite signs and the product does not
        // round to zero; with |sp| > 1e-20 and |det| < 1e20 its magnitude exceeds 1e-40, so the
        // reference's u < 0 rejection is decided here without the division (same outcome, bit for bit).
        if (fabsf(sp) > 1e-20f && fabsf(det) < 1e20f && (sp < 0.0f) != (det < 0.0f)) return false;
        const float invDet = 1.0f / det;
        u = sp * invDet;
        if (u < 0.0f || u > 1.0f) return false;
        const float3 q = mt_cross(s, e1);
        v = mt_dot(d, q) * invDet;
        if (v < 0.0f || u + v > 1.0f) return false;
        t = mt_dot(e2, q) * invDet;
        return true;
    }

    struct HitRecord
    {
        float t;
        uint32_t tri;    // input-order triangle index, kInvalid when none
        float u, v;
        uint32_t model;
    };

    // Closest-hit acceptance with the deterministic tie rule: the smaller input index wins
    // at a bit-identical t.
    PT_HD bool better_hit(float t, uint32_t orig, float tmin, float bestT, uint32_t bestTri)
    {
        return t >= tmin && (t < bestT || (t == bestT && bestTri != kInvalid && orig < bestTri));
    }
}
