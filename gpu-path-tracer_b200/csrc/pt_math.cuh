// Vector algebra and the transcendental functions of the path tracer.
//
// The scalar operator order of the vector helpers is the one of cuda-samples' helper_math.h that
// the reference kernels use (External/cuda-samples/Common/helper_math.h: dot :1264, cross :1436,
// reflect :1427, lerp :1154, clamp :1168, normalize :1325), so expressions written like the
// reference's compile to the same operations.
//
// Two arithmetic modes, chosen per translation unit by PT_CUDA_MATH:
//   1  the product build (libgpt_b200.so). Compiled as the reference's kernels are (nvcc's
//      default multiply-add contraction), and the transcendentals are CUDA's own, called where
//      the reference calls them (MaterialEval.cu:224-228, 397, 442, 511, 589-591, 649;
//      Intersect.cu:131; Image.cu:31; rsqrtf in helper_math's normalize). Its results are the
//      reference build's on the same GPU.
//   0  the deterministic build (libgpt_b200_det.so, and the scene-upload kernels of every build,
//      which restate host code). Compiled with -fmad=false, so every float operator rounds once
//      in source order, and the transcendentals are defined below from the mathematics,
//      evaluated in IEEE double and rounded once to float: sin/cos by reduction modulo pi/2 and
//      Taylor series to r^15/r^16; pow(x, y) = exp(y ln x) with ln from the atanh series and exp
//      by reduction modulo ln 2 (the two-constant split of ln 2 published with fdlibm's e_exp.c,
//      Sun Microsystems 1993, used here only as the reduction's constants) and a Taylor series;
//      x^5 by repeated double multiplication; rsqrt(x) = 1/sqrt(x). These results are
//      reproducible bit for bit on any IEEE machine, which is what the CPU oracle relies on.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <math.h>

#define PT_HD __host__ __device__ __forceinline__

#ifndef PT_CUDA_MATH
#define PT_CUDA_MATH 0
#endif

namespace pt
{
    // ---------------------------------------------------------------- float3 algebra
    PT_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
    PT_HD float3 f3(float s) { return make_float3(s, s, s); }
    PT_HD float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
    PT_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
    PT_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
    PT_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
    PT_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
    PT_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
    PT_HD float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
    PT_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
    PT_HD float3 operator+(float3 a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
    PT_HD float3 operator-(float3 a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
    PT_HD float3 operator-(float s, float3 a) { return make_float3(s - a.x, s - a.y, s - a.z); }
    PT_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
    PT_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
    PT_HD float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
    PT_HD float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
    PT_HD float4 operator*(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }

    PT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    PT_HD float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
    PT_HD float3 cross(float3 a, float3 b)
    {
        return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    }
    PT_HD float rsqrt_ieee(float x) { return 1.0f / sqrtf(x); }
    PT_HD float length(float3 v) { return sqrtf(dot(v, v)); }
    PT_HD float3 reflect(float3 i, float3 n) { return i - 2.0f * n * dot(n, i); }
    PT_HD float clampf(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
    PT_HD float lerpf(float a, float b, float t) { return a + t * (b - a); }
    PT_HD float3 lerp3(float3 a, float3 b, float t) { return a + t * (b - a); }
    PT_HD float max3(float3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
    PT_HD float sqr(float v) { return v * v; }

    constexpr float kPi = 3.141592654f;
    constexpr float kInvPi = 1.0f / kPi;
    constexpr float kTwoPi = 2.0f * kPi;
    constexpr float kInvTwoPi = 1.0f / kTwoPi;
    constexpr float kOneMinusEpsilon = 0x1.fffffep-1f;

    // ---------------------------------------------------------------- deterministic transcendentals
    PT_HD double bits_to_double(uint64_t b)
    {
#ifdef __CUDA_ARCH__
        return __longlong_as_double(static_cast<long long>(b));
#else
        double d;
        __builtin_memcpy(&d, &b, sizeof(d));
        return d;
#endif
    }
    PT_HD uint64_t double_to_bits(double d)
    {
#ifdef __CUDA_ARCH__
        return static_cast<uint64_t>(__double_as_longlong(d));
#else
        uint64_t b;
        __builtin_memcpy(&b, &d, sizeof(b));
        return b;
#endif
    }
    PT_HD float as_float(uint32_t b)
    {
#ifdef __CUDA_ARCH__
        return __uint_as_float(b);
#else
        float f;
        __builtin_memcpy(&f, &b, sizeof(f));
        return f;
#endif
    }
    PT_HD uint32_t as_uint(float f)
    {
#ifdef __CUDA_ARCH__
        return __float_as_uint(f);
#else
        uint32_t b;
        __builtin_memcpy(&b, &f, sizeof(b));
        return b;
#endif
    }
    PT_HD double round_even(double x)
    {
#ifdef __CUDA_ARCH__
        return rint(x);
#else
        return __builtin_nearbyint(x);
#endif
    }
    PT_HD double pow2i(int n)
    {
        n = n > 1000 ? 1000 : (n < -1000 ? -1000 : n);
        return bits_to_double(static_cast<uint64_t>(static_cast<int64_t>(n) + 1023) << 52);
    }

    // sin and cos of a float angle.
    PT_HD void sincos_det(float xf, float* s, float* c)
    {
        const double x = static_cast<double>(xf);
        const double q = round_even(x * 0.63661977236758134308);
        const double r = x - q * 1.57079632679489661923;
        const double r2 = r * r;
        double ps = -1.0 / 1307674368000.0;
        ps = ps * r2 + 1.0 / 6227020800.0;
        ps = ps * r2 + -1.0 / 39916800.0;
        ps = ps * r2 + 1.0 / 362880.0;
        ps = ps * r2 + -1.0 / 5040.0;
        ps = ps * r2 + 1.0 / 120.0;
        ps = ps * r2 + -1.0 / 6.0;
        ps = ps * r2 + 1.0;
        ps = ps * r;
        double pc = 1.0 / 20922789888000.0;
        pc = pc * r2 + -1.0 / 87178291200.0;
        pc = pc * r2 + 1.0 / 479001600.0;
        pc = pc * r2 + -1.0 / 3628800.0;
        pc = pc * r2 + 1.0 / 40320.0;
        pc = pc * r2 + -1.0 / 720.0;
        pc = pc * r2 + 1.0 / 24.0;
        pc = pc * r2 + -0.5;
        pc = pc * r2 + 1.0;
        const int quadrant = static_cast<int>(static_cast<long long>(q) & 3);
        double sv, cv;
        if (quadrant == 0) { sv = ps; cv = pc; }
        else if (quadrant == 1) { sv = pc; cv = -ps; }
        else if (quadrant == 2) { sv = -ps; cv = -pc; }
        else { sv = -pc; cv = ps; }
        *s = static_cast<float>(sv);
        *c = static_cast<float>(cv);
    }

    PT_HD double log_det(double x)
    {
        uint64_t b = double_to_bits(x);
        int e = 0;
        int raw = static_cast<int>((b >> 52) & 0x7FF);
        if (raw == 0)
        {
            x = x * 18014398509481984.0;
            b = double_to_bits(x);
            raw = static_cast<int>((b >> 52) & 0x7FF);
            e = -54;
        }
        e += raw - 1023;
        double m = bits_to_double((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
        if (m > 1.41421356237309504880)
        {
            m = m * 0.5;
            e += 1;
        }
        const double s = (m - 1.0) / (m + 1.0);
        const double s2 = s * s;
        double p = 1.0 / 19.0;
        p = p * s2 + 1.0 / 17.0;
        p = p * s2 + 1.0 / 15.0;
        p = p * s2 + 1.0 / 13.0;
        p = p * s2 + 1.0 / 11.0;
        p = p * s2 + 1.0 / 9.0;
        p = p * s2 + 1.0 / 7.0;
        p = p * s2 + 1.0 / 5.0;
        p = p * s2 + 1.0 / 3.0;
        p = p * s2 + 1.0;
        const double lnm = 2.0 * s * p;
        const double ed = static_cast<double>(e);
        return ed * 6.93147180369123816490e-01 + (ed * 1.90821492927058770002e-10 + lnm);
    }

    PT_HD double exp_det(double t)
    {
        if (t > 709.0) return static_cast<double>(INFINITY);
        if (t < -745.0) return 0.0;
        const double n = round_even(t * 1.44269504088896338700);
        const double f = (t - n * 6.93147180369123816490e-01) - n * 1.90821492927058770002e-10;
        double p = 1.0 / 6227020800.0;
        p = p * f + 1.0 / 479001600.0;
        p = p * f + 1.0 / 39916800.0;
        p = p * f + 1.0 / 3628800.0;
        p = p * f + 1.0 / 362880.0;
        p = p * f + 1.0 / 40320.0;
        p = p * f + 1.0 / 5040.0;
        p = p * f + 1.0 / 720.0;
        p = p * f + 1.0 / 120.0;
        p = p * f + 1.0 / 24.0;
        p = p * f + 1.0 / 6.0;
        p = p * f + 0.5;
        p = p * f + 1.0;
        p = p * f + 1.0;
        int ni = static_cast<int>(n);
        if (ni < -1000)
        {
            p = p * pow2i(-1000);
            ni += 1000;
        }
        return p * pow2i(ni);
    }

    PT_HD float pow_det(float x, float y)
    {
        if (y == 0.0f) return 1.0f;
        if (x == 1.0f) return 1.0f;
        if (!(x >= 0.0f)) return NAN;
        if (x == 0.0f) return y > 0.0f ? 0.0f : INFINITY;
        if (x == INFINITY) return y > 0.0f ? INFINITY : 0.0f;
        return static_cast<float>(exp_det(static_cast<double>(y) * log_det(static_cast<double>(x))));
    }

    PT_HD float pow5_det(float x)
    {
        const double d = static_cast<double>(x);
        const double d2 = d * d;
        const double d4 = d2 * d2;
        return static_cast<float>(d4 * d);
    }

    // ---------------------------------------------------------------- the build's arithmetic
    // The two modes live in differently named inline namespaces, so translation units of both
    // modes link into one library without two definitions of one function.
#if PT_CUDA_MATH
    inline namespace cuda_math
    {
        // helper_math.h:78 and its device rsqrtf: CUDA's reciprocal square root on the GPU
        PT_HD float rsqrt_f(float x)
        {
#ifdef __CUDA_ARCH__
            return rsqrtf(x);
#else
            return 1.0f / sqrtf(x);
#endif
        }
        PT_HD void sincos_f(float x, float* s, float* c)
        {
            *c = cosf(x);
            *s = sinf(x);
        }
        PT_HD float pow_f(float x, float y) { return powf(x, y); }
        PT_HD float pow5_f(float x) { return powf(x, 5.0f); }

        // Moller-Trumbore with the multiply-add placement of the reference's own build
        // (Intersect.cu:25-60 through helper_math's cross and dot, nvcc 12.9 for sm_100a with its
        // default contraction). The placement was read off the bits of that build's (u, v, t) for
        // 120,000 captured closest hits, where one choice per operation reproduced all of them, and
        // is written here with explicit rounding intrinsics, so it no longer depends on how the
        // compiler schedules the code around it:
        //   every cross component a*b - c*d          fma(a, b, -(c*d))
        //   det = dot(e1, p), dot(d, q), dot(e2, q)  fma(z, z', fma(x, x', y*y'))
        //   dot(s, p)                                fma(z, z', fma(y, y', x*x'))
        PT_HD float fma_rn(float a, float b, float c)
        {
#ifdef __CUDA_ARCH__
            return __fmaf_rn(a, b, c);
#else
            return fmaf(a, b, c);
#endif
        }
        PT_HD float mul_rn(float a, float b)
        {
#ifdef __CUDA_ARCH__
            return __fmul_rn(a, b);
#else
            return a * b;
#endif
        }
        PT_HD float3 mt_cross(float3 a, float3 b)
        {
            return make_float3(fma_rn(a.y, b.z, -mul_rn(a.z, b.y)), fma_rn(a.z, b.x, -mul_rn(a.x, b.z)),
                               fma_rn(a.x, b.y, -mul_rn(a.y, b.x)));
        }
        PT_HD float mt_dot(float3 a, float3 b) { return fma_rn(a.z, b.z, fma_rn(a.x, b.x, mul_rn(a.y, b.y))); }
        PT_HD float mt_dot_sp(float3 a, float3 b) { return fma_rn(a.z, b.z, fma_rn(a.y, b.y, mul_rn(a.x, b.x))); }
#else
    inline namespace ieee_math
    {
        PT_HD float rsqrt_f(float x) { return rsqrt_ieee(x); }
        PT_HD void sincos_f(float x, float* s, float* c) { sincos_det(x, s, c); }
        PT_HD float pow_f(float x, float y) { return pow_det(x, y); }
        PT_HD float pow5_f(float x) { return pow5_det(x); }
        // Moller-Trumbore: every operator rounds once, in helper_math's order
        PT_HD float3 mt_cross(float3 a, float3 b) { return cross(a, b); }
        PT_HD float mt_dot(float3 a, float3 b) { return dot(a, b); }
        PT_HD float mt_dot_sp(float3 a, float3 b) { return dot(a, b); }
#endif
        PT_HD float3 normalize(float3 v)
        {
            float invLen = rsqrt_f(dot(v, v));
            return v * invLen;
        }
    }
}
