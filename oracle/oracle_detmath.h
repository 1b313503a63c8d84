// Oracle (test infrastructure): deterministic transcendental functions.
//
// The reference kernels call CUDA's sinf/cosf/powf/rsqrtf
// (Core/Source/Graphics/Cuda/PathTracing/Kernels/MaterialEval.cu:224-228,397-398,
// 589-591,649; Kernels/Image.cu:31; helper_math.h:1325-1328). Those functions are
// not reproducible on a CPU, so the oracle fixes a deterministic specification
// of each one, written from the mathematics (Taylor series about 0 with range
// reduction, evaluated in IEEE double and rounded once to float):
//
//   sin/cos(x)  : reduce x by the nearest multiple of pi/2, Taylor series to r^15/r^16
//   pow(x, y)   : exp(y * ln x), ln via the atanh series ln m = 2 atanh((m-1)/(m+1)),
//                 exp via reduction by ln 2 and a Taylor series to f^13
//   pow5(x)     : x*x*x*x*x in double
//   rsqrt(x)    : 1.0f / sqrtf(x)  (helper_math's own host definition, helper_math.h:78)
//
// Every operation used is an IEEE-754 basic operation (+ - * / sqrt), so a CPU
// build without FMA contraction and a GPU build without FMA contraction give
// bit-identical results. The GPU product implements the same specification
// independently; the parity tests compare the two.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle
{
    inline double dm_ldexp_int(double v, int n)
    {
        // multiply by 2^n built from its bit pattern (exact for the normal range)
        if (n > 1000) n = 1000;
        if (n < -1000) n = -1000;
        uint64_t bits = static_cast<uint64_t>(static_cast<int64_t>(n) + 1023) << 52;
        double scale;
        std::memcpy(&scale, &bits, sizeof(scale));
        return v * scale;
    }

    inline void dm_sincos(float xf, float* s, float* c)
    {
        const double halfPi = 1.57079632679489661923;
        const double invHalfPi = 0.63661977236758134308;
        double x = static_cast<double>(xf);
        double q = std::nearbyint(x * invHalfPi);
        double r = x - q * halfPi;
        double r2 = r * r;
        double sp = -1.0 / 1307674368000.0;
        sp = sp * r2 + 1.0 / 6227020800.0;
        sp = sp * r2 + -1.0 / 39916800.0;
        sp = sp * r2 + 1.0 / 362880.0;
        sp = sp * r2 + -1.0 / 5040.0;
        sp = sp * r2 + 1.0 / 120.0;
        sp = sp * r2 + -1.0 / 6.0;
        sp = sp * r2 + 1.0;
        sp = sp * r;
        double cp = 1.0 / 20922789888000.0;
        cp = cp * r2 + -1.0 / 87178291200.0;
        cp = cp * r2 + 1.0 / 479001600.0;
        cp = cp * r2 + -1.0 / 3628800.0;
        cp = cp * r2 + 1.0 / 40320.0;
        cp = cp * r2 + -1.0 / 720.0;
        cp = cp * r2 + 1.0 / 24.0;
        cp = cp * r2 + -0.5;
        cp = cp * r2 + 1.0;
        long long qi = static_cast<long long>(q);
        int quadrant = static_cast<int>(qi & 3);
        double sv, cv;
        switch (quadrant)
        {
            case 0: sv = sp; cv = cp; break;
            case 1: sv = cp; cv = -sp; break;
            case 2: sv = -sp; cv = -cp; break;
            default: sv = -cp; cv = sp; break;
        }
        *s = static_cast<float>(sv);
        *c = static_cast<float>(cv);
    }

    inline float dm_sin(float x) { float s, c; dm_sincos(x, &s, &c); return s; }
    inline float dm_cos(float x) { float s, c; dm_sincos(x, &s, &c); return c; }

    inline double dm_log(double x)
    {
        // x > 0 and finite
        int e = 0;
        uint64_t bits;
        std::memcpy(&bits, &x, sizeof(bits));
        int rawExp = static_cast<int>((bits >> 52) & 0x7FF);
        if (rawExp == 0)
        {
            x = x * 18014398509481984.0; // 2^54
            std::memcpy(&bits, &x, sizeof(bits));
            rawExp = static_cast<int>((bits >> 52) & 0x7FF);
            e = -54;
        }
        e += rawExp - 1023;
        bits = (bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
        double m;
        std::memcpy(&m, &bits, sizeof(m));
        if (m > 1.41421356237309504880)
        {
            m = m * 0.5;
            e += 1;
        }
        double s = (m - 1.0) / (m + 1.0);
        double s2 = s * s;
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
        double lnm = 2.0 * s * p;
        const double ln2Hi = 6.93147180369123816490e-01;
        const double ln2Lo = 1.90821492927058770002e-10;
        return static_cast<double>(e) * ln2Hi + (static_cast<double>(e) * ln2Lo + lnm);
    }

    inline double dm_exp(double t)
    {
        if (t > 709.0) return INFINITY;
        if (t < -745.0) return 0.0;
        const double invLn2 = 1.44269504088896338700;
        const double ln2Hi = 6.93147180369123816490e-01;
        const double ln2Lo = 1.90821492927058770002e-10;
        double n = std::nearbyint(t * invLn2);
        double f = (t - n * ln2Hi) - n * ln2Lo;
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
            p = dm_ldexp_int(p, -1000);
            ni += 1000;
        }
        return dm_ldexp_int(p, ni);
    }

    inline float dm_pow(float x, float y)
    {
        if (y == 0.0f) return 1.0f;
        if (x == 1.0f) return 1.0f;
        if (!(x >= 0.0f)) return NAN;
        if (x == 0.0f) return y > 0.0f ? 0.0f : INFINITY;
        if (std::isinf(x)) return y > 0.0f ? INFINITY : 0.0f;
        double t = static_cast<double>(y) * dm_log(static_cast<double>(x));
        return static_cast<float>(dm_exp(t));
    }

    inline float dm_pow5(float x)
    {
        double d = static_cast<double>(x);
        double d2 = d * d;
        double d4 = d2 * d2;
        return static_cast<float>(d4 * d);
    }

    inline float dm_rsqrt(float x)
    {
        return 1.0f / std::sqrt(x);
    }
}
