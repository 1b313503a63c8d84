// Camera-path resampling for simulation sequences: Capture::ResampleMotion
// (Core/Source/Capture/Resampling.cpp:17-55). A recorded path of (state, time) samples becomes one
// state per frame at a fixed interval from the first sample's time. Between two recorded samples the
// position is interpolated linearly, a (1 - t) + b t (glm::mix, Utils/Math/Interpolation.hpp Lerp), and
// the rotation by spherical linear interpolation (Shoemake, "Animating Rotation with Quaternion Curves",
// SIGGRAPH 1985) along the shorter arc, then renormalised (Interpolation.hpp SlerpShortest). Host code.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../../include/gpt_b200.h"

namespace
{
    struct Quat
    {
        float w, x, y, z;
    };

    Quat load(const float* r) { return Quat{r[0], r[1], r[2], r[3]}; }

    float dot(const Quat& a, const Quat& b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }

    Quat scaled(const Quat& q, float s) { return Quat{q.w * s, q.x * s, q.y * s, q.z * s}; }

    Quat added(const Quat& a, const Quat& b) { return Quat{a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z}; }

    // unit quaternion of the same direction; a zero quaternion becomes the identity
    Quat normalised(const Quat& q)
    {
        const float len = std::sqrt(dot(q, q));
        if (!(len > 0.0f)) return Quat{1.0f, 0.0f, 0.0f, 0.0f};
        const float inv = 1.0f / len;
        return scaled(q, inv);
    }

    float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }

    // slerp of a towards b (b already on a's hemisphere): near-parallel rotations, where sin(theta)
    // vanishes, fall back to componentwise linear interpolation
    Quat slerp(const Quat& a, const Quat& b, float t)
    {
        const float cosTheta = dot(a, b);
        if (cosTheta > 1.0f - std::numeric_limits<float>::epsilon())
            return Quat{mix(a.w, b.w, t), mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t)};
        const float theta = std::acos(cosTheta);
        return scaled(added(scaled(a, std::sin((1.0f - t) * theta)), scaled(b, std::sin(t * theta))), 1.0f / std::sin(theta));
    }

    gpt_motion_state interpolate(const gpt_motion_state& p, const gpt_motion_state& c, float t)
    {
        gpt_motion_state out{};
        for (int k = 0; k < 3; k++) out.position[k] = mix(p.position[k], c.position[k], t);
        const Quat a = load(p.rotation);
        Quat b = load(c.rotation);
        if (dot(a, b) < 0.0f) b = scaled(b, -1.0f);  // shorter arc
        const Quat q = normalised(slerp(a, b, t));
        out.rotation[0] = q.w;
        out.rotation[1] = q.x;
        out.rotation[2] = q.y;
        out.rotation[3] = q.z;
        return out;
    }
}

extern "C" int gpt_resample_motion(const gpt_motion_sample* samples, uint32_t count, float interval, gpt_motion_state* states,
                                   uint32_t capacity, uint32_t* stateCount)
{
    if (!stateCount || (count > 0 && !samples)) return GPT_ERR_INVALID_ARGUMENT;
    if (!(interval > 0.0f)) return GPT_ERR_INVALID_ARGUMENT;
    std::vector<gpt_motion_state> out;
    if (count == 1)
        out.push_back(samples[0].state);
    else if (count > 1)
    {
        const float first = samples[0].time;
        out.push_back(samples[0].state);
        for (uint32_t i = 1; i < count; i++)
        {
            const gpt_motion_sample& prev = samples[i - 1];
            const gpt_motion_sample& cur = samples[i];
            if (!(cur.time > prev.time)) return GPT_ERR_INVALID_ARGUMENT;
            for (;;)
            {
                const float target = first + static_cast<float>(out.size()) * interval;
                if (target > cur.time) break;
                const float t = (target - prev.time) / (cur.time - prev.time);
                out.push_back(interpolate(prev.state, cur.state, t));
                if (out.size() > (1u << 24)) return GPT_ERR_CAPACITY;
            }
        }
    }
    *stateCount = static_cast<uint32_t>(out.size());
    if (out.size() > capacity) return GPT_ERR_CAPACITY;
    if (!out.empty())
    {
        if (!states) return GPT_ERR_INVALID_ARGUMENT;
        std::memcpy(states, out.data(), out.size() * sizeof(gpt_motion_state));
    }
    return GPT_OK;
}
