// special.cuh -- the special functions the alpha optimiser needs, with the
// arithmetic tomotopy uses, so that the optimiser's fixed point matches:
//   digammaT(x)      float 3-segment linear-interpolation table
//                    (src/Utils/math.h:134-150 with LUT3, src/Utils/LUT.hpp:11-70)
//   digammaf(x)      the float recursion + Chebyshev series that fills it
//                    (src/Utils/math.h:72-115)
//   digammaApprox(z) ln(z+4) - 1/(2(z+4)) - 1/(12(z+4)^2) - 1/z - 1/(z+1) - 1/(z+2) - 1/(z+3)
//                    evaluated in float (src/Utils/math.h:170-176)
// The table is built on the host once and copied to the device; lookups run
// on either side.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <vector>
#include <thread>
#include <algorithm>
#include "philox.cuh"   // TMT_HD

namespace tmt {

// Segment layout of the digamma table: [0, 1) step 1/1024, [1, 101) step
// 1/64, then 1000 points of step 1/4; closed forms below 0.001 and beyond.
struct DigammaTable {
    static constexpr int N = 1024, M = 100 * 64, L = 1000 * 4;
    static constexpr int S = 1024, T = 64, U = 4;
    const float* points;   // N + M + L entries

    TMT_HD static float small_form(float x)
    {
        if (x == 0) return -INFINITY;
        float x2 = x + 2;
        return logf(x2) - 0.5f / x2 - 1 / 12.f / (x2 * x2) - 1 / (x + 1) - 1 / x;
    }
    TMT_HD static float large_form(float x)
    {
        return logf(x) - 0.5f / x - 1 / 12.f / (x * x);
    }

    TMT_HD float operator()(float x) const
    {
        const float P = (float)(1. / S), Q = (float)(1. / T), R = (float)(1. / U);
        if (!(x == x)) return NAN;
        if (x == INFINITY) return INFINITY;
        if (x < 0) return NAN;
        if (x < (float)0.001) return small_form(x);
        if (x >= N * P + M * Q + (L - 1) * R) return large_form(x);
        size_t idx;
        float a;
        float nx = x;
        if (x < N * P) {
            idx = (size_t)(nx / P);
            a = (nx - idx * P) / P;
        } else {
            nx -= N * P;
            if (nx < M * Q) {
                idx = (size_t)(nx / Q);
                a = (nx - idx * Q) / Q;
                idx += N;
            } else {
                nx -= M * Q;
                idx = (size_t)(nx / R);
                a = (nx - idx * R) / R;
                idx += N + M;
            }
        }
        return points[idx] + a * (points[idx + 1] - points[idx]);
    }
};

// The float digamma that fills the table: reflection below 0, recurrence
// below 1, exact values at 1, 2, 3, duplication above 3 and a Chebyshev
// series on (1, 3) in between.
inline float digamma_series_f(float x)
{
    const float pi = 3.14159265f, gam = 0.577215664f, ln2 = 0.693147180f;
    if (x < 0.0f) return digamma_series_f(1.0f - x) + pi / tanf(pi * (1.0f - x));
    if (x < 1.0f) return digamma_series_f(1.0f + x) - 1.0f / x;
    if (x == 1.0f) return -gam;
    if (x == 2.0f) return (float)(1.0L - gam);
    if (x == 3.0f) return (float)(1.5L - gam);
    if (x > 3.0f) return 0.5f * (digamma_series_f(x / 2.0f) + digamma_series_f((x + 1.0f) / 2.0f)) + ln2;
    static const float coef[] = { .304591985f, .720379774f, -.124549592f, .277694573e-1f,
        -.677623714e-2f, .172387551e-2f, -.448176990e-3f, .117936600e-3f, -.312538942e-4f,
        .831739970e-5f, -.221914276e-5f, .593022667e-6f, -.158630511e-6f, .424592039e-7f,
        -.113691296e-7f, .304502217e-8f, -.815684550e-9f };
    float t_prev = 1.0f;
    float t = (float)(x - 2.0);
    float acc = coef[0] + coef[1] * t;
    float y = (float)(x - 2.0L);
    for (size_t n = 2; n < sizeof(coef) / sizeof(float); ++n) {
        const float t_next = (float)(2.0L * y * t - t_prev);
        acc += coef[n] * t_next;
        t_prev = t;
        t = t_next;
    }
    return acc;
}

// point i of the table (each point is independent of the others)
inline float digamma_point(size_t i)
{
    using T_ = DigammaTable;
    const float P = (float)(1. / T_::S), Q = (float)(1. / T_::T), R = (float)(1. / T_::U);
    if (i < (size_t)T_::N) return digamma_series_f(i ? i * P : (float)0.0001);
    i -= T_::N;
    if (i < (size_t)T_::M) return digamma_series_f(i * Q + T_::N * P);
    i -= T_::M;
    return digamma_series_f(i * R + T_::N * P + T_::M * Q);
}

inline std::vector<float> build_digamma_points()
{
    using T_ = DigammaTable;
    std::vector<float> p(T_::N + T_::M + T_::L);
    for (size_t i = 0; i < p.size(); ++i) p[i] = digamma_point(i);
    return p;
}

// The table's points, built once per process on up to 16 host threads: the
// series recurses on halved arguments above 3, so the 11,424 points take tens
// of milliseconds on one thread.  A pure function of the constants above.
inline const std::vector<float>& digamma_points()
{
    static const std::vector<float> pts = [] {
        using T_ = DigammaTable;
        std::vector<float> p(T_::N + T_::M + T_::L);
        const size_t n = p.size();
        const size_t T = std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
        auto part = [&p, T, n](size_t t) {
            for (size_t i = t; i < n; i += T) p[i] = digamma_point(i);
        };
        std::vector<std::thread> th;
        for (size_t t = 0; t < T; ++t) {
            try {
                th.emplace_back(part, t);
            } catch (...) {
                part(t);      // no thread to be had: this one computes the share
            }
        }
        for (auto& x : th) x.join();
        return p;
    }();
    return pts;
}

TMT_HD float digamma_approx_f(float z)
{
    float z4 = z + 4;
    return logf(z4) - 1.f / 2.f / z4 - 1.f / 12.f / (z4 * z4)
        - 1.f / z - 1.f / (z + 1) - 1.f / (z + 2) - 1.f / (z + 3);
}

} // namespace tmt
