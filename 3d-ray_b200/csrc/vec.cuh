// Float3 arithmetic shared by the host world builder and the device kernels.
//
// The reductions keep 3d-ray's System.Numerics.Vector3 evaluation order —
// Dot = (x*x + y*y) + z*z, Length = sqrt(Dot), Normalize = v / Length,
// division of a vector by a scalar is a per-component IEEE divide — and the
// library is built without FMA contraction (-fmad=false on the device,
// -ffp-contract=off on the host), so hit tests, lobe probabilities and every
// other +,-,*,/,sqrt result are bit-identical to the C# arithmetic.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define RT_HD __host__ __device__ __forceinline__
#define RT_D __device__ __forceinline__
#else
#define RT_HD inline
#define RT_D inline
#endif

namespace rt {

struct V3 {
    float x, y, z;
};

RT_HD V3 v3(float a) { return V3{a, a, a}; }
RT_HD V3 v3(float a, float b, float c) { return V3{a, b, c}; }
RT_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RT_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RT_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
RT_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
RT_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
RT_HD V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
RT_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
RT_HD V3 operator/(V3 a, V3 b) { return V3{a.x / b.x, a.y / b.y, a.z / b.z}; }
RT_HD bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
RT_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RT_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
RT_HD float length_sq(V3 a) { return dot(a, a); }
RT_HD float length(V3 a) { return sqrtf(length_sq(a)); }
RT_HD V3 normalize(V3 a) { return a / length(a); }
RT_HD V3 vmin(V3 a, V3 b) { return V3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
RT_HD V3 vmax(V3 a, V3 b) { return V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
RT_HD V3 lerp(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
RT_HD float lerpf(float a, float b, float t) { return a + (b - a) * t; }
RT_HD float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
RT_HD float axis_of(V3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
RT_HD float max3(V3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
RT_HD float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
RT_HD bool near_zero(V3 v) {
    const float s = 1e-8f;
    return fabsf(v.x) < s && fabsf(v.y) < s && fabsf(v.z) < s;
}

constexpr float kPi = 3.14159265358979323846f;
constexpr float kEps = 1e-4f;               // MathUtils.Epsilon
constexpr float kInf = 3.40282347e+38f;     // MathUtils.Infinity (float.MaxValue)
constexpr float kInv4Pi = 0.0795774715f;    // MathUtils.Inv4Pi
constexpr float kDeltaAlpha = 2.5e-3f;      // DisneyBsdf.DeltaAlphaThreshold

RT_HD V3 offset_origin(V3 p, V3 n) { return p + n * kEps; }
RT_HD V3 reflect(V3 v, V3 n) { return v - 2.0f * dot(v, n) * n; }

}  // namespace rt
