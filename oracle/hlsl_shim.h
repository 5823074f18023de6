// hlsl_shim.h - TEST INFRASTRUCTURE ONLY (oracle).  Enough of HLSL's types and
// intrinsics, in C++, to compile the reference's compute shaders unchanged in
// meaning after the token-level rewrites of hlsl2cpp.py.  The intrinsics are
// the ones of ae_math.h, the same definitions the CUDA kernels and the oracle
// restatement use, so "the reference's code on the CPU" and "our kernels"
// differ only in the algorithm text, never in what dot() or sin() mean.
//
// Everything lives in namespace hlsl; the transpiled shader is included inside
// that namespace, so its globals (cbuffer fields, buffers, `seed`) and its
// `main` are hlsl:: names.
#pragma once
#include <stdint.h>
#include <string.h>

#include "../aviatorengine2_b200/csrc/ae_math.h"

namespace hlsl {

typedef uint32_t uint;

struct float2;
struct float3;
struct float4;

struct uint2;
struct float2 {
    float x, y;
    float2() : x(0), y(0) {}
    float2(float s) : x(s), y(s) {}
    float2(float a, float b) : x(a), y(b) {}
    explicit float2(const uint2 &u);
};
struct float3 {
    float x, y, z;
    float3() : x(0), y(0), z(0) {}
    float3(float s) : x(s), y(s), z(s) {}
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
    float3(float2 a, float c) : x(a.x), y(a.y), z(c) {}
    float2 xy() const { return float2(x, y); }
    float3 &operator+=(const float3 &o);
    float3 &operator-=(const float3 &o);
    float3 &operator*=(const float3 &o);
    float3 &operator/=(const float3 &o);
};
struct float4 {
    float x, y, z, w;
    float4() : x(0), y(0), z(0), w(0) {}
    float4(float s) : x(s), y(s), z(s), w(s) {}
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float4(float3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    float3 xyz() const { return float3(x, y, z); }
    float3 rgb() const { return float3(x, y, z); }
    float2 xy() const { return float2(x, y); }
    float2 zw() const { return float2(z, w); }
    float r_() const { return x; }
};
struct uint2 {
    uint x, y;
    uint2() : x(0), y(0) {}
    uint2(uint a, uint b) : x(a), y(b) {}
    explicit uint2(float2 f) : x(uint(f.x)), y(uint(f.y)) {}
    explicit uint2(const struct int2 &v);
};
inline uint2 min(uint2 a, uint2 b) { return uint2(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y); }
struct uint3 {
    uint x, y, z;
    uint3() : x(0), y(0), z(0) {}
    uint3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
    uint2 xy() const { return uint2(x, y); }
};
struct int2 {
    int x, y;
    int2() : x(0), y(0) {}
    int2(int a, int b) : x(a), y(b) {}
    explicit int2(uint2 u) : x(int(u.x)), y(int(u.y)) {}
    explicit int2(float2 f) : x(int(f.x)), y(int(f.y)) {}
};
struct int3 {
    int x, y, z;
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
    int3(int2 a, int c) : x(a.x), y(a.y), z(c) {}
    int3(uint2 a, int c) : x(int(a.x)), y(int(a.y)), z(c) {}
};
struct bool2 {
    bool x, y;
};
inline uint2::uint2(const int2 &v) : x(uint(v.x)), y(uint(v.y)) {}
inline float2::float2(const uint2 &u) : x(float(u.x)), y(float(u.y)) {}
inline bool all(bool2 b) { return b.x && b.y; }
inline bool2 operator>=(int2 a, int b) { return bool2{a.x >= b, a.y >= b}; }
inline bool2 operator<(int2 a, int2 b) { return bool2{a.x < b.x, a.y < b.y}; }
inline int2 operator+(int2 a, int2 b) { return int2(a.x + b.x, a.y + b.y); }
inline int2 operator-(int2 a, int b) { return int2(a.x - b, a.y - b); }
inline int2 clamp(int2 v, int2 lo, int2 hi) {
    return int2(v.x < lo.x ? lo.x : (v.x > hi.x ? hi.x : v.x), v.y < lo.y ? lo.y : (v.y > hi.y ? hi.y : v.y));
}
inline float2 to_float2(uint2 u) { return float2(float(u.x), float(u.y)); }
struct float4x4 {
    float m[4][4];
};
// mul(M, v) for a row-major matrix: each row dotted with v, left to right.
inline float4 mul(const float4x4 &M, const float4 &v) {
    float r[4];
    for (int i = 0; i < 4; i++)
        r[i] = AE_ADD(AE_ADD(AE_ADD(AE_MUL(M.m[i][0], v.x), AE_MUL(M.m[i][1], v.y)), AE_MUL(M.m[i][2], v.z)),
                      AE_MUL(M.m[i][3], v.w));
    return float4(r[0], r[1], r[2], r[3]);
}

// --- float3 arithmetic through ae:: (IEEE, no contraction) ---------------
inline ae::f3 A(const float3 &v) { return ae::mk(v.x, v.y, v.z); }
inline float3 B(const ae::f3 &v) { return float3(v.x, v.y, v.z); }
inline float3 operator+(const float3 &a, const float3 &b) { return B(A(a) + A(b)); }
inline float3 operator-(const float3 &a, const float3 &b) { return B(A(a) - A(b)); }
inline float3 operator*(const float3 &a, const float3 &b) { return B(A(a) * A(b)); }
inline float3 operator/(const float3 &a, const float3 &b) { return B(A(a) / A(b)); }
inline float3 operator*(const float3 &a, float s) { return B(A(a) * s); }
inline float3 operator*(float s, const float3 &a) { return B(s * A(a)); }
inline float3 operator/(const float3 &a, float s) { return B(A(a) / s); }
inline float3 operator/(float s, const float3 &a) { return B(s / A(a)); }
inline float3 operator+(const float3 &a, float s) { return B(A(a) + s); }
inline float3 operator-(const float3 &a, float s) { return B(A(a) - s); }
inline float3 operator+(float s, const float3 &a) { return B(ae::splat(s) + A(a)); }
inline float3 operator-(float s, const float3 &a) { return B(ae::splat(s) - A(a)); }
inline float3 operator-(const float3 &a) { return B(-A(a)); }
inline float3 &float3::operator+=(const float3 &o) { *this = *this + o; return *this; }
inline float3 &float3::operator-=(const float3 &o) { *this = *this - o; return *this; }
inline float3 &float3::operator*=(const float3 &o) { *this = *this * o; return *this; }
inline float3 &float3::operator/=(const float3 &o) { *this = *this / o; return *this; }

inline float2 operator+(const float2 &a, const float2 &b) { return float2(AE_ADD(a.x, b.x), AE_ADD(a.y, b.y)); }
inline float2 operator-(const float2 &a, const float2 &b) { return float2(AE_SUB(a.x, b.x), AE_SUB(a.y, b.y)); }
inline float2 operator*(const float2 &a, const float2 &b) { return float2(AE_MUL(a.x, b.x), AE_MUL(a.y, b.y)); }
inline float2 operator/(const float2 &a, const float2 &b) { return float2(AE_DIV(a.x, b.x), AE_DIV(a.y, b.y)); }
inline float2 operator*(const float2 &a, float s) { return float2(AE_MUL(a.x, s), AE_MUL(a.y, s)); }
inline float2 operator*(float s, const float2 &a) { return float2(AE_MUL(s, a.x), AE_MUL(s, a.y)); }
inline float2 operator/(const float2 &a, float s) { return float2(AE_DIV(a.x, s), AE_DIV(a.y, s)); }
inline float2 operator+(const float2 &a, float s) { return float2(AE_ADD(a.x, s), AE_ADD(a.y, s)); }
inline float2 operator-(const float2 &a, float s) { return float2(AE_SUB(a.x, s), AE_SUB(a.y, s)); }
inline float2 operator-(const float2 &a) { return float2(-a.x, -a.y); }

inline float4 operator*(const float4 &a, float s) {
    return float4(AE_MUL(a.x, s), AE_MUL(a.y, s), AE_MUL(a.z, s), AE_MUL(a.w, s));
}
inline float4 operator+(const float4 &a, const float4 &b) {
    return float4(AE_ADD(a.x, b.x), AE_ADD(a.y, b.y), AE_ADD(a.z, b.z), AE_ADD(a.w, b.w));
}

// --- intrinsics ------------------------------------------------------------
inline float dot(const float3 &a, const float3 &b) { return ae::dot(A(a), A(b)); }
inline float dot(const float2 &a, const float2 &b) { return AE_ADD(AE_MUL(a.x, b.x), AE_MUL(a.y, b.y)); }
inline float3 cross(const float3 &a, const float3 &b) { return B(ae::cross(A(a), A(b))); }
inline float length(const float3 &a) { return ae::length(A(a)); }
inline float length(const float2 &a) { return AE_SQRT(dot(a, a)); }
inline float distance(const float3 &a, const float3 &b) { return ae::distance(A(a), A(b)); }
inline float3 normalize(const float3 &a) { return B(ae::normalize(A(a))); }
inline float3 reflect(const float3 &i, const float3 &n) { return B(ae::reflect(A(i), A(n))); }
inline float3 refract(const float3 &i, const float3 &n, float eta) { return B(ae::refract(A(i), A(n), eta)); }
inline float min(float a, float b) { return AE_FMIN(a, b); }
inline float max(float a, float b) { return AE_FMAX(a, b); }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float3 min(const float3 &a, const float3 &b) { return B(ae::vmin(A(a), A(b))); }
inline float3 max(const float3 &a, const float3 &b) { return B(ae::vmax(A(a), A(b))); }
inline float abs(float x) { return AE_FABS(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float3 abs(const float3 &a) { return float3(AE_FABS(a.x), AE_FABS(a.y), AE_FABS(a.z)); }
inline float sqrt(float x) { return AE_SQRT(x); }
inline float sin(float x) { return ae::sinf_(x); }
inline float cos(float x) { return ae::cosf_(x); }
inline float tan(float x) { return ae::tanf_(x); }
inline float acos(float x) { return ae::acosf_(x); }
inline float atan2(float y, float x) { return ae::atan2f_(y, x); }
inline float exp(float x) { return ae::expf_(x); }
inline float log(float x) { return ae::logf_(x); }
inline float pow(float x, float y) { return ae::powf_(x, y); }
inline float3 pow(const float3 &x, float y) { return float3(ae::powf_(x.x, y), ae::powf_(x.y, y), ae::powf_(x.z, y)); }
inline float floor(float x) { return AE_FLOOR(x); }
inline float2 floor(const float2 &v) { return float2(AE_FLOOR(v.x), AE_FLOOR(v.y)); }
inline float2 ceil(const float2 &v) { return float2(__builtin_ceilf(v.x), __builtin_ceilf(v.y)); }
inline float3 frac(const float3 &v) { return float3(ae::fracf(v.x), ae::fracf(v.y), ae::fracf(v.z)); }
inline float frac(float x) { return ae::fracf(x); }
inline float sign(float x) { return ae::signf(x); }
inline float saturate(float x) { return ae::saturate(x); }
inline float3 saturate(const float3 &a) { return B(ae::saturate(A(a))); }
inline float2 saturate(const float2 &a) { return float2(ae::saturate(a.x), ae::saturate(a.y)); }
inline float clamp(float x, float lo, float hi) { return ae::clampf(x, lo, hi); }
inline int clamp(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
inline float radians(float d) { return ae::radians(d); }
inline float lerp(float a, float b, float t) { return ae::lerpf(a, b, t); }
inline float3 lerp(const float3 &a, const float3 &b, float t) { return B(ae::lerp(A(a), A(b), t)); }
inline float3 lerp(const float3 &a, const float3 &b, const float3 &t) { return a + t * (b - a); }

// --- resources -------------------------------------------------------------
template <typename T>
struct StructuredBuffer {
    const T *data = nullptr;
    uint count = 0;
    const T &operator[](uint i) const { return data[i]; }
};
// Storage images hold float4 at full precision.  The reference's targets are
// RGBA16F / RGBA8; the comparison is defined on the FP32 values written.
template <typename T>
struct RWTexture2D {
    T *data = nullptr;
    uint width = 0, height = 0;
    T &operator[](uint2 id) { return data[size_t(id.y) * width + id.x]; }
};
template <typename T>
struct Texture2D {
    const T *data = nullptr;
    uint width = 0, height = 0;
    T Load(const int3 &p) const { return data[size_t(p.y) * width + size_t(p.x)]; }
    T operator[](uint2 id) const { return data[size_t(id.y) * width + id.x]; }
};
struct SamplerState {};
// The material texture array as the harness binds it (RGBA8 sRGB words,
// layer-major).  SampleLevel uses the library's one definition of the
// renderer's linear REPEAT sampler at level 0 (ae_math.h texture_sample); the
// array layer is the coordinate rounded to nearest, clamped to the last.
struct Texture2DArray {
    const uint32_t *texels = nullptr;
    uint width = 0, height = 0, layers = 0;
    float4 SampleLevel(const SamplerState &, const float3 &c, float) const {
        static float lut[256];
        static bool ready = false;
        if (!ready) {
            for (uint32_t b = 0; b < 256; b++) lut[b] = ae::srgb_to_linear(b);
            ready = true;
        }
        const uint32_t layer = c.z <= 0.0f ? 0u : uint32_t(AE_FLOOR(c.z + 0.5f));
        const ae::f3 t = ae::texture_sample(texels, lut, width, height, layers, layer, c.x, c.y);
        return float4(t.x, t.y, t.z, 1.0f);
    }
};

}  // namespace hlsl
