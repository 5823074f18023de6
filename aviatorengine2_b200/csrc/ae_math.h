// ae_math.h - one definition of every shader intrinsic the ray path uses,
// compiled identically for the host (g++ -ffp-contract=off) and the device
// (nvcc).  Each arithmetic step is a correctly rounded IEEE-754 binary32
// operation: the device side spells multiplies and adds with __fmul_rn /
// __fadd_rn so no file's --fmad setting can fuse them, and division and
// square root are the IEEE ones.  The transcendental functions are written
// here from their series (no libm, no CUDA math library), so host and device
// produce the same bits, which is what makes RNG-driven paths comparable bit
// for bit.
//
// HLSL semantics restated (the reference shaders call these by their HLSL
// names, e.g. shaders/ray_trace.comp.hybrid.hlsl):
//   normalize(v) = v * (1 / sqrt(dot(v, v)))
//   lerp(a,b,t)  = a + t * (b - a)
//   reflect(i,n) = i - 2 * dot(n, i) * n
//   refract(i,n,eta): k = 1 - eta*eta*(1 - dot(n,i)^2); k < 0 -> 0,
//                     else eta*i - (eta*dot(n,i) + sqrt(k)) * n
//   min/max      = fminf/fmaxf (a NaN operand yields the other operand)
//   pow(x, y)    = exact square-and-multiply for integer y in [-64, 64],
//                  exp(y * log(x)) otherwise
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define AE_HD __host__ __device__ __forceinline__
#else
#define AE_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define AE_MUL(a, b) __fmul_rn((a), (b))
#define AE_ADD(a, b) __fadd_rn((a), (b))
#define AE_SUB(a, b) __fsub_rn((a), (b))
#define AE_DIV(a, b) __fdiv_rn((a), (b))
#define AE_SQRT(a) __fsqrt_rn(a)
#define AE_FMIN(a, b) fminf((a), (b))
#define AE_FMAX(a, b) fmaxf((a), (b))
#define AE_FABS(a) fabsf(a)
#define AE_FLOOR(a) floorf(a)
#define AE_RINT(a) rintf(a)
#define AE_U2F(u) __uint2float_rn(u)
#define AE_LDEXP(x, e) ldexpf((x), (e))
#else
#define AE_MUL(a, b) ((a) * (b))
#define AE_ADD(a, b) ((a) + (b))
#define AE_SUB(a, b) ((a) - (b))
#define AE_DIV(a, b) ((a) / (b))
#define AE_SQRT(a) __builtin_sqrtf(a)
#define AE_FMIN(a, b) __builtin_fminf((a), (b))
#define AE_FMAX(a, b) __builtin_fmaxf((a), (b))
#define AE_FABS(a) __builtin_fabsf(a)
#define AE_FLOOR(a) __builtin_floorf(a)
#define AE_RINT(a) __builtin_rintf(a)
#define AE_U2F(u) ((float)(uint32_t)(u))
#define AE_LDEXP(x, e) __builtin_ldexpf((x), (e))
#endif

namespace ae {

// ---------------------------------------------------------------------------
// float3
// ---------------------------------------------------------------------------
struct f3 {
    float x, y, z;
};

AE_HD f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
AE_HD f3 splat(float s) { return mk(s, s, s); }
AE_HD f3 operator+(f3 a, f3 b) { return mk(AE_ADD(a.x, b.x), AE_ADD(a.y, b.y), AE_ADD(a.z, b.z)); }
AE_HD f3 operator-(f3 a, f3 b) { return mk(AE_SUB(a.x, b.x), AE_SUB(a.y, b.y), AE_SUB(a.z, b.z)); }
AE_HD f3 operator*(f3 a, f3 b) { return mk(AE_MUL(a.x, b.x), AE_MUL(a.y, b.y), AE_MUL(a.z, b.z)); }
AE_HD f3 operator/(f3 a, f3 b) { return mk(AE_DIV(a.x, b.x), AE_DIV(a.y, b.y), AE_DIV(a.z, b.z)); }
AE_HD f3 operator*(f3 a, float s) { return mk(AE_MUL(a.x, s), AE_MUL(a.y, s), AE_MUL(a.z, s)); }
AE_HD f3 operator*(float s, f3 a) { return mk(AE_MUL(s, a.x), AE_MUL(s, a.y), AE_MUL(s, a.z)); }
AE_HD f3 operator/(f3 a, float s) { return mk(AE_DIV(a.x, s), AE_DIV(a.y, s), AE_DIV(a.z, s)); }
AE_HD f3 operator/(float s, f3 a) { return mk(AE_DIV(s, a.x), AE_DIV(s, a.y), AE_DIV(s, a.z)); }
AE_HD f3 operator+(f3 a, float s) { return mk(AE_ADD(a.x, s), AE_ADD(a.y, s), AE_ADD(a.z, s)); }
AE_HD f3 operator-(f3 a, float s) { return mk(AE_SUB(a.x, s), AE_SUB(a.y, s), AE_SUB(a.z, s)); }
AE_HD f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }

// dot = (ax*bx + ay*by) + az*bz, left to right as HLSL's dot is spelled out.
AE_HD float dot(f3 a, f3 b) { return AE_ADD(AE_ADD(AE_MUL(a.x, b.x), AE_MUL(a.y, b.y)), AE_MUL(a.z, b.z)); }
AE_HD f3 cross(f3 a, f3 b) {
    return mk(AE_SUB(AE_MUL(a.y, b.z), AE_MUL(a.z, b.y)),
              AE_SUB(AE_MUL(a.z, b.x), AE_MUL(a.x, b.z)),
              AE_SUB(AE_MUL(a.x, b.y), AE_MUL(a.y, b.x)));
}
AE_HD float length(f3 a) { return AE_SQRT(dot(a, a)); }
AE_HD float distance(f3 a, f3 b) { return length(a - b); }
AE_HD f3 normalize(f3 a) {
    const float inv = AE_DIV(1.0f, AE_SQRT(dot(a, a)));
    return a * inv;
}
AE_HD float fmin_(float a, float b) { return AE_FMIN(a, b); }
AE_HD float fmax_(float a, float b) { return AE_FMAX(a, b); }
AE_HD f3 vmin(f3 a, f3 b) { return mk(AE_FMIN(a.x, b.x), AE_FMIN(a.y, b.y), AE_FMIN(a.z, b.z)); }
AE_HD f3 vmax(f3 a, f3 b) { return mk(AE_FMAX(a.x, b.x), AE_FMAX(a.y, b.y), AE_FMAX(a.z, b.z)); }
AE_HD float saturate(float x) { return AE_FMIN(AE_FMAX(x, 0.0f), 1.0f); }
AE_HD f3 saturate(f3 a) { return mk(saturate(a.x), saturate(a.y), saturate(a.z)); }
AE_HD float clampf(float x, float lo, float hi) { return AE_FMIN(AE_FMAX(x, lo), hi); }
AE_HD float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
AE_HD float lerpf(float a, float b, float t) { return AE_ADD(a, AE_MUL(t, AE_SUB(b, a))); }
AE_HD f3 lerp(f3 a, f3 b, float t) { return a + t * (b - a); }
AE_HD f3 reflect(f3 i, f3 n) { return i - AE_MUL(2.0f, dot(n, i)) * n; }
AE_HD f3 refract(f3 i, f3 n, float eta) {
    const float cosi = dot(n, i);
    const float k = AE_SUB(1.0f, AE_MUL(AE_MUL(eta, eta), AE_SUB(1.0f, AE_MUL(cosi, cosi))));
    if (k < 0.0f) return splat(0.0f);
    return eta * i - AE_ADD(AE_MUL(eta, cosi), AE_SQRT(k)) * n;
}
AE_HD float maxc(f3 a) { return AE_FMAX(a.x, AE_FMAX(a.y, a.z)); }

// ---------------------------------------------------------------------------
// Transcendentals, from their Taylor series with Cody-Waite reduction.
// ---------------------------------------------------------------------------

// pi/2 split so that k * c1 and k * c2 are exact for |k| < 4096.
#define AE_PIO2_1 1.57080078125f
#define AE_PIO2_2 (-4.453584551811218e-06f)
#define AE_PIO2_3 (-8.705516307827565e-10f)

// sin and cos of r in [-pi/4, pi/4] (Taylor to r^9 and r^10).
AE_HD float sin_poly(float r) {
    const float r2 = AE_MUL(r, r);
    float p = 2.7557319223985893e-06f;                      //  1/9!
    p = AE_ADD(AE_MUL(p, r2), -1.984126984126984e-04f);      // -1/7!
    p = AE_ADD(AE_MUL(p, r2), 8.333333333333333e-03f);       //  1/5!
    p = AE_ADD(AE_MUL(p, r2), -1.6666666666666666e-01f);     // -1/3!
    return AE_ADD(r, AE_MUL(AE_MUL(r, r2), p));
}
AE_HD float cos_poly(float r) {
    const float r2 = AE_MUL(r, r);
    float p = -2.755731922398589e-07f;                       // -1/10!
    p = AE_ADD(AE_MUL(p, r2), 2.48015873015873e-05f);        //  1/8!
    p = AE_ADD(AE_MUL(p, r2), -1.388888888888889e-03f);      // -1/6!
    p = AE_ADD(AE_MUL(p, r2), 4.1666666666666664e-02f);      //  1/4!
    return AE_ADD(AE_SUB(1.0f, AE_MUL(0.5f, r2)), AE_MUL(AE_MUL(r2, r2), p));
}
// Reduce x to r in [-pi/4, pi/4] and the quadrant k mod 4.  Valid for
// |x| < 4096 * pi/2; larger arguments are reduced in double precision.
AE_HD float reduce_pio2(float x, int &quadrant) {
    const float k = AE_RINT(AE_MUL(x, 0.6366197723675814f));
    float r;
    if (AE_FABS(k) < 4096.0f) {
        r = AE_SUB(x, AE_MUL(k, AE_PIO2_1));
        r = AE_SUB(r, AE_MUL(k, AE_PIO2_2));
        r = AE_SUB(r, AE_MUL(k, AE_PIO2_3));
    } else {
        const double kd = (double)k;
        r = (float)(((double)x - kd * 1.5707963267948966) - kd * 6.123233995736766e-17);
    }
    quadrant = ((int)k) & 3;
    return r;
}
AE_HD float sinf_(float x) {
    int q;
    const float r = reduce_pio2(x, q);
    switch (q) {
    case 0: return sin_poly(r);
    case 1: return cos_poly(r);
    case 2: return -sin_poly(r);
    default: return -cos_poly(r);
    }
}
AE_HD float cosf_(float x) {
    int q;
    const float r = reduce_pio2(x, q);
    switch (q) {
    case 0: return cos_poly(r);
    case 1: return -sin_poly(r);
    case 2: return -cos_poly(r);
    default: return sin_poly(r);
    }
}
AE_HD float tanf_(float x) { return AE_DIV(sinf_(x), cosf_(x)); }

// exp: x = k ln2 + r, |r| <= ln2/2, e^r by Taylor to r^8.
AE_HD float expf_(float x) {
    if (x != x) return x;
    if (x > 88.72283905206835f) return __builtin_huge_valf();
    if (x < -103.97207708f) return 0.0f;
    const float k = AE_RINT(AE_MUL(x, 1.4426950408889634f));
    float r = AE_SUB(x, AE_MUL(k, 0.693115234375f));
    r = AE_SUB(r, AE_MUL(k, 3.194618329871446e-05f));
    float p = 2.48015873015873e-05f;                         // 1/8!
    p = AE_ADD(AE_MUL(p, r), 1.984126984126984e-04f);        // 1/7!
    p = AE_ADD(AE_MUL(p, r), 1.388888888888889e-03f);        // 1/6!
    p = AE_ADD(AE_MUL(p, r), 8.333333333333333e-03f);        // 1/5!
    p = AE_ADD(AE_MUL(p, r), 4.1666666666666664e-02f);       // 1/4!
    p = AE_ADD(AE_MUL(p, r), 1.6666666666666666e-01f);       // 1/3!
    p = AE_ADD(AE_MUL(p, r), 0.5f);
    p = AE_ADD(AE_MUL(p, r), 1.0f);
    p = AE_ADD(AE_MUL(p, r), 1.0f);
    // Two-step scaling keeps 2^k representable near the subnormal range.
    const int ki = (int)k;
    if (ki < -125) return AE_LDEXP(AE_LDEXP(p, ki + 60), -60);
    return AE_LDEXP(p, ki);
}

// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
// s = (m-1)/(m+1), series to s^13.
AE_HD float logf_(float x) {
    if (x != x || x < 0.0f) return __builtin_nanf("");
    if (x == 0.0f) return -__builtin_huge_valf();
    if (x == __builtin_huge_valf()) return x;
    int e = 0;
    float m = x;
    // Normalise subnormals first.
    if (m < 1.17549435e-38f) { m = AE_MUL(m, 16777216.0f); e -= 24; }
    union { float f; uint32_t u; } b;
    b.f = m;
    e += (int)((b.u >> 23) & 0xffu) - 127;
    b.u = (b.u & 0x007fffffu) | 0x3f800000u;  // m in [1, 2)
    m = b.f;
    if (m > 1.4142135623730951f) { m = AE_MUL(m, 0.5f); e += 1; }
    const float s = AE_DIV(AE_SUB(m, 1.0f), AE_ADD(m, 1.0f));
    const float s2 = AE_MUL(s, s);
    float p = 7.6923076923076927e-02f;                       // 1/13
    p = AE_ADD(AE_MUL(p, s2), 9.0909090909090912e-02f);      // 1/11
    p = AE_ADD(AE_MUL(p, s2), 1.1111111111111110e-01f);      // 1/9
    p = AE_ADD(AE_MUL(p, s2), 1.4285714285714285e-01f);      // 1/7
    p = AE_ADD(AE_MUL(p, s2), 2.0000000000000001e-01f);      // 1/5
    p = AE_ADD(AE_MUL(p, s2), 3.3333333333333331e-01f);      // 1/3
    const float lnm = AE_MUL(2.0f, AE_ADD(s, AE_MUL(AE_MUL(s, s2), p)));
    const float ef = (float)e;
    return AE_ADD(AE_ADD(AE_MUL(ef, 3.194618329871446e-05f), lnm), AE_MUL(ef, 0.693115234375f));
}

AE_HD float powf_(float x, float y) {
    if (y == AE_FLOOR(y) && AE_FABS(y) <= 64.0f) {
        int n = (int)AE_FABS(y);
        float base = x, acc = 1.0f;
        while (n > 0) {
            if (n & 1) acc = AE_MUL(acc, base);
            n >>= 1;
            if (n) base = AE_MUL(base, base);
        }
        return y < 0.0f ? AE_DIV(1.0f, acc) : acc;
    }
    if (x == 0.0f) return y > 0.0f ? 0.0f : __builtin_huge_valf();
    return expf_(AE_MUL(y, logf_(x)));
}

// atan of |x| <= 1 by reduction about tan(pi/6) and Taylor to x^11.
AE_HD float atan_unit(float x) {
    float off = 0.0f;
    if (x > 0.2679491924311227f) {  // tan(pi/12)
        x = AE_DIV(AE_SUB(AE_MUL(x, 1.7320508075688772f), 1.0f), AE_ADD(x, 1.7320508075688772f));
        off = 0.5235987755982988f;  // pi/6
    }
    const float x2 = AE_MUL(x, x);
    float p = -9.0909090909090912e-02f;                      // -1/11
    p = AE_ADD(AE_MUL(p, x2), 1.1111111111111110e-01f);      //  1/9
    p = AE_ADD(AE_MUL(p, x2), -1.4285714285714285e-01f);     // -1/7
    p = AE_ADD(AE_MUL(p, x2), 2.0000000000000001e-01f);      //  1/5
    p = AE_ADD(AE_MUL(p, x2), -3.3333333333333331e-01f);     // -1/3
    return AE_ADD(off, AE_ADD(x, AE_MUL(AE_MUL(x, x2), p)));
}
AE_HD float atan2f_(float y, float x) {
    if (x != x || y != y) return __builtin_nanf("");
    const float ax = AE_FABS(x), ay = AE_FABS(y);
    if (ax == 0.0f && ay == 0.0f) {
        const bool xneg = (x < 0.0f) || (1.0f / x < 0.0f);
        const float base = xneg ? 3.14159265358979f : 0.0f;
        return (y < 0.0f || (1.0f / y < 0.0f)) ? -base : base;
    }
    float a;
    if (ay <= ax) a = atan_unit(AE_DIV(ay, ax));
    else a = AE_SUB(1.5707963267948966f, atan_unit(AE_DIV(ax, ay)));
    if (x < 0.0f) a = AE_SUB(3.14159265358979f, a);
    return y < 0.0f ? -a : a;
}
// acos(x) = 2 atan2(sqrt(1-x), sqrt(1+x))
AE_HD float acosf_(float x) {
    if (x > 1.0f || x < -1.0f) return __builtin_nanf("");
    return AE_MUL(2.0f, atan2f_(AE_SQRT(AE_SUB(1.0f, x)), AE_SQRT(AE_ADD(1.0f, x))));
}
AE_HD float radians(float deg) { return AE_MUL(deg, 0.017453292519943295f); }
AE_HD float fracf(float x) { return AE_SUB(x, AE_FLOOR(x)); }

// ---------------------------------------------------------------------------
// RNG: the reference's per-pixel PCG-style hash (hybrid:238-243).
// ---------------------------------------------------------------------------
AE_HD float rng_next(uint32_t &seed) {
    seed = seed * 747796405u + 2891336453u;
    const uint32_t x = ((seed >> ((seed >> 28u) + 4u)) ^ seed) * 277803737u;
    return AE_MUL(AE_U2F((x >> 22u) ^ x), 2.3283064365386963e-10f);  // / 2^32 (exact)
}

// ---------------------------------------------------------------------------
// Texture sampling: GlobalTextureArray.SampleLevel(GlobalSampler,
// float3(uv, layer), 0) (hybrid:919-925) on the reference's texture array and
// sampler.  The array is RGBA8 sRGB, `layers` images of w x h texels of one
// size (scene/texture.h:110-230, one level); the sampler filters linearly and
// repeats on u and v (renderer/renderer.cpp:226-233).  Texels are decoded from
// sRGB to linear before filtering, as the sRGB format requires, through a
// 256-entry table of srgb_to_linear; the bilinear weights and blends are
// binary32 operations (graphics hardware uses fixed-point sub-texel weights,
// which no specification pins down).  A layer beyond the last is clamped to
// it; non-finite coordinates sample at 0.
// ---------------------------------------------------------------------------
AE_HD float srgb_to_linear(uint32_t byte) {
    const float c = AE_DIV(AE_U2F(byte), 255.0f);
    return c <= 0.04045f ? AE_DIV(c, 12.92f) : powf_(AE_DIV(AE_ADD(c, 0.055f), 1.055f), 2.4f);
}

// Texel index of floor(x) (an integral float) under REPEAT addressing.
AE_HD uint32_t repeat_index(float fl, uint32_t n) {
    const float g = AE_FMIN(AE_FMAX(fl, -1073741824.0f), 1073741824.0f);
    const int64_t i = (int64_t)g;
    int64_t m = i % (int64_t)n;
    if (m < 0) m += (int64_t)n;
    return (uint32_t)m;
}

AE_HD f3 texel_linear(const uint32_t *layer, const float *lut, uint32_t w, uint32_t x, uint32_t y) {
    const uint32_t t = layer[(size_t)y * w + x];
    return mk(lut[t & 0xffu], lut[(t >> 8) & 0xffu], lut[(t >> 16) & 0xffu]);
}

// texels: layers * h * w RGBA8 words (r in the low byte), layer-major.
AE_HD f3 texture_sample(const uint32_t *texels, const float *lut, uint32_t w, uint32_t h, uint32_t layers,
                        uint32_t layer, float u, float v) {
    if (layers == 0u || w == 0u || h == 0u) return splat(1.0f);  // BuildGPUArray's white layer
    if (layer >= layers) layer = layers - 1u;
    if (!(AE_FABS(u) <= 3.4028234e38f)) u = 0.0f;
    if (!(AE_FABS(v) <= 3.4028234e38f)) v = 0.0f;
    const float x = AE_SUB(AE_MUL(u, AE_U2F(w)), 0.5f), y = AE_SUB(AE_MUL(v, AE_U2F(h)), 0.5f);
    const float fx = AE_FLOOR(x), fy = AE_FLOOR(y);
    const float ax = AE_SUB(x, fx), ay = AE_SUB(y, fy);
    const uint32_t x0 = repeat_index(fx, w), x1 = repeat_index(AE_ADD(fx, 1.0f), w);
    const uint32_t y0 = repeat_index(fy, h), y1 = repeat_index(AE_ADD(fy, 1.0f), h);
    const uint32_t *L = texels + (size_t)layer * w * h;
    const f3 c00 = texel_linear(L, lut, w, x0, y0), c10 = texel_linear(L, lut, w, x1, y0);
    const f3 c01 = texel_linear(L, lut, w, x0, y1), c11 = texel_linear(L, lut, w, x1, y1);
    const f3 top = c00 + (c10 - c00) * ax;
    const f3 bottom = c01 + (c11 - c01) * ax;
    return top + (bottom - top) * ay;
}

// Quaternion rotate, math/quat.hpp:211-217 and hybrid:521-526:
// v + w t + u x t with t = 2 (u x v).
AE_HD f3 quat_rotate(float qx, float qy, float qz, float qw, f3 v) {
    const f3 u = mk(qx, qy, qz);
    const f3 t = 2.0f * cross(u, v);
    return v + qw * t + cross(u, t);
}

}  // namespace ae
