// exact_math.h -- bit-exact float arithmetic shared by the host and the sm_100a kernels.
//
// Everything here is written with explicit round-to-nearest intrinsics on the device (__fadd_rn,
// __fmul_rn, __fmaf_rn, __fdiv_rn, __frcp_rn, __fsqrt_rn), which the compiler never contracts or
// reassociates, so a kernel computes exactly the IEEE-754 binary32 operation sequence the
// reference's C++ performs (compiled without contraction).
#pragma once

#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD inline
#include <cmath>
#endif

namespace pt {

#ifdef __CUDA_ARCH__
PT_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
PT_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
PT_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
PT_HD float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
PT_HD float fdiv(float a, float b) { return __fdiv_rn(a, b); }
PT_HD float frcp(float a) { return __frcp_rn(a); }
PT_HD float fsqrt(float a) { return __fsqrt_rn(a); }
PT_HD uint32_t fbits(float f) { return __float_as_uint(f); }
PT_HD float bitsf(uint32_t u) { return __uint_as_float(u); }
PT_HD int clz64(uint64_t x) { return __clzll((long long)x); }
#else
PT_HD float fadd(float a, float b) { return a + b; }
PT_HD float fsub(float a, float b) { return a - b; }
PT_HD float fmul(float a, float b) { return a * b; }
PT_HD float ffma(float a, float b, float c) { return std::fma(a, b, c); }
PT_HD float fdiv(float a, float b) { return a / b; }
PT_HD float frcp(float a) { return 1.0f / a; }
PT_HD float fsqrt(float a) { return std::sqrt(a); }
PT_HD uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
PT_HD float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
PT_HD int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
#endif
PT_HD float fabs_(float a) { return bitsf(fbits(a) & 0x7FFFFFFFu); }

// Read-only loads and the error flag, portable so the path code also builds for the host
// (used only by an off-line debugging harness; the library never runs it on the CPU).
template <class T>
PT_HD T ldg(const T* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
// L2 residency of the scene versus the ray stream.  A ray query reads its 32-B ray and writes its
// 16-B hit once, while every ray re-reads the upper tree and many leaves; on the 1.3 M-face
// microbench the 768 MiB of rays and hits per launch streamed through the same L2 as the 113 MB
// tree and pushed its hit rate down to 69 %.  With PT_L2_HINTS >= 1 rays and hits are loaded and
// stored cache-streaming (evict-first in L1 and L2); with PT_L2_HINTS >= 2 node and face loads
// also carry an L2::evict_last cache-hint policy.  Both are per-instruction hints: no device,
// context or stream attribute is set.
#ifndef PT_L2_HINTS
#define PT_L2_HINTS 2
#endif

#if defined(__CUDA_ARCH__) && PT_L2_HINTS >= 2
__device__ __forceinline__ uint64_t l2_keep_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
#endif

// One 32-byte node record (two uint4) with a single 256-bit read-only load on the device; the
// record must be 32-byte aligned (node arrays are cudaMalloc'd and nodes are 32 bytes).
PT_HD void ldg_node(const uint4* p, uint4& a, uint4& b) {
#if defined(__CUDA_ARCH__) && PT_L2_HINTS >= 2
    asm("ld.global.nc.L2::cache_hint.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p), "l"(l2_keep_policy()));
#elif defined(__CUDA_ARCH__)
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
#else
    a = p[0];
    b = p[1];
#endif
}
// One 16-byte part of a face record (read-only, kept in L2 like the nodes).
PT_HD float4 ldg_face(const float4* p) {
#if defined(__CUDA_ARCH__) && PT_L2_HINTS >= 2
    float4 v;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(l2_keep_policy()));
    return v;
#elif defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}
// Ray records read once and hit records written once: streamed past the caches.
PT_HD float4 ld_stream(const float4* p) {
#if defined(__CUDA_ARCH__) && PT_L2_HINTS >= 1
    return __ldcs(p);
#elif defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}
PT_HD void st_stream(uint4* p, uint4 v) {
#if defined(__CUDA_ARCH__) && PT_L2_HINTS >= 1
    __stcs(p, v);
#else
    *p = v;
#endif
}
PT_HD void raise_flag(int* flag) {
#ifdef __CUDA_ARCH__
    atomicExch(flag, 1);
#else
    *flag = 1;
#endif
}
PT_HD float next_up(float x) { return nextafterf(x, bitsf(0x7F800000u)); }
PT_HD float next_down(float x) { return nextafterf(x, bitsf(0xFF800000u)); }

// constants.h:62,142-148: gamma_n = (n * eps) / (1 - n * eps) with eps = 2^-24, in float, and
// BoundingBox.cpp:27: 1 + 2 * Gamma(3).  Bit patterns (checked against the host compiler's
// constant folding by the CPU tests).
#define PT_GAMMA2_BITS 0x34000001u
#define PT_GAMMA3_BITS 0x34400002u
#define PT_GAMMA5_BITS 0x34A00003u
#define PT_GAMMA7_BITS 0x34E00006u
#define PT_GAMMA_MUL_BITS 0x3F800003u

// constants.h:121-126
PT_HD float diff_prod(float a, float b, float c, float d) {
    const float cd = fmul(c, d);
    const float dop = ffma(a, b, -cd);
    const float err = ffma(-c, d, cd);
    return fadd(dop, err);
}
// constants.h:128-133
PT_HD float sum_prod(float a, float b, float c, float d) {
    const float cd = fmul(c, d);
    const float sop = ffma(a, b, cd);
    const float err = ffma(c, d, -cd);
    return fadd(sop, err);
}

// ------------------------------------------------------------------------------------------------
// (float)((double)a * (double)b - (double)c * (double)d) without FP64 instructions.
//
// The two double products are exact (24 + 24 bit significands).  Their difference is formed
// exactly in a 128-bit integer, rounded to 53 significant bits (the double subtraction), then to
// 24 bits with binary32 range handling (the conversion) -- both round-half-to-even, reproducing
// the double rounding of mesh.cpp:252-264.  When the exponents of the two products differ by more
// than 72, the smaller one lies entirely below the guard bit of the 53-bit rounding and is
// replaced by a single sticky unit, which leaves both roundings unchanged.  Non-finite inputs
// follow IEEE rules (NaN payloads are not reproduced).
namespace detail {
struct Prod { uint32_t sign; uint64_t mant; int exp; int kind; };  // kind: 0 finite, 1 inf, 2 nan

PT_HD void decompose(float f, uint32_t& sign, uint32_t& mant, int& exp, int& kind) {
    const uint32_t u = fbits(f);
    sign = u >> 31;
    const uint32_t e = (u >> 23) & 0xFFu, m = u & 0x7FFFFFu;
    if (e == 0xFFu) { kind = m ? 2 : 1; mant = 0; exp = 0; return; }
    kind = 0;
    if (e == 0) { mant = m; exp = -149; }
    else { mant = m | 0x800000u; exp = (int)e - 150; }
}

PT_HD Prod product(float a, float b) {
    uint32_t sa, sb, ma, mb; int ea, eb, ka, kb;
    decompose(a, sa, ma, ea, ka);
    decompose(b, sb, mb, eb, kb);
    Prod p;
    p.sign = sa ^ sb;
    if (ka == 2 || kb == 2) { p.kind = 2; p.mant = 0; p.exp = 0; return p; }
    if (ka == 1 || kb == 1) {
        const bool other_zero = (ka == 1) ? (kb == 0 && mb == 0) : (ka == 0 && ma == 0);
        p.kind = other_zero ? 2 : 1; p.mant = 0; p.exp = 0; return p;
    }
    p.kind = 0;
    p.mant = (uint64_t)ma * (uint64_t)mb;
    p.exp = ea + eb;
    return p;
}

PT_HD int topbit64(uint64_t x) { return 63 - clz64(x); }

// Round the exact value sign * q * 2^e (0 < q < 2^54) to binary32, half to even.
PT_HD float to_float(uint32_t sign, uint64_t q, int e) {
    const int tq = topbit64(q);
    const bool normal = (e + tq) >= -126;
    const int sh = normal ? (tq - 23) : (-149 - e);  // low bits to drop
    uint64_t m;
    if (sh <= 0) {
        m = q << (-sh);
    } else if (sh > 62) {
        m = 0;  // q < 2^54 <= half an ulp
    } else {
        m = q >> sh;
        const uint64_t rem = q & ((1ull << sh) - 1);
        const uint64_t half = 1ull << (sh - 1);
        if (rem > half || (rem == half && (m & 1))) m++;
    }
    int ef = e + sh;  // value = m * 2^ef
    uint32_t bits;
    if (!normal) {
        bits = (uint32_t)m;  // subnormal; m == 2^23 encodes the smallest normal
    } else {
        if (m == (1ull << 24)) { m >>= 1; ef += 1; }
        const int biased = ef + 23 + 127;
        bits = biased >= 255 ? 0x7F800000u : (((uint32_t)biased << 23) | ((uint32_t)m & 0x7FFFFFu));
    }
    return bitsf(bits | (sign << 31));
}
}  // namespace detail

#ifdef __CUDACC__
inline __host__ __device__ __noinline__  // rare path: kept out of line to spare registers
#else
inline
#endif
float f64_diff_emulated(float a, float b, float c, float d) {
    using namespace detail;
    const Prod A = product(a, b);
    Prod B = product(c, d);
    B.sign ^= 1u;                          // A - B = A + (-B)
    if (A.kind == 2 || B.kind == 2) return bitsf(0x7FC00000u);
    if (A.kind == 1 && B.kind == 1) return A.sign == B.sign ? bitsf(A.sign << 31 | 0x7F800000u) : bitsf(0x7FC00000u);
    if (A.kind == 1) return bitsf(A.sign << 31 | 0x7F800000u);
    if (B.kind == 1) return bitsf(B.sign << 31 | 0x7F800000u);
    if (A.mant == 0 && B.mant == 0) return bitsf((A.sign & B.sign) << 31);  // -0 only for (-0) + (-0)
    if (A.mant == 0) return to_float(B.sign, B.mant, B.exp);
    if (B.mant == 0) return to_float(A.sign, A.mant, A.exp);
    // normalize both significands to 48 bits (bit 47 set)
    uint64_t ma = A.mant, mb = B.mant;
    int ea = A.exp, eb = B.exp;
    const int sa = 47 - topbit64(ma), sb = 47 - topbit64(mb);
    ma <<= sa; ea -= sa;
    mb <<= sb; eb -= sb;
    uint32_t sbig = A.sign, ssmall = B.sign;
    uint64_t mbig = ma, msmall = mb;
    int ebig = ea, esmall = eb;
    if (eb > ea) { sbig = B.sign; ssmall = A.sign; mbig = mb; msmall = ma; ebig = eb; esmall = ea; }
    int dshift = ebig - esmall;
    if (dshift > 72) { msmall = 1; dshift = 72; esmall = ebig - 72; }
    // X = mbig << dshift (<= 120 bits) as (hi, lo); Y = msmall (< 2^48)
    uint64_t xhi, xlo;
    if (dshift == 0) { xhi = 0; xlo = mbig; }
    else if (dshift < 64) { xhi = mbig >> (64 - dshift); xlo = mbig << dshift; }
    else { xhi = mbig << (dshift - 64); xlo = 0; }
    uint64_t dhi, dlo;
    uint32_t sign;
    if (sbig == ssmall) {  // magnitudes add
        dlo = xlo + msmall;
        dhi = xhi + (dlo < xlo ? 1u : 0u);
        sign = sbig;
    } else {               // magnitudes subtract; |X| >= |Y| unless dshift == 0
        bool x_ge = (xhi != 0) || (xlo >= msmall);
        if (x_ge) {
            dlo = xlo - msmall;
            dhi = xhi - (xlo < msmall ? 1u : 0u);
            sign = sbig;
        } else {
            dlo = msmall - xlo;
            dhi = 0;
            sign = ssmall;
        }
        if (dhi == 0 && dlo == 0) return 0.0f;  // exact cancellation: +0
    }
    // round the 128-bit magnitude to 53 bits (double subtraction)
    int t = dhi ? 64 + topbit64(dhi) : topbit64(dlo);
    uint64_t q;
    int e2 = esmall;
    if (t > 52) {
        const int sh = t - 52;  // 1 .. 68
        uint64_t rem_hi, rem_lo, half_hi, half_lo;
        if (sh < 64) {
            q = (dlo >> sh) | (sh ? (dhi << (64 - sh)) : 0);
            rem_hi = 0; rem_lo = dlo & ((1ull << sh) - 1);
            half_hi = 0; half_lo = 1ull << (sh - 1);
        } else {
            q = dhi >> (sh - 64);
            rem_hi = dhi & ((sh - 64) ? ((1ull << (sh - 64)) - 1) : 0);
            rem_lo = dlo;
            if (sh == 64) { half_hi = 0; half_lo = 1ull << 63; }
            else { half_hi = 1ull << (sh - 65); half_lo = 0; }
        }
        const bool gt = rem_hi > half_hi || (rem_hi == half_hi && rem_lo > half_lo);
        const bool eq = rem_hi == half_hi && rem_lo == half_lo;
        if (gt || (eq && (q & 1))) q++;
        e2 += sh;
        if (q >> 53) { q >>= 1; e2 += 1; }
    } else {
        q = dlo;
    }
    return detail::to_float(sign, q, e2);
}

// ------------------------------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
PT_HD void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
PT_HD float u01(uint32_t x) { return fmul((float)(x >> 8), 5.9604644775390625e-08f); }

// sin/cos of 2*pi*u, u in [0, 1): quadrant q = rint(4u), r = 4u - q in [-1/2, 1/2], then Taylor
// polynomials of sin(pi/2 r) (to r^9) and cos(pi/2 r) (to r^10) with fma Horner steps.
PT_HD void sincos_2pi(float u, float& s, float& c) {
    const float f = fmul(4.0f, u);
#ifdef __CUDA_ARCH__
    const float q = rintf(f);
#else
    const float q = std::nearbyint(f);
#endif
    const float r = fsub(f, q);
    const float r2 = fmul(r, r);
    float ps = ffma(r2, 0.000160441184787359821833f, -0.00468175413531868810256f);
    ps = ffma(r2, ps, 0.0796926262461670451206f);
    ps = ffma(r2, ps, -0.645964097506246253655f);
    ps = ffma(r2, ps, 1.57079632679489661923f);
    const float sr = fmul(r, ps);
    float pc = ffma(r2, -0.0000252020423730606054811f, 0.000919260274839426215087f);
    pc = ffma(r2, pc, -0.0208634807633529608730f);
    pc = ffma(r2, pc, 0.253669507901048014030f);
    pc = ffma(r2, pc, -1.23370055013616982735f);
    const float cr = ffma(r2, pc, 1.0f);
    const int quad = ((int)q) & 3;
    if (quad == 0) { s = sr; c = cr; }
    else if (quad == 1) { s = cr; c = -sr; }
    else if (quad == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
}

}  // namespace pt
