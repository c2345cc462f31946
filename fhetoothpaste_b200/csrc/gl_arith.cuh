// Goldilocks (p = 2^64 - 2^32 + 1) arithmetic for sm_100a.
//
// Functions take and return canonical residues in [0, p) unless their comment
// says otherwise (the _lazy forms return any 64-bit representative). The 64x64-bit
// product is built from 32-bit IMAD chains (Blackwell has no 64-bit integer
// multiplier); the 128-bit result x = r0 + r1 2^32 + r2 2^64 + r3 2^96 is reduced
// with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p):  x = (r1:r0) - r3 + r2 (2^32 - 1).
#pragma once

#include <cstdint>

namespace tp {

constexpr uint64_t kP = 0xFFFFFFFF00000001ull;
constexpr uint64_t kEps = 0x00000000FFFFFFFFull;  // 2^64 mod p

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }
__device__ __forceinline__ uint64_t pack64(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }

// a + b mod p.  a + (b + eps) carries out iff a + b >= p, and then its low 64
// bits are a + b - p; without the carry the eps is taken back. The carry picks
// the correction directly: 0xFFFFFFFF + carry is 0 with it and eps without.
// (b < p keeps b + eps below 2^64; for any 64-bit a the result is still a
// 64-bit value congruent to a + b.)
__device__ __forceinline__ uint64_t gl_add(uint64_t a, uint64_t b) {
    uint32_t sl, sh;
    asm("{\n\t"
        ".reg .u32 bl, bh, m;\n\t"
        "add.cc.u32 bl, %2, 0xFFFFFFFF;\n\t"
        "addc.u32 bh, %3, 0;\n\t"
        "add.cc.u32 %0, %4, bl;\n\t"
        "addc.cc.u32 %1, %5, bh;\n\t"
        "addc.u32 m, 0xFFFFFFFF, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(sl), "=r"(sh)
        : "r"(lo32(b)), "r"(hi32(b)), "r"(lo32(a)), "r"(hi32(a)));
    return pack64(sl, sh);
}

// a + b as a 64-bit value congruent to it mod p (not necessarily below p), for
// any 64-bit a and b < p: a + b < 2^64 + p, so after a carry out the sum's low
// 64 bits plus eps stay below 2^64. Six instructions against gl_add's seven.
// (The carry is read with addc and negated with sub: a subc right after the
// addc.cc, reading the add's carry as a borrow, gave wrong words here.)
__device__ __forceinline__ uint64_t gl_add_lazy(uint64_t a, uint64_t b) {
    uint32_t sl, sh;
    asm("{\n\t"
        ".reg .u32 c, m;\n\t"
        "add.cc.u32 %0, %2, %4;\n\t"
        "addc.cc.u32 %1, %3, %5;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "sub.u32 m, 0, c;\n\t"
        "add.cc.u32 %0, %0, m;\n\t"
        "addc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(sl), "=r"(sh)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    return pack64(sl, sh);
}

// a - b mod p: on borrow add p, i.e. subtract eps modulo 2^64. For any 64-bit
// a and b < p the result is a 64-bit value congruent to a - b (a borrow means
// a < b, so a - b + 2^64 > 2^64 - p and taking eps off cannot underflow).
__device__ __forceinline__ uint64_t gl_sub(uint64_t a, uint64_t b) {
    uint32_t dl, dh;
    asm("{\n\t"
        ".reg .u32 m;\n\t"
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, %5;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(dl), "=r"(dh)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    return pack64(dl, dh);
}

// Canonical residue of any 64-bit value.
__device__ __forceinline__ uint64_t gl_canon(uint64_t x) { return x >= kP ? x - kP : x; }

// -a mod p.
__device__ __forceinline__ uint64_t gl_neg(uint64_t a) { return a == 0 ? 0 : kP - a; }

// 128-bit product a*b as four 32-bit words.
__device__ __forceinline__ void mul_wide(uint64_t a, uint64_t b, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                         uint32_t& r3) {
    asm("{\n\t"
        "mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
}

// Reduces x = r0 + r1 2^32 + r2 2^64 + r3 2^96 (any 128-bit value) to [0, p).
//   t = (r1:r0) - r3            (a borrow takes eps off: t stays >= 2^64 - 2^33 + 2)
//   S = t + r2 (2^32 - 1)       (the value to reduce, below 2^65 - 2^33)
// S + eps = t + (r2 2^32 + (2^32 - 1 - r2)), i.e. t plus the word pair
// (r2, ~r2): no multiply. If that sum carries out, S >= p and its low 64 bits
// are S - p, which is below p; otherwise S < p and the result is the sum minus
// eps (no underflow: the sum is at least eps). As in gl_add, 0xFFFFFFFF +
// carry gives the correction.
__device__ __forceinline__ uint64_t gl_reduce128(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t s0, s1;
    asm("{\n\t"
        ".reg .u32 t0, t1, b, n, m;\n\t"
        "sub.cc.u32 t0, %2, %5;\n\t"
        "subc.cc.u32 t1, %3, 0;\n\t"
        "subc.u32 b, 0, 0;\n\t"
        "sub.cc.u32 t0, t0, b;\n\t"
        "subc.u32 t1, t1, 0;\n\t"
        "not.b32 n, %4;\n\t"
        "add.cc.u32 %0, t0, n;\n\t"
        "addc.cc.u32 %1, t1, %4;\n\t"
        "addc.u32 m, 0xFFFFFFFF, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(s0), "=r"(s1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return pack64(s0, s1);
}

// a * b mod p.
__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    mul_wide(a, b, r0, r1, r2, r3);
    return gl_reduce128(r0, r1, r2, r3);
}

// acc + a*b as an exact 128-bit value (acc, a, b any 64-bit: the sum stays
// below 2^128), accumulated inside the multiply's carry chain.
__device__ __forceinline__ void mad_wide(uint64_t acc, uint64_t a, uint64_t b, uint32_t& r0, uint32_t& r1,
                                         uint32_t& r2, uint32_t& r3) {
    asm("{\n\t"
        "mad.lo.cc.u32 %0, %4, %6, %8;\n\t"
        "madc.hi.cc.u32 %1, %4, %6, %9;\n\t"
        "madc.lo.cc.u32 %2, %5, %7, 0;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)), "r"(lo32(acc)), "r"(hi32(acc)));
}

// acc + a*b mod p, canonical (any 64-bit inputs). The accumulate rides in the
// product's carry chain; the carry-form reduction needs no IMAD, which the
// product's own chain keeps busy (measured: +2% CGGI, +4% BMMP over a
// reduction that folds r2 (2^32 - 1) with mad.hi/mad.wide).
__device__ __forceinline__ uint64_t gl_fma(uint64_t acc, uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    mad_wide(acc, a, b, r0, r1, r2, r3);
    return gl_reduce128(r0, r1, r2, r3);
}

// hi * 2^64 + lo mod p as a 64-bit representative (not necessarily below p),
// for any hi, lo: hi 2^64 = h0 2^64 + h1 2^96 = h0 (2^32 - 1) - h1.
__device__ __forceinline__ uint64_t gl_fold(uint64_t hi, uint64_t lo) {
    const uint64_t h0 = hi & 0xFFFFFFFFull, h1 = hi >> 32;
    uint64_t t = lo - h1;
    if (lo < h1) t -= kEps;              // t was >= 2^64 - 2^32: no underflow
    const uint64_t u = (h0 << 32) - h0;  // h0 (2^32 - 1) < 2^64
    uint64_t s = t + u;
    if (s < u) s += kEps;                // wrapped s < u <= 2^64 - 2^33 + 1: no overflow
    return s;
}

// x * 2^K mod p for a compile-time K (canonical in and out), with shifts and
// adds only. Every root of unity of order dividing 64 is a power of two in this
// field (2 has order 192), so the twiddles of the first NTT levels are such
// shifts.
template <int K>
__device__ __forceinline__ uint64_t gl_mul_pow2(uint64_t x) {
    static_assert(K >= 0 && K < 192, "exponent out of range");
    if constexpr (K >= 96) {
        return gl_neg(gl_mul_pow2<K - 96>(x));  // 2^96 = -1
    } else if constexpr (K == 0) {
        return x;
    } else if constexpr (K < 64) {
        return gl_canon(gl_fold(x >> (64 - K), x << K));
    } else if constexpr (K == 64) {
        return gl_canon(gl_fold(x, 0));
    } else {
        return gl_canon(gl_fold(gl_fold(x >> (128 - K), x << (K - 64)), 0));
    }
}


}  // namespace tp
