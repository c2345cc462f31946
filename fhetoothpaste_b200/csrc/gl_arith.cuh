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
// 64 bits plus eps stay below 2^64. Six instructions against gl_add's seven; the
// five carry adds are written as multiply-adds by 1 so that they issue on the
// IMAD pipe: the forward transforms that use this sum are otherwise ALU-bound
// (their butterflies put 9 IMADs against 22 ALU instructions). Measured on the
// rotation kernel: +2.0% CGGI ternary N = 2048, +1.2% binary N = 1024, +0.8%
// BMMP; moving gl_add's or the reduction's adds as well measured slower.
// (The carry is read with addc and negated with sub: a subc right after the
// addc.cc, reading the add's carry as a borrow, gave wrong words here.)
__device__ __forceinline__ uint64_t gl_add_lazy(uint64_t a, uint64_t b) {
    uint32_t sl, sh;
    asm("{\n\t"
        ".reg .u32 c, m;\n\t"
        "mad.lo.cc.u32 %0, %2, 1, %4;\n\t"
        "madc.lo.cc.u32 %1, %3, 1, %5;\n\t"
        "madc.lo.u32 c, 0, 0, 0;\n\t"
        "sub.u32 m, 0, c;\n\t"
        "mad.lo.cc.u32 %0, m, 1, %0;\n\t"
        "madc.lo.u32 %1, %1, 1, 0;\n\t"
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

// Exact sum of many 64x64-bit products, reduced once at the end. D holds the
// sum of x0 k0 + x1 k1 2^64 in five words (d4 counts carries out of 2^128), M
// the cross products x0 k1 + x1 k0 in three words weighted 2^32; a term costs
// the product's eight IMADs and three carry adds, against a product chain plus
// an eleven-instruction reduction per term for a running canonical sum. Up to
// 2^32 terms fit (the carry words cannot wrap).
struct WideAcc {
    uint32_t d0, d1, d2, d3, d4, m0, m1, m2;
};

__device__ __forceinline__ void wide_zero(WideAcc& a) { a = WideAcc{0, 0, 0, 0, 0, 0, 0, 0}; }

// a += x * k (x, k any 64-bit values).
__device__ __forceinline__ void wide_mad(WideAcc& a, uint64_t x, uint64_t k) {
    asm("{\n\t"
        "mad.lo.cc.u32 %0, %8, %10, %0;\n\t"
        "madc.hi.cc.u32 %1, %8, %10, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        "mad.lo.cc.u32 %5, %8, %11, %5;\n\t"
        "madc.hi.cc.u32 %6, %8, %11, %6;\n\t"
        "addc.u32 %7, %7, 0;\n\t"
        "mad.lo.cc.u32 %5, %9, %10, %5;\n\t"
        "madc.hi.cc.u32 %6, %9, %10, %6;\n\t"
        "addc.u32 %7, %7, 0;\n\t"
        "}"
        : "+r"(a.d0), "+r"(a.d1), "+r"(a.d2), "+r"(a.d3), "+r"(a.d4), "+r"(a.m0), "+r"(a.m1), "+r"(a.m2)
        : "r"(lo32(x)), "r"(hi32(x)), "r"(lo32(k)), "r"(hi32(k)));
}

// The accumulated value mod p, canonical. V = s0 + s1 2^32 + s2 2^64 + s3 2^96
// + s4 2^128 with s = D + M 2^32; 2^128 = -2^32 and 2^96 = -1 make
// V = (s1:s0) - (s4:s3) + s2 (2^32 - 1): gl_reduce128 with a two-word
// subtrahend ((s4:s3) is far below p, so adding p after a borrow keeps t >= 0).
__device__ __forceinline__ uint64_t wide_reduce(const WideAcc& a) {
    uint32_t s0, s1;
    asm("{\n\t"
        ".reg .u32 w1, w2, w3, w4, t0, t1, b, n, m;\n\t"
        "add.cc.u32 w1, %3, %7;\n\t"
        "addc.cc.u32 w2, %4, %8;\n\t"
        "addc.cc.u32 w3, %5, %9;\n\t"
        "addc.u32 w4, %6, 0;\n\t"
        "sub.cc.u32 t0, %2, w3;\n\t"
        "subc.cc.u32 t1, w1, w4;\n\t"
        "subc.u32 b, 0, 0;\n\t"
        "sub.cc.u32 t0, t0, b;\n\t"
        "subc.u32 t1, t1, 0;\n\t"
        "not.b32 n, w2;\n\t"
        "add.cc.u32 %0, t0, n;\n\t"
        "addc.cc.u32 %1, t1, w2;\n\t"
        "addc.u32 m, 0xFFFFFFFF, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(s0), "=r"(s1)
        : "r"(a.d0), "r"(a.d1), "r"(a.d2), "r"(a.d3), "r"(a.d4), "r"(a.m0), "r"(a.m1), "r"(a.m2));
    return pack64(s0, s1);
}

// Multiplication by powers of two. 2 has order 192 in this field (2^96 = -1),
// and every root of unity of order dividing 64 is a power of two, so the
// twiddles of the first NTT levels are such multiplications. Each form below
// takes any 64-bit x and returns a canonical residue, with shifts and adds
// only (no IMAD).

// (W1:W0) + W2 2^64 = (W1:W0) + W2 (2^32 - 1) mod p, canonical: the tail of
// gl_reduce128 (t + the word pair (W2, ~W2), the carry picks the correction).
__device__ __forceinline__ uint64_t gl_reduce96(uint32_t w0, uint32_t w1, uint32_t w2) {
    uint32_t s0, s1;
    asm("{\n\t"
        ".reg .u32 n, m;\n\t"
        "not.b32 n, %4;\n\t"
        "add.cc.u32 %0, %2, n;\n\t"
        "addc.cc.u32 %1, %3, %4;\n\t"
        "addc.u32 m, 0xFFFFFFFF, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(s0), "=r"(s1)
        : "r"(w0), "r"(w1), "r"(w2));
    return pack64(s0, s1);
}

// x 2^K mod p for a compile-time K in [0, 64). For K < 32, x 2^K is the three
// words (x0 << K, funnel(x0, x1), x1 >> (32 - K)); for K >= 32 those words of
// x 2^(K-32) sit one word higher and the four-word reduction folds them.
template <int K>
__device__ __forceinline__ uint64_t gl_shl(uint64_t x) {
    static_assert(K >= 0 && K < 64, "shift out of range");
    constexpr int R = K & 31;
    const uint32_t x0 = lo32(x), x1 = hi32(x);
    const uint32_t w0 = R ? x0 << R : x0;
    const uint32_t w1 = R ? __funnelshift_l(x0, x1, R) : x1;
    const uint32_t w2 = R ? x1 >> ((32 - R) & 31) : 0u;
    if constexpr (K == 0) {
        return gl_canon(x);
    } else if constexpr (K < 32) {
        return gl_reduce96(w0, w1, w2);
    } else {
        return gl_reduce128(0u, w0, w1, w2);
    }
}

// x 2^-K mod p for a compile-time K in [1, 32]. With x = h 2^K + l (l < 2^K),
// l 2^-K = l 2^(192-K) = -l 2^(96-K) = -y 2^64 = -y (2^32 - 1), y = l 2^(32-K)
// below 2^32 (the low word of x shifted up). So x 2^-K = A - B with
// A = h + y and B = y 2^32; on a borrow p is added (eps taken off modulo 2^64).
// B - A <= y (2^32 - 1) < p, so the result is canonical.
template <int K>
__device__ __forceinline__ uint64_t gl_shr(uint64_t x) {
    static_assert(K >= 1 && K <= 32, "shift out of range");
    const uint32_t x0 = lo32(x), x1 = hi32(x);
    const uint32_t h0 = K < 32 ? __funnelshift_r(x0, x1, K & 31) : x1;
    const uint32_t h1 = K < 32 ? x1 >> (K & 31) : 0u;
    const uint32_t y = K < 32 ? x0 << ((32 - K) & 31) : x0;
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 a0, a1, d1, m;\n\t"
        "add.cc.u32 a0, %2, %4;\n\t"
        "addc.u32 a1, %3, 0;\n\t"
        "sub.cc.u32 d1, a1, %4;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, a0, m;\n\t"
        "subc.u32 %1, d1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(h0), "r"(h1), "r"(y));
    return pack64(r0, r1);
}

// 2^E (E taken mod 192) as +-2^SHIFT with SHIFT in (-32, 64): exponents in
// [64, 96) and [160, 192) become negative shifts (2^E = -2^(E-96), 2^(E-192)),
// [96, 160) a sign and E - 96.
template <int E>
struct Pow2 {
    static constexpr int e = ((E % 192) + 192) % 192;
    static constexpr bool NEG = e >= 64 && e < 160;
    static constexpr int SHIFT = e < 64 ? e : (e < 160 ? e - 96 : e - 192);
};

// |2^E| x: x 2^SHIFT of Pow2<E> (the sign is the caller's: butterflies swap
// their add and subtract instead of negating).
template <int E>
__device__ __forceinline__ uint64_t gl_pow2_mag(uint64_t x) {
    constexpr int S = Pow2<E>::SHIFT;
    if constexpr (S >= 0) return gl_shl<(S >= 0 ? S : 0)>(x);
    else return gl_shr<(S < 0 ? -S : 1)>(x);
}

// x * N^-1 mod p for N = 2^LOGN (N^-1 = 2^-LOGN): a shift multiply.
template <int LOGN>
__device__ __forceinline__ uint64_t gl_div_pow2(uint64_t x) {
    return gl_shr<LOGN <= 32 ? LOGN : 32>(x);
}

// x * 2^K mod p for a compile-time K (canonical out, any 64-bit x in).
template <int K>
__device__ __forceinline__ uint64_t gl_mul_pow2(uint64_t x) {
    const uint64_t t = gl_pow2_mag<K>(x);
    return Pow2<K>::NEG ? gl_neg(t) : t;
}

}  // namespace tp
