// Thread-block negacyclic NTT over Goldilocks for one polynomial of N = 2^LOGN
// coefficients held E = 2^LOGE per thread (E = 8 or 4) by T = N/E threads.
//
// The transform is the reference's (lib/src/backend/solinas.cpp:228-313):
// forward = Cooley-Tukey, natural-order coefficients in, evaluations out in
// bit-reversed order (slot k = a(psi^(2 brv(k) + 1))), block i of the level
// with m blocks using psi^brv(m+i); backward = Gentleman-Sande with
// psi^-brv(m+i), natural order out, scaled by 1/N. Since every value is an
// exact residue, any evaluation order of the same butterflies gives the same
// words as the reference.
//
// Levels are processed in passes of up to LOGE (radix-E groups in registers).
// Radix-4 passes read a second table of twiddle products at tw + N (below).
// Between passes the data goes through a shared-memory exchange buffer of N
// words. Passes whose blocks span at most 32*E coefficients touch only their
// own warp's 32*E-word region, so those exchanges need only __syncwarp; the
// others use __syncthreads.
//
// Register layouts ("where thread t holds what"):
//   coefficient layout: x[j] = coefficient t + j*T            (pass 0 groups)
//   slot layout:        x[j] = slot E*t + j                    (last pass groups)
// forward: coefficient layout -> slot layout; backward: slot -> coefficient.
//
// Exchange-buffer hazards: a transform's first shared-memory write may race
// with another warp still reading the previous transform's last exchange, so
// callers alternate between two buffers; every transform run by more than one
// warp contains a block-wide barrier (its first exchange spans the whole
// polynomial), which orders transform k's reads before transform k+2's writes
// to the same buffer.
#pragma once

#include <type_traits>

#include "gl_arith.cuh"

namespace tp {

template <int LOGN, int LOGE = 3>
struct NttShape {
    static constexpr int N = 1 << LOGN;
    static constexpr int E = 1 << LOGE;       // coefficients per thread
    static constexpr int T = N / E;
    static constexpr int NPASS = (LOGN + LOGE - 1) / LOGE;
    __host__ __device__ static constexpr int L0(int p) { return LOGE * p; }
    __host__ __device__ static constexpr int S(int p) { return LOGE * p + LOGE <= LOGN ? LOGE : LOGN - LOGE * p; }
    // A pass whose level-L0 blocks have at most 32*E coefficients stays inside
    // the 32*E-word region of its warp.
    __host__ __device__ static constexpr bool WarpLocal(int p) { return LOGN - L0(p) <= 5 + LOGE; }
    static constexpr bool SingleWarp = (T <= 32);
};

// Swizzled position of coefficient/slot `idx` in an exchange buffer.
//  E = 8: 16-byte chunk c = idx/2 is stored at chunk c ^ ((c >> 3) & 7); keeps
//         every pass's 8-byte accesses (per half-warp) and the last pass's
//         16-byte accesses (per quarter-warp) free of bank conflicts.
//  E = 4: word idx is stored at idx ^ (5 * ((idx >> 4) & 3)) inside its 16-word
//         row. A half-warp's 8-byte accesses then hit 16 distinct bank pairs
//         for every pass shape (runs of 1, 2, 4, 8 or >= 16 consecutive words
//         at a stride of 4x the run); the last pass uses 8-byte accesses too.
template <int LOGE>
__device__ __forceinline__ int xpos(int idx) {
    if constexpr (LOGE == 3) {
        const int c = idx >> 1;
        return ((c ^ ((c >> 3) & 7)) << 1) | (idx & 1);
    } else {
        return idx ^ (5 * ((idx >> 4) & 3));
    }
}

// Index of the e-th register (0..E-1) of thread t in pass P.
template <int LOGN, int LOGE, int P>
__device__ __forceinline__ int pass_index(int t, int e) {
    using SH = NttShape<LOGN, LOGE>;
    constexpr int S = SH::S(P);
    constexpr int G = 1 << S;
    constexpr int PER = SH::E / G;
    constexpr int TMIN = SH::N >> (SH::L0(P) + S);
    const int q = e / G, j = e % G;
    const int g = PER * t + q;
    const int blk = g / TMIN, off = g % TMIN;
    return blk * G * TMIN + off + j * TMIN;
}

template <int LOGN, int LOGE>
__device__ __forceinline__ void ntt_sync(bool block_wide) {
    using SH = NttShape<LOGN, LOGE>;
    if (SH::T < 32 || block_wide) __syncthreads();
    else __syncwarp();
}

// The functions below transform K polynomials at once (x[k] is polynomial k;
// its exchange area is buf + k*N). The K transforms share every twiddle load
// and every synchronisation, and their independent butterflies interleave.

// Fused radix-4 passes (E = 4, optional) combine their two levels. With W1 = tw[m + b] (level L0,
// m = 2^L0, block b), W2 = tw[2m + 2b] and W3 = tw[2m + 2b + 1] = W2 w4, where
// w4 = psi^(N/2) = 2^48 is the 4th root of unity (brv(2i+1) = brv(2i) + N/2),
// the four outputs of the forward levels are
//   t1 = W1 x2, t2 = W2 x1, t3 = W1W2 x3
//   y0 = (x0 + t1) + (t2 + t3)     y1 = (x0 + t1) - (t2 + t3)
//   y2 = (x0 - t1) + w4 (t2 - t3)  y3 = (x0 - t1) - w4 (t2 - t3)
// three general products and one shift instead of four products. W1W2 is read
// from the product table at tw[N + m + b]. In pass 0 (b = 0) the twiddles are
// 2^48, 2^120, 2^168 and every product is a shift. This trades IMADs (FMA
// pipe) for shifts and adds (ALU pipe); it measured faster only where the FMA
// pipe is the busier one (BMMP, whose key MAC is 1.5x CGGI ternary's).
template <int LOGN, int P, int K, bool LAZY>
__device__ __forceinline__ void fwd_radix4(uint64_t (&x)[K][4], int t, const uint64_t* __restrict__ tw) {
    using SH = NttShape<LOGN, 2>;
    constexpr int TMIN = SH::N >> (SH::L0(P) + 2);
    constexpr int M = 1 << SH::L0(P);
    const int b = t / TMIN;
    uint64_t w1 = 0, w2 = 0, w12 = 0;
    if constexpr (P > 0) {
        w1 = tw[M + b];
        w2 = tw[2 * M + 2 * b];
        w12 = tw[SH::N + M + b];
    }
#pragma unroll
    for (int p = 0; p < K; ++p) {
        uint64_t t1, t2, t3;
        if constexpr (P == 0) {
            t1 = gl_mul_pow2<48>(x[p][2]);
            t2 = gl_mul_pow2<120>(x[p][1]);
            t3 = gl_mul_pow2<168>(x[p][3]);
        } else {
            t1 = gl_mul(x[p][2], w1);
            t2 = gl_mul(x[p][1], w2);
            t3 = gl_mul(x[p][3], w12);
        }
        // with LAZY, x0 may be any 64-bit value; t1, c and d are canonical
        const uint64_t a = LAZY ? gl_add_lazy(x[p][0], t1) : gl_add(x[p][0], t1), bb = gl_sub(x[p][0], t1);
        const uint64_t c = gl_add(t2, t3), d = gl_mul_pow2<48>(gl_sub(t2, t3));
        x[p][0] = LAZY ? gl_add_lazy(a, c) : gl_add(a, c);
        x[p][1] = gl_sub(a, c);
        x[p][2] = LAZY ? gl_add_lazy(bb, d) : gl_add(bb, d);
        x[p][3] = gl_sub(bb, d);
    }
}

// Inverse of the above (Gentleman-Sande, levels L0+1 then L0) with V = tw_inv:
//   g = x0 + x1, h = x2 + x3, e = x0 - x1, f = w4^-1 (x2 - x3)
//   y0 = g + h, y2 = V1 (g - h), y1 = V2 (e + f), y3 = V1V2 (e - f)
// In pass 0 the twiddles are 2^144, 2^72, 2^24 (w4^-1 = 2^144).
template <int LOGN, int P, int K>
__device__ __forceinline__ void inv_radix4(uint64_t (&x)[K][4], int t, const uint64_t* __restrict__ tw) {
    using SH = NttShape<LOGN, 2>;
    constexpr int TMIN = SH::N >> (SH::L0(P) + 2);
    constexpr int M = 1 << SH::L0(P);
    const int b = t / TMIN;
    uint64_t v1 = 0, v2 = 0, v12 = 0;
    if constexpr (P > 0) {
        v1 = tw[M + b];
        v2 = tw[2 * M + 2 * b];
        v12 = tw[SH::N + M + b];
    }
#pragma unroll
    for (int p = 0; p < K; ++p) {
        const uint64_t g = gl_add(x[p][0], x[p][1]), h = gl_add(x[p][2], x[p][3]);
        const uint64_t e = gl_sub(x[p][0], x[p][1]), f = gl_mul_pow2<144>(gl_sub(x[p][2], x[p][3]));
        x[p][0] = gl_add(g, h);
        if constexpr (P == 0) {
            x[p][2] = gl_mul_pow2<144>(gl_sub(g, h));
            x[p][1] = gl_mul_pow2<72>(gl_add(e, f));
            x[p][3] = gl_mul_pow2<24>(gl_sub(e, f));
        } else {
            x[p][2] = gl_mul(gl_sub(g, h), v1);
            x[p][1] = gl_mul(gl_add(e, f), v2);
            x[p][3] = gl_mul(gl_sub(e, f), v12);
        }
    }
}

// Exponent e of the power-of-two twiddle 2^e = psi^(+-brv(2^l + i)) of level
// l < 5, block i (the same for every N: psi^(N/2^(l+1)) = 2^g_l with g = 48,
// 120, 156, 78, 39, and block i uses 2^(g_l (2 brv_l(i) + 1))); the inverse
// table holds the negated exponents.
__host__ __device__ constexpr int pow2_twiddle_exp(int level, int block, bool inverse) {
    constexpr int g[5] = {48, 120, 156, 78, 39};
    int r = 0;
    for (int b = 0; b < level; ++b) r |= ((block >> b) & 1) << (level - 1 - b);
    const int e = (g[level] * (2 * r + 1)) % 192;
    return inverse ? (192 - e) % 192 : e;
}

// The butterflies of one pass whose first level L0 has its block B known at
// compile time (pass 0: B = 0; later passes: one instantiation per block, picked
// by a warp-uniform switch, below). Level L0 + LV pairs registers J and
// J + G/2^(LV+1) with twiddle block (B << LV) + (J >> (S - LV)), as the table
// path of fwd_pass_math does. Levels below 5 take their power-of-two twiddles as
// shifts (gl_pow2_mag): a sign of the twiddle swaps the butterfly's add and
// subtract. Deeper levels read the table.
template <int S, int L0, int B, int LV, int J, int K, bool LAZY>
__device__ __forceinline__ void fwd_blk_level(uint64_t (&x)[K][1 << S], const uint64_t* __restrict__ tw) {
    constexpr int G = 1 << S;
    if constexpr (J < G) {
        constexpr int half = G >> (LV + 1);
        if constexpr ((J & half) == 0) {
            constexpr int LVL = L0 + LV;
            constexpr int BI = (B << LV) + (J >> (S - LV));
            if constexpr (LVL < 5) {
                constexpr int EX = pow2_twiddle_exp(LVL, BI, false);
#pragma unroll
                for (int p = 0; p < K; ++p) {
                    const uint64_t u = x[p][J];
                    const uint64_t t = gl_pow2_mag<EX>(x[p][J + half]);
                    const uint64_t sum = LAZY ? gl_add_lazy(u, t) : gl_add(u, t);
                    const uint64_t dif = gl_sub(u, t);
                    x[p][J] = Pow2<EX>::NEG ? dif : sum;
                    x[p][J + half] = Pow2<EX>::NEG ? sum : dif;
                }
            } else {
                const uint64_t w = tw[(1 << LVL) + BI];
#pragma unroll
                for (int p = 0; p < K; ++p) {
                    const uint64_t u = x[p][J];
                    const uint64_t v = gl_mul(x[p][J + half], w);
                    x[p][J] = LAZY ? gl_add_lazy(u, v) : gl_add(u, v);
                    x[p][J + half] = gl_sub(u, v);
                }
            }
        }
        fwd_blk_level<S, L0, B, LV, J + 1, K, LAZY>(x, tw);
    }
}
template <int S, int L0, int B, int LV, int K, bool LAZY>
__device__ __forceinline__ void fwd_blk_pass(uint64_t (&x)[K][1 << S], const uint64_t* __restrict__ tw) {
    if constexpr (LV < S) {
        fwd_blk_level<S, L0, B, LV, 0, K, LAZY>(x, tw);
        fwd_blk_pass<S, L0, B, LV + 1, K, LAZY>(x, tw);
    }
}
// Inverse (Gentleman-Sande): (u, v) -> (u + v, (u - v) w); a negative
// power-of-two twiddle multiplies v - u by its magnitude instead.
template <int S, int L0, int B, int LV, int J, int K>
__device__ __forceinline__ void inv_blk_level(uint64_t (&x)[K][1 << S], const uint64_t* __restrict__ tw) {
    constexpr int G = 1 << S;
    if constexpr (J < G) {
        constexpr int half = G >> (LV + 1);
        if constexpr ((J & half) == 0) {
            constexpr int LVL = L0 + LV;
            constexpr int BI = (B << LV) + (J >> (S - LV));
            if constexpr (LVL < 5) {
                constexpr int EX = pow2_twiddle_exp(LVL, BI, true);
#pragma unroll
                for (int p = 0; p < K; ++p) {
                    const uint64_t u = x[p][J];
                    const uint64_t v = x[p][J + half];
                    x[p][J] = gl_add(u, v);
                    x[p][J + half] = gl_pow2_mag<EX>(Pow2<EX>::NEG ? gl_sub(v, u) : gl_sub(u, v));
                }
            } else {
                const uint64_t w = tw[(1 << LVL) + BI];
#pragma unroll
                for (int p = 0; p < K; ++p) {
                    const uint64_t u = x[p][J];
                    const uint64_t v = x[p][J + half];
                    x[p][J] = gl_add(u, v);
                    x[p][J + half] = gl_mul(gl_sub(u, v), w);
                }
            }
        }
        inv_blk_level<S, L0, B, LV, J + 1, K>(x, tw);
    }
}
template <int S, int L0, int B, int LV, int K>
__device__ __forceinline__ void inv_blk_pass(uint64_t (&x)[K][1 << S], const uint64_t* __restrict__ tw) {
    if constexpr (LV >= 0) {
        inv_blk_level<S, L0, B, LV, 0, K>(x, tw);
        inv_blk_pass<S, L0, B, LV - 1, K>(x, tw);
    }
}

// f(std::integral_constant<int, b>{}) for a runtime b in [0, NB), NB <= 16: one
// instantiation per block, entered through a switch. Callers pass a b that is the
// same across the warp, so the jump does not diverge.
template <int NB, class F>
__device__ __forceinline__ void block_switch(int b, F&& f) {
    static_assert(NB >= 1 && NB <= 16, "up to 16 blocks");
#define TP_BLOCK_CASE(i)                                              \
    case i:                                                           \
        if constexpr (i < NB) f(std::integral_constant<int, i>{});    \
        break;
    switch (b) {
        TP_BLOCK_CASE(0) TP_BLOCK_CASE(1) TP_BLOCK_CASE(2) TP_BLOCK_CASE(3)
        TP_BLOCK_CASE(4) TP_BLOCK_CASE(5) TP_BLOCK_CASE(6) TP_BLOCK_CASE(7)
        TP_BLOCK_CASE(8) TP_BLOCK_CASE(9) TP_BLOCK_CASE(10) TP_BLOCK_CASE(11)
        TP_BLOCK_CASE(12) TP_BLOCK_CASE(13) TP_BLOCK_CASE(14) TP_BLOCK_CASE(15)
        default: break;
    }
#undef TP_BLOCK_CASE
}

// Transform forms: template flags of the pass functions below.
constexpr int kNttRadix4 = 1;       // fused radix-4 passes (4 coefficients per thread)
constexpr int kNttTablePasses = 2;  // later passes read table twiddles even on power-of-two levels

// A later pass (P > 0) takes its power-of-two levels as shifts when its twiddle
// block is the same for a whole warp: one radix-G group per thread (G = E) and
// at least 32 threads per block (TMIN >= 32), so blk = t / TMIN is warp-uniform
// and selects a compile-time instantiation. Only passes that start with at most
// 4 blocks (first level 2 with 4 per thread, levels 2-3; level 3 with 8, levels
// 3-5 of which 3-4 shift): the 16-way form that also takes level 4 with 4 per
// thread made the rotation kernels spill and measured slower.
template <int LOGN, int LOGE, int P>
__host__ __device__ constexpr bool pow2_block_pass() {
    using SH = NttShape<LOGN, LOGE>;
    return P > 0 && SH::S(P) == LOGE && SH::L0(P) < 5 && (SH::N >> (SH::L0(P) + SH::S(P))) >= 32 &&
           (1 << SH::L0(P)) <= 4;
}

// Forward butterflies of pass P on the thread's registers (FORM: kNttRadix4 uses
// the fused radix-4 form for radix-4 passes, kNttTablePasses keeps the later
// passes on table twiddles; LAZY: see ntt_forward_k).
template <int LOGN, int P, int K, int LOGE, int FORM, bool LAZY>
__device__ __forceinline__ void fwd_pass_math(uint64_t (&x)[K][1 << LOGE], int t, const uint64_t* __restrict__ tw) {
    using SH = NttShape<LOGN, LOGE>;
    constexpr int S = SH::S(P);
    if constexpr ((FORM & kNttRadix4) && LOGE == 2 && S == 2) {
        fwd_radix4<LOGN, P, K, LAZY>(x, t, tw);
    } else if constexpr (P == 0 && S == LOGE) {
        fwd_blk_pass<LOGE, 0, 0, 0, K, LAZY>(x, tw);
    } else if constexpr (!(FORM & kNttTablePasses) && pow2_block_pass<LOGN, LOGE, P>()) {
        constexpr int TMIN = SH::N >> (SH::L0(P) + S);
        block_switch<(1 << SH::L0(P))>(t / TMIN, [&](auto blk) {
            fwd_blk_pass<LOGE, SH::L0(P), decltype(blk)::value, 0, K, LAZY>(x, tw);
        });
    } else {
        constexpr int G = 1 << S;
        constexpr int PER = SH::E / G;
        constexpr int TMIN = SH::N >> (SH::L0(P) + S);
        constexpr int L0 = SH::L0(P);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int blk = (PER * t + q) / TMIN;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int half = G >> (k + 1);
#pragma unroll
                for (int j = 0; j < G; ++j) {
                    if (j & half) continue;
                    const uint64_t w = tw[(1 << (L0 + k)) + (blk << k) + (j >> (S - k))];
#pragma unroll
                    for (int p = 0; p < K; ++p) {
                        const uint64_t u = x[p][q * G + j];
                        const uint64_t v = gl_mul(x[p][q * G + j + half], w);
                        x[p][q * G + j] = LAZY ? gl_add_lazy(u, v) : gl_add(u, v);
                        x[p][q * G + j + half] = gl_sub(u, v);
                    }
                }
            }
        }
    }
}

// Inverse butterflies of pass P (levels in reverse order).
template <int LOGN, int P, int K, int LOGE, int FORM>
__device__ __forceinline__ void inv_pass_math(uint64_t (&x)[K][1 << LOGE], int t, const uint64_t* __restrict__ tw) {
    using SH = NttShape<LOGN, LOGE>;
    constexpr int S = SH::S(P);
    if constexpr ((FORM & kNttRadix4) && LOGE == 2 && S == 2) {
        inv_radix4<LOGN, P, K>(x, t, tw);
    } else if constexpr (P == 0 && S == LOGE) {
        inv_blk_pass<LOGE, 0, 0, LOGE - 1, K>(x, tw);
    } else if constexpr (!(FORM & kNttTablePasses) && pow2_block_pass<LOGN, LOGE, P>()) {
        constexpr int TMIN = SH::N >> (SH::L0(P) + S);
        block_switch<(1 << SH::L0(P))>(t / TMIN, [&](auto blk) {
            inv_blk_pass<LOGE, SH::L0(P), decltype(blk)::value, LOGE - 1, K>(x, tw);
        });
    } else {
        constexpr int G = 1 << S;
        constexpr int PER = SH::E / G;
        constexpr int TMIN = SH::N >> (SH::L0(P) + S);
        constexpr int L0 = SH::L0(P);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int blk = (PER * t + q) / TMIN;
#pragma unroll
            for (int k = S - 1; k >= 0; --k) {
                const int half = G >> (k + 1);
#pragma unroll
                for (int j = 0; j < G; ++j) {
                    if (j & half) continue;
                    const uint64_t w = tw[(1 << (L0 + k)) + (blk << k) + (j >> (S - k))];
#pragma unroll
                    for (int p = 0; p < K; ++p) {
                        const uint64_t u = x[p][q * G + j];
                        const uint64_t v = x[p][q * G + j + half];
                        x[p][q * G + j] = gl_add(u, v);
                        x[p][q * G + j + half] = gl_mul(gl_sub(u, v), w);
                    }
                }
            }
        }
    }
}

template <int LOGN, int P, int K, int LOGE>
__device__ __forceinline__ void xstore(uint64_t* buf, const uint64_t (&x)[K][1 << LOGE], int t) {
    using SH = NttShape<LOGN, LOGE>;
#pragma unroll
    for (int p = 0; p < K; ++p) {
        uint64_t* b = buf + p * SH::N;
        if constexpr (P == SH::NPASS - 1 && LOGE == 3) {
            // slot layout: 8 contiguous words, written as four 16-byte chunks
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int idx = 8 * t + 2 * c;
                *reinterpret_cast<ulonglong2*>(b + xpos<LOGE>(idx)) = make_ulonglong2(x[p][2 * c], x[p][2 * c + 1]);
            }
        } else {
#pragma unroll
            for (int e = 0; e < SH::E; ++e) b[xpos<LOGE>(pass_index<LOGN, LOGE, P>(t, e))] = x[p][e];
        }
    }
}

template <int LOGN, int P, int K, int LOGE>
__device__ __forceinline__ void xload(const uint64_t* buf, uint64_t (&x)[K][1 << LOGE], int t) {
    using SH = NttShape<LOGN, LOGE>;
#pragma unroll
    for (int p = 0; p < K; ++p) {
        const uint64_t* b = buf + p * SH::N;
        if constexpr (P == SH::NPASS - 1 && LOGE == 3) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int idx = 8 * t + 2 * c;
                const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(b + xpos<LOGE>(idx));
                x[p][2 * c] = v.x;
                x[p][2 * c + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int e = 0; e < SH::E; ++e) x[p][e] = b[xpos<LOGE>(pass_index<LOGN, LOGE, P>(t, e))];
        }
    }
}

template <int LOGN, int P, int K, int LOGE, int FORM, bool LAZY>
__device__ __forceinline__ void fwd_passes_from(uint64_t (&x)[K][1 << LOGE], int t, uint64_t* buf,
                                                const uint64_t* tw) {
    using SH = NttShape<LOGN, LOGE>;
    fwd_pass_math<LOGN, P, K, LOGE, FORM, LAZY>(x, t, tw);
    if constexpr (P + 1 < SH::NPASS) {
        xstore<LOGN, P, K, LOGE>(buf, x, t);
        ntt_sync<LOGN, LOGE>(!SH::WarpLocal(P));
        xload<LOGN, P + 1, K, LOGE>(buf, x, t);
        fwd_passes_from<LOGN, P + 1, K, LOGE, FORM, LAZY>(x, t, buf, tw);
    }
}

template <int LOGN, int P, int K, int LOGE, int FORM>
__device__ __forceinline__ void inv_passes_from(uint64_t (&x)[K][1 << LOGE], int t, uint64_t* buf,
                                                const uint64_t* tw) {
    using SH = NttShape<LOGN, LOGE>;
    inv_pass_math<LOGN, P, K, LOGE, FORM>(x, t, tw);
    if constexpr (P > 0) {
        xstore<LOGN, P, K, LOGE>(buf, x, t);
        ntt_sync<LOGN, LOGE>(!SH::WarpLocal(P - 1));
        xload<LOGN, P - 1, K, LOGE>(buf, x, t);
        inv_passes_from<LOGN, P - 1, K, LOGE, FORM>(x, t, buf, tw);
    }
}

// Forward NTT of K polynomials: coefficient layout -> slot layout. buf holds K*N words.
// FORM: kNttRadix4 (4 coefficients per thread only) selects the fused radix-4
// butterflies, whose twiddle products sit at tw_fwd + N; kNttTablePasses keeps
// the power-of-two levels of passes after the first on table twiddles.
// LAZY: the outputs are 64-bit values congruent to the evaluations but not
// necessarily below p, for callers that only multiply them (gl_mul,
// gl_fma take any 64-bit operand). Each butterfly's sum then skips the
// canonical step (gl_add_lazy: its right operand, the twiddle product, is
// canonical; the left may be any 64-bit value, and gl_sub takes that too). The
// inputs must be canonical (the radix-4 form's first pass shifts them).
template <int LOGN, int K, int LOGE = 3, int FORM = 0, bool LAZY = false>
__device__ __forceinline__ void ntt_forward_k(uint64_t (&x)[K][1 << LOGE], int t, uint64_t* buf,
                                              const uint64_t* tw_fwd) {
    fwd_passes_from<LOGN, 0, K, LOGE, FORM, LAZY>(x, t, buf, tw_fwd);
}

// The rest of a forward transform whose pass 0 the caller has already applied to x
// (same layouts and LAZY rule as ntt_forward_k).
template <int LOGN, int K, int LOGE, int FORM = 0, bool LAZY = false>
__device__ __forceinline__ void ntt_forward_after_pass0(uint64_t (&x)[K][1 << LOGE], int t, uint64_t* buf,
                                                        const uint64_t* tw_fwd) {
    using SH = NttShape<LOGN, LOGE>;
    if constexpr (SH::NPASS > 1) {
        xstore<LOGN, 0, K, LOGE>(buf, x, t);
        ntt_sync<LOGN, LOGE>(!SH::WarpLocal(0));
        xload<LOGN, 1, K, LOGE>(buf, x, t);
        fwd_passes_from<LOGN, 1, K, LOGE, FORM, LAZY>(x, t, buf, tw_fwd);
    }
}

// Pass 0 of the forward transform (levels 0 and 1, 4 coefficients per thread) for
// small signed inputs d_j (coefficients t + jT), in exact 64-bit integer arithmetic.
// Its twiddles are 2^48 (level 0), 2^120 = -2^24 and 2^168 = 2^-24 (level 1); with
// 2^72 = 2^40 - 2^8 and 2^88 = 2^56 - 2^24 (mod p) the four outputs are
//   y0 = A - P, y1 = A + P, y2 = B - Q, y3 = B + Q,
//   A = d0 + 2^48 d2, B = d0 - 2^48 d2,
//   P = 2^24 d1 + (2^40 - 2^8) d3, Q = (2^40 - 2^8) d1 + 2^24 d3,
// exact as long as |d_j| (1 + 2^8 + 2^24 + 2^40 + 2^48) < 2^63, i.e. |d_j| <= 2^14.
// A negative y is its 64-bit pattern y + 2^64 = y + eps (mod p), so eps is taken off
// (giving y + p); the outputs are canonical. Replaces two levels of butterflies.
__device__ __forceinline__ int64_t shl_signed(int64_t v, int k) { return (int64_t)((uint64_t)v << k); }

__device__ __forceinline__ void ntt_pass0_small(const int64_t (&d)[4], uint64_t (&y)[4]) {
    const int64_t a = d[0] + shl_signed(d[2], 48), b = d[0] - shl_signed(d[2], 48);
    const int64_t pp = shl_signed(d[1], 24) + shl_signed(d[3], 40) - shl_signed(d[3], 8);
    const int64_t qq = shl_signed(d[1], 40) - shl_signed(d[1], 8) + shl_signed(d[3], 24);
    const int64_t v[4] = {a - pp, a + pp, b - qq, b + qq};
#pragma unroll
    for (int j = 0; j < 4; ++j) y[j] = (uint64_t)v[j] - (v[j] < 0 ? kEps : 0ull);
}

// Backward NTT of K polynomials without the 1/N factor: slot -> coefficient layout.
template <int LOGN, int K, int LOGE = 3, int FORM = 0>
__device__ __forceinline__ void ntt_backward_unscaled_k(uint64_t (&x)[K][1 << LOGE], int t, uint64_t* buf,
                                                        const uint64_t* tw_inv) {
    inv_passes_from<LOGN, NttShape<LOGN, LOGE>::NPASS - 1, K, LOGE, FORM>(x, t, buf, tw_inv);
}

// One polynomial, 8 coefficients per thread.
template <int LOGN>
__device__ __forceinline__ void ntt_forward(uint64_t (&x)[8], int t, uint64_t* buf, const uint64_t* tw_fwd) {
    ntt_forward_k<LOGN, 1, 3>(reinterpret_cast<uint64_t(&)[1][8]>(x), t, buf, tw_fwd);
}

template <int LOGN>
__device__ __forceinline__ void ntt_backward_unscaled(uint64_t (&x)[8], int t, uint64_t* buf,
                                                      const uint64_t* tw_inv) {
    ntt_backward_unscaled_k<LOGN, 1, 3>(reinterpret_cast<uint64_t(&)[1][8]>(x), t, buf, tw_inv);
}

}  // namespace tp
