// Negacyclic NTT of one polynomial of N = 2^LOGN coefficients spread over a
// cluster of S = 2^LOGS CTAs, S = 2 .. 16 (N > 4096: one CTA's shared memory
// cannot hold a rotation at that size). 4 coefficients per thread, T = N / (4 S)
// threads per CTA; the local size NL = N / S.
//
// Layouts (CTA rank r of the cluster):
//   coefficient layout: CTA r holds the coefficients i = i' S + r (the
//     subsequence r), local index i' in the NttShape<LOGN - LOGS> coefficient
//     layout of the block engine (thread t holds i' = t + j T).
//   slot layout: CTA r holds the slots r NL .. r NL + NL - 1, thread t the four
//     slots r NL + 4t + j (the block engine's slot layout on the local block).
//
// Forward (the reference's Cooley-Tukey order, lib/src/backend/solinas.cpp:228-261):
// the first LOGN - LOGS levels pair coefficients at distances of at least S, all
// inside one subsequence: they are exactly the NL-point negacyclic transform of
// the subsequence (psi_N^S = psi_NL and psi_N^brv_N(x) = psi_NL^brv_NL(x) for
// x < NL, so even the twiddle words agree), run by the block engine on each CTA.
// After it, position P = i' S + r holds the partial value of slot-group i'; the
// last LOGS levels combine the S positions of a group (distances S/2 .. 1, block
// index P / (2 distance)) with twiddles from the N-point table. One exchange
// through distributed shared memory brings every group to the CTA that owns its
// slots (group g to CTA g / (NL / S)); those levels then run in registers.
// Backward (Gentleman-Sande, solinas.cpp:263-313) is the mirror image: the group
// levels first on the owner, one exchange back to the subsequence owners, then the
// local NL-point backward transform. No 1/N factor (callers scale by 2^-LOGN).
//
// Exchanges alternate between two receive areas of NL words per CTA, and each is
// followed by one cluster barrier: transform k's remote writes go to area k mod 2,
// whose readers finished with it (transform k-2) before they arrived at transform
// k-1's barrier, which the writers have passed.
#pragma once

#include <cooperative_groups.h>

#include "gl_arith.cuh"
#include "ntt_block.cuh"

namespace tp {

template <int LOGN, int LOGS>
struct ClusterShape {
    static constexpr int N = 1 << LOGN;
    static constexpr int S = 1 << LOGS;
    static constexpr int LOGL = LOGN - LOGS;
    static constexpr int NL = 1 << LOGL;
    static constexpr int T = NL / 4;
    static constexpr int G = NL / S;  // slot groups owned per CTA
    static_assert(LOGS >= 1 && LOGS <= 4, "clusters of 2, 4, 8 or 16 CTAs");
    static_assert(LOGS == 1 ? G == 2 * T : (G % 4 == 0 && G <= T),
                  "a thread's four local slots belong to one group owner");
};

// Group levels of the forward transform on the S positions of group g (global
// group index), y[c] = position g S + c; level LOGL + k pairs (c, c + S/2^(k+1))
// with twiddle tw[2^(LOGL+k) + (g << k) + (c >> (LOGS - k))].
template <int LOGN, int LOGS, bool LAZY>
__device__ __forceinline__ void cluster_group_fwd(uint64_t (&y)[1 << LOGS], uint32_t g, const uint64_t* __restrict__ tw) {
    using CS = ClusterShape<LOGN, LOGS>;
#pragma unroll
    for (int k = 0; k < LOGS; ++k) {
        const int half = CS::S >> (k + 1);
#pragma unroll
        for (int c = 0; c < CS::S; ++c) {
            if (c & half) continue;
            const uint64_t w = __ldg(tw + (1u << (CS::LOGL + k)) + (g << k) + (uint32_t)(c >> (LOGS - k)));
            const uint64_t u = y[c];
            const uint64_t v = gl_mul(y[c + half], w);
            y[c] = LAZY ? gl_add_lazy(u, v) : gl_add(u, v);
            y[c + half] = gl_sub(u, v);
        }
    }
}

// Group levels of the backward transform (levels LOGN-1 down to LOGL).
template <int LOGN, int LOGS>
__device__ __forceinline__ void cluster_group_inv(uint64_t (&y)[1 << LOGS], uint32_t g, const uint64_t* __restrict__ tw) {
    using CS = ClusterShape<LOGN, LOGS>;
#pragma unroll
    for (int k = LOGS - 1; k >= 0; --k) {
        const int half = CS::S >> (k + 1);
#pragma unroll
        for (int c = 0; c < CS::S; ++c) {
            if (c & half) continue;
            const uint64_t w = __ldg(tw + (1u << (CS::LOGL + k)) + (g << k) + (uint32_t)(c >> (LOGS - k)));
            const uint64_t u = y[c];
            const uint64_t v = y[c + half];
            y[c] = gl_add(u, v);
            y[c + half] = gl_mul(gl_sub(u, v), w);
        }
    }
}

// Second half of the forward transform. In: x = this thread's four local slots
// 4t + j of the subsequence's NL-point transform (block engine slot layout). Out:
// x = the four global slots r NL + 4t + j. `recv` is this CTA's receive area for
// this exchange (NL words), `buf` a free exchange buffer of NL words (S > 4 only),
// tw the N-point forward table.
template <int LOGN, int LOGS, bool LAZY>
__device__ __forceinline__ void cluster_fwd_tail(uint64_t (&x)[4], int t, int r, uint64_t* recv, uint64_t* buf,
                                                 const uint64_t* __restrict__ tw) {
    using CS = ClusterShape<LOGN, LOGS>;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    // local slot i' = 4t + j is position i' S + r of group i', owned by CTA i' / G,
    // stored there at [r G + i' mod G] (four consecutive words)
    const int owner = (4 * t) / CS::G;
    uint64_t* dst = cluster.map_shared_rank(recv, owner) + r * CS::G + ((4 * t) % CS::G);
    reinterpret_cast<ulonglong2*>(dst)[0] = make_ulonglong2(x[0], x[1]);
    reinterpret_cast<ulonglong2*>(dst)[1] = make_ulonglong2(x[2], x[3]);
    cluster.sync();
    if constexpr (CS::S == 2) {
        // G = 2T: thread t owns groups g = r G + 2t and g + 1, whose two positions each
        // are its four slots (one butterfly per group, twiddle tw[NL + g])
        const ulonglong2 p0 = *reinterpret_cast<const ulonglong2*>(recv + 2 * t);          // position 0
        const ulonglong2 p1 = *reinterpret_cast<const ulonglong2*>(recv + CS::G + 2 * t);  // position 1
        const uint32_t g = (uint32_t)(r * CS::G + 2 * t);
        const uint64_t v0 = gl_mul(p1.x, __ldg(tw + CS::NL + g));
        const uint64_t v1 = gl_mul(p1.y, __ldg(tw + CS::NL + g + 1));
        x[0] = LAZY ? gl_add_lazy(p0.x, v0) : gl_add(p0.x, v0);
        x[1] = gl_sub(p0.x, v0);
        x[2] = LAZY ? gl_add_lazy(p0.y, v1) : gl_add(p0.y, v1);
        x[3] = gl_sub(p0.y, v1);
    } else if constexpr (CS::S == 4) {
        // G = T: thread t owns group r G + t, whose slots are its own four
#pragma unroll
        for (int c = 0; c < 4; ++c) x[c] = recv[c * CS::G + t];
        cluster_group_fwd<LOGN, LOGS, LAZY>(reinterpret_cast<uint64_t(&)[4]>(x), (uint32_t)(r * CS::G + t), tw);
    } else {
        // threads t < G each take one group of S slots, then the slots are dealt out
        // four per thread through `buf` (block barrier: every group written first)
        if (t < CS::G) {
            uint64_t y[CS::S];
#pragma unroll
            for (int c = 0; c < CS::S; ++c) y[c] = recv[c * CS::G + t];
            cluster_group_fwd<LOGN, LOGS, LAZY>(y, (uint32_t)(r * CS::G + t), tw);
#pragma unroll
            for (int c = 0; c < CS::S; c += 2)
                *reinterpret_cast<ulonglong2*>(buf + t * CS::S + c) = make_ulonglong2(y[c], y[c + 1]);
        }
        __syncthreads();
        const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(buf + 4 * t);
        const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(buf + 4 * t + 2);
        x[0] = a.x;
        x[1] = a.y;
        x[2] = b.x;
        x[3] = b.y;
    }
}

// First half of the backward transform. In: x = global slots r NL + 4t + j. Out:
// x = this thread's four local slots 4t + j of the subsequence, ready for the
// block engine's NL-point backward transform. tw: the N-point backward table.
template <int LOGN, int LOGS>
__device__ __forceinline__ void cluster_inv_head(uint64_t (&x)[4], int t, int r, uint64_t* recv, uint64_t* buf,
                                                 const uint64_t* __restrict__ tw) {
    using CS = ClusterShape<LOGN, LOGS>;
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    if constexpr (CS::S == 2) {
        // groups g = r G + 2t (slots x0, x1) and g + 1 (x2, x3); position c of each goes
        // to CTA c as its local slot g, g + 1
        const uint32_t g = (uint32_t)(r * CS::G + 2 * t);
        const uint64_t a0 = gl_add(x[0], x[1]), b0 = gl_mul(gl_sub(x[0], x[1]), __ldg(tw + CS::NL + g));
        const uint64_t a1 = gl_add(x[2], x[3]), b1 = gl_mul(gl_sub(x[2], x[3]), __ldg(tw + CS::NL + g + 1));
        *reinterpret_cast<ulonglong2*>(cluster.map_shared_rank(recv, 0) + g) = make_ulonglong2(a0, a1);
        *reinterpret_cast<ulonglong2*>(cluster.map_shared_rank(recv, 1) + g) = make_ulonglong2(b0, b1);
    } else if constexpr (CS::S == 4) {
        const uint32_t g = (uint32_t)(r * CS::G + t);
        cluster_group_inv<LOGN, LOGS>(reinterpret_cast<uint64_t(&)[4]>(x), g, tw);
        // position g S + c goes to CTA c as its local slot g
#pragma unroll
        for (int c = 0; c < 4; ++c) cluster.map_shared_rank(recv, c)[g] = x[c];
    } else {
        *reinterpret_cast<ulonglong2*>(buf + 4 * t) = make_ulonglong2(x[0], x[1]);
        *reinterpret_cast<ulonglong2*>(buf + 4 * t + 2) = make_ulonglong2(x[2], x[3]);
        __syncthreads();
        if (t < CS::G) {
            const uint32_t g = (uint32_t)(r * CS::G + t);
            uint64_t y[CS::S];
#pragma unroll
            for (int c = 0; c < CS::S; c += 2) {
                const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(buf + t * CS::S + c);
                y[c] = v.x;
                y[c + 1] = v.y;
            }
            cluster_group_inv<LOGN, LOGS>(y, g, tw);
#pragma unroll
            for (int c = 0; c < CS::S; ++c) cluster.map_shared_rank(recv, c)[g] = y[c];
        }
    }
    cluster.sync();
    const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(recv + 4 * t);
    const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(recv + 4 * t + 2);
    x[0] = a.x;
    x[1] = a.y;
    x[2] = b.x;
    x[3] = b.y;
}

}  // namespace tp
