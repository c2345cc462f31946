// Key switching on the GPU: RLWE -> RLWE key switch, automorphism evaluation,
// the merge/trace steps of n-LWE -> RLWE packing, and LWE -> LWE key switch.
//
// The RLWE kernels share one core with the blind rotation: a block of
// T = N/E threads (E = 2^LOGE = 4 or 8 coefficients per thread) takes the
// coefficient-domain A part of one ciphertext, forms its signed gadget digits
// (lib/include/static/gadget_decomp.h:156-205), runs a forward NTT per digit and
// multiply-accumulates against the key rows (lib/src/operators/rlwe_conversion.cpp:
// 224-249). Key rows are laid out like the blind-rotation key of the same tile
// (C = 2 components, A and B, per slot).
#pragma once

#include <cooperative_groups.h>

#include "cluster_ntt.cuh"
#include "gl_arith.cuh"
#include "ntt_block.cuh"

namespace tp {

enum KsMode : int {
    kKsRlwe = 0,   // out -= KS(in.A coef); out.B += in.B (NTT)
    kKsAuto = 1,   // out -= KS(aut_t(in.A)); out.B += NTT(aut_t(in.B)); in coefficient domain
    kKsMerge = 2,  // packing merge: left <- (right + X^s left) + INTT(AutoKS(right - X^s left))
    kKsTrace = 3,  // trace step:    x <- x + INTT(AutoKS(x))
    kKsSplit = 4   // SAP truncation tree node: y = INTT(AutoKS(x)); x <- x + y; out1 <- X^-s (x - y)
};
constexpr int kKsModes = 5;
constexpr uint32_t kNoNode = 0xFFFFFFFFu;

struct KsKernelParams {
    const uint64_t* key;      // device layout: [digit][c][jp][t][2], C = 2, jp < E/2
    const uint64_t* tw_fwd;
    const uint64_t* tw_inv;
    const uint64_t* in;       // per item: 2N words (kKsRlwe/kKsAuto), node pairs (kKsMerge), node (kKsTrace)
    uint64_t* out;
    uint64_t items;           // ciphertexts (or merges)
    uint64_t in_stride;       // words between items' inputs
    uint64_t out_stride;      // words between items' outputs
    uint64_t right_offset;    // kKsMerge: words from left node to right node; kKsSplit: to the second child
    uint32_t digits;
    uint32_t auto_index;      // t (odd)
    uint32_t auto_index_inv;  // t^-1 mod 2N
    uint32_t shift;           // kKsMerge: X^shift rotation of the left node; kKsSplit: X^-shift of the difference
    uint64_t n_inv;
    // kKsMerge over a compacted tree (PackConsecutively): item it of pack p = it / pair_count
    // merges nodes pairs[2q] (left) and pairs[2q+1] (right) of the pack's previous level,
    // q = it % pair_count, each node at in + (p * prev_count + slot) * in_stride; a slot of
    // kNoNode stands for an empty subtree, read as `zero` (2N zero words)
    const uint32_t* pairs;
    const uint64_t* zero;
    uint32_t pair_count;
    uint32_t prev_count;
    uint64_t corr;
    uint32_t dshift[8];
    uint64_t dmask[8];
    uint64_t ddelta[8];
};

// Shared memory of a key-switching block, in words: twiddles (2N) + two exchange buffers (2N);
// on a cluster of S CTAs (N > 4096) the same of the local size N/S plus two receive areas.
__host__ __device__ constexpr size_t ks_smem_words(int N, int S = 1) { return (S > 1 ? 6 : 4) * (size_t)(N / S); }

// Coefficient m of aut_t(x) for x in the coefficient domain: x_i moves to
// i*t mod 2N with a sign flip past N (automorphism_evaluation.cpp:183-206), so
// m comes from i = m * t^-1 mod 2N.
template <int LOGN>
__device__ __forceinline__ uint64_t aut_coeff(const uint64_t* x, uint32_t m, uint32_t tinv) {
    constexpr uint32_t N = 1u << LOGN;
    const uint32_t i = (m * tinv) & (2 * N - 1);
    const uint64_t v = x[i & (N - 1)];
    return i >= N ? gl_neg(v) : v;
}

// Coefficient m of X^s * x (negacyclic shift; lwe_to_rlwe_packing.cpp:192-196).
template <int LOGN>
__device__ __forceinline__ uint64_t rot_coeff(const uint64_t* x, uint32_t m, uint32_t s) {
    constexpr uint32_t N = 1u << LOGN;
    return m >= s ? x[m - s] : gl_neg(x[N + m - s]);
}

// sum_d NTT(digit_d(a)) * key_d for both components (canonical), a in the
// coefficient layout and canonical. On a cluster (LOGS > 0, rank cr) a holds the
// CTA's subsequence, o its slot block, and the key row part cr (2 NL words) is read.
template <int LOGN, int LOGE, int LOGS = 0>
__device__ __forceinline__ void ks_mac(uint64_t (&a)[1 << LOGE], const KsKernelParams& prm, int t, uint64_t* buf0,
                                       uint64_t* buf1, int& sel, const uint64_t* tw_f, uint64_t (&o)[2][1 << LOGE],
                                       int cr = 0, uint64_t* recv0 = nullptr, uint64_t* recv1 = nullptr,
                                       int* rsel = nullptr) {
    constexpr int N = 1 << LOGN;
    constexpr int LOGL = LOGN - LOGS;
    constexpr int NL = 1 << LOGL;
    constexpr int E = 1 << LOGE;
    constexpr int T = NL / E;
#pragma unroll
    for (int j = 0; j < E; ++j) {
        a[j] = gl_add(a[j], prm.corr);
        o[0][j] = 0;
        o[1][j] = 0;
    }
#pragma unroll 1
    for (uint32_t d = 0; d < prm.digits; ++d) {
        const uint32_t sh = prm.dshift[d];
        const uint64_t mk = prm.dmask[d];
        const uint64_t dl = prm.ddelta[d];
        uint64_t x[1][E];
#pragma unroll
        for (int j = 0; j < E; ++j) x[0][j] = gl_sub((a[j] >> sh) & mk, dl);
        const uint64_t* kr = prm.key + (uint64_t)d * (2 * N) + (uint64_t)cr * (2 * NL);
        // with 4 coefficients per thread the digit's key words (8 registers) are
        // requested before its NTT, which hides their L2 latency; with 8 they
        // would not fit next to the NTT's registers and are read after it
        ulonglong2 kv[2][E / 2];
        if constexpr (LOGE == 2) {
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int jp = 0; jp < E / 2; ++jp)
                    kv[c][jp] = __ldg(reinterpret_cast<const ulonglong2*>(kr + ((c * (E / 2) + jp) * T + t) * 2));
        }
        ntt_forward_k<LOGL, 1, LOGE, false, true>(x, t, sel ? buf1 : buf0, tw_f);
        sel ^= 1;
        if constexpr (LOGS > 0) {
            uint64_t* rv = *rsel ? recv1 : recv0;
            *rsel ^= 1;
            uint64_t* fb = sel ? buf1 : buf0;
            if constexpr ((1 << LOGS) > 4) sel ^= 1;
            cluster_fwd_tail<LOGN, LOGS, true>(reinterpret_cast<uint64_t(&)[4]>(x[0]), t, cr, rv, fb, prm.tw_fwd);
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
            for (int jp = 0; jp < E / 2; ++jp) {
                if constexpr (LOGE != 2)
                    kv[c][jp] = __ldg(reinterpret_cast<const ulonglong2*>(kr + ((c * (E / 2) + jp) * T + t) * 2));
                o[c][2 * jp] = gl_fma(o[c][2 * jp], x[0][2 * jp], kv[c][jp].x);
                o[c][2 * jp + 1] = gl_fma(o[c][2 * jp + 1], x[0][2 * jp + 1], kv[c][jp].y);
            }
        }
    }
}

// Blocks per SM the kernel is compiled for: two where two blocks of N/E threads
// still leave 128 registers per thread (N/E <= 256), else one.
template <int LOGN, int LOGE>
constexpr int ks_min_blocks() { return ((1 << LOGN) >> LOGE) <= 256 ? 2 : 1; }

// LOGS > 0 (N > 4096): one item per cluster of 2^LOGS CTAs, launched with that
// cluster size (cluster_ntt.cuh): CTA r holds the coefficients m = m' 2^LOGS + r and
// the slots r NL .. r NL + NL - 1; inputs are read from global memory at their
// global indices, so the automorphisms' gathers need no exchange.
template <int LOGN, int MODE, int LOGE, int LOGS = 0>
__global__ void __launch_bounds__((1 << (LOGN - LOGS)) >> LOGE, ks_min_blocks<LOGN - LOGS, LOGE>())
ks_kernel(const KsKernelParams prm) {
    constexpr int N = 1 << LOGN;
    constexpr int LOGL = LOGN - LOGS;
    constexpr int NL = 1 << LOGL;
    constexpr int E = 1 << LOGE;
    constexpr int T = NL / E;
    static_assert(LOGS == 0 || LOGE == 2, "clusters run with 4 coefficients per thread");
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* tw_f = smem;          // the first NL words of the N-point tables (the NL-point tables)
    uint64_t* tw_i = smem + NL;
    uint64_t* buf0 = smem + 2 * NL;
    uint64_t* buf1 = smem + 3 * NL;
    uint64_t* recv0 = smem + 4 * NL;  // cluster exchange areas
    uint64_t* recv1 = smem + 5 * NL;
    const int t = threadIdx.x;
    int cr = 0;
    if constexpr (LOGS > 0) {
        cr = (int)cooperative_groups::this_cluster().block_rank();
        cooperative_groups::this_cluster().sync();  // every CTA of the cluster running before remote stores
    }
    const uint32_t sbase = (uint32_t)cr << LOGL;
    // global index of this thread's local coefficient t + j T
    auto gm = [&](int j) -> uint32_t { return ((uint32_t)(t + j * T) << LOGS) + (uint32_t)cr; };
    int rsel = 0;
    for (int i = t; i < NL; i += T) {
        tw_f[i] = prm.tw_fwd[i];
        tw_i[i] = prm.tw_inv[i];
    }
    int sel = 0;
    // kKsRlwe: this block's next ciphertext's A half, requested while the
    // current one is switched (items are the block's own: no other block
    // writes them, so the early read is safe in place too). Measured +4-5% at
    // N = 1024 / 2048 with 4 coefficients per thread; at 1024 threads per block
    // (64 registers) it cost 6%, and with 8 per thread it would spill.
    constexpr bool PF = MODE == kKsRlwe && LOGE == 2 && T <= 512 && LOGS == 0;
    uint64_t a_next[E];
    if constexpr (PF) {
        if (blockIdx.x < prm.items) {
#pragma unroll
            for (int j = 0; j < E; ++j) a_next[j] = prm.in[blockIdx.x * prm.in_stride + t + j * T];
        }
    }
    for (uint64_t it = blockIdx.x >> LOGS; it < prm.items; it += gridDim.x >> LOGS) {
        __syncthreads();
        const uint64_t* in = prm.in + it * prm.in_stride;
        uint64_t* out = prm.out + it * prm.out_stride;
        uint64_t a[E], bb[E], base[2][E];
        // ---- gather inputs (every global read precedes the first barrier below,
        //      so kKsMerge/kKsTrace may write their result in place) ----
        if constexpr (PF) {
            const uint64_t nx = it + gridDim.x;
#pragma unroll
            for (int j = 0; j < E; ++j) a[j] = a_next[j];
            if (nx < prm.items) {
#pragma unroll
                for (int j = 0; j < E; ++j) a_next[j] = prm.in[nx * prm.in_stride + t + j * T];
            }
        } else if constexpr (MODE == kKsRlwe) {
#pragma unroll
            for (int j = 0; j < E; ++j) a[j] = in[gm(j)];
        } else if constexpr (MODE == kKsAuto) {
#pragma unroll
            for (int j = 0; j < E; ++j) {
                a[j] = aut_coeff<LOGN>(in, gm(j), prm.auto_index_inv);
                bb[j] = aut_coeff<LOGN>(in + N, gm(j), prm.auto_index_inv);
            }
        } else {
            const uint64_t* left = in;
            const uint64_t* right = in + (MODE == kKsMerge ? prm.right_offset : 0);
            if constexpr (MODE == kKsMerge) {
                if (prm.pairs) {
                    const uint64_t pk = it / prm.pair_count, q = it % prm.pair_count;
                    const uint32_t ls = prm.pairs[2 * q], rs = prm.pairs[2 * q + 1];
                    const uint64_t* base = prm.in + pk * prm.prev_count * prm.in_stride;
                    left = ls == kNoNode ? prm.zero : base + ls * prm.in_stride;
                    right = rs == kNoNode ? prm.zero : base + rs * prm.in_stride;
                }
            }
            const uint32_t s = prm.shift;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const uint32_t m = gm(j);
                    // diff = right - X^s left at the automorphism's source index
                    const uint32_t i = (m * prm.auto_index_inv) & (2 * N - 1);
                    const uint32_t src = i & (N - 1);
                    uint64_t dv = right[h * N + src];
                    uint64_t sv = right[h * N + m];
                    if constexpr (MODE == kKsMerge) {
                        dv = gl_sub(dv, rot_coeff<LOGN>(left + h * N, src, s));
                        sv = gl_add(sv, rot_coeff<LOGN>(left + h * N, m, s));
                    }
                    if (i >= N) dv = gl_neg(dv);
                    if (h == 0) a[j] = dv;
                    else bb[j] = dv;
                    base[h][j] = sv;
                }
            }
        }
        // ---- key switch of the A part ----
        uint64_t o[2][E];
        ks_mac<LOGN, LOGE, LOGS>(a, prm, t, buf0, buf1, sel, tw_f, o, cr, recv0, recv1, &rsel);
        if constexpr (MODE == kKsRlwe) {
            // out -= KS; out.B += in.B (rlwe_conversion.cpp:243-248); slots E t .. E t + E - 1
#pragma unroll
            for (int j = 0; j < E; ++j) {
                const uint32_t k = sbase + E * t + j;
                out[k] = gl_sub(out[k], o[0][j]);
                out[N + k] = gl_add(gl_sub(out[N + k], o[1][j]), in[N + k]);
            }
        } else {
            // NTT of the automorphism's B part (automorphism_evaluation.cpp:156)
            ntt_forward_k<LOGL, 1, LOGE>(reinterpret_cast<uint64_t(&)[1][E]>(bb), t, sel ? buf1 : buf0, tw_f);
            sel ^= 1;
            if constexpr (LOGS > 0) {
                uint64_t* rv = rsel ? recv1 : recv0;
                rsel ^= 1;
                uint64_t* fb = sel ? buf1 : buf0;
                if constexpr ((1 << LOGS) > 4) sel ^= 1;
                cluster_fwd_tail<LOGN, LOGS, false>(reinterpret_cast<uint64_t(&)[4]>(bb), t, cr, rv, fb, prm.tw_fwd);
            }
            if constexpr (MODE == kKsAuto) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const uint32_t k = sbase + E * t + j;
                    out[k] = gl_sub(out[k], o[0][j]);
                    out[N + k] = gl_add(gl_sub(out[N + k], o[1][j]), bb[j]);
                }
            } else {
                // Auto eval output (NTT) -> coefficients, added to the sum half
                // (lwe_to_rlwe_packing.cpp:205-210, 228-233)
                uint64_t r[1][E];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int j = 0; j < E; ++j) r[0][j] = h == 0 ? gl_neg(o[0][j])
                                                                 : gl_sub(bb[j], o[1][j]);
                    if constexpr (LOGS > 0) {
                        uint64_t* rv = rsel ? recv1 : recv0;
                        rsel ^= 1;
                        uint64_t* fb = sel ? buf1 : buf0;
                        if constexpr ((1 << LOGS) > 4) sel ^= 1;
                        cluster_inv_head<LOGN, LOGS>(reinterpret_cast<uint64_t(&)[4]>(r[0]), t, cr, rv, fb,
                                                     prm.tw_inv);
                    }
                    ntt_backward_unscaled_k<LOGL, 1, LOGE>(r, t, sel ? buf1 : buf0, tw_i);
                    sel ^= 1;
                    if constexpr (MODE == kKsSplit) {
                        // children of a truncation-tree node (sap_decomposer.cpp:266-284, in the
                        // coefficient domain): x + y in place, X^-s (x - y) at right_offset
                        uint64_t* out1 = out + prm.right_offset + h * N;
                        const uint32_t s = prm.shift;
#pragma unroll
                        for (int j = 0; j < E; ++j) {
                            const uint32_t m = gm(j);
                            const uint64_t y = gl_div_pow2<LOGN>(r[0][j]);
                            out[h * N + m] = gl_add(base[h][j], y);
                            const uint64_t z = gl_sub(base[h][j], y);
                            if (m >= s) out1[m - s] = z;
                            else out1[m + N - s] = gl_neg(z);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < E; ++j)
                            out[h * N + gm(j)] = gl_add(base[h][j], gl_div_pow2<LOGN>(r[0][j]));
                    }
                }
            }
        }
    }
}

}  // namespace tp
