// Blind rotation with two or four thread blocks per ciphertext (a cluster of S
// CTAs on S SMs), for batches smaller than the number of SMs.
//
// The persistent kernel in br_kernels.cuh gives each ciphertext one block, so a
// batch of 1 or 37 leaves most SMs idle and each rotation takes n serial
// iterations on one SM.
//
// S = 2: CTA h (h = 0: the A half, 1: the B half) of a pair owns accumulator
// half h and its l gadget rows: per iteration it runs the backward NTT of its
// half, the l digit NTTs and the multiply-accumulate of those rows into all
// C = 2G key components, i.e. half of the iteration's work. The components of
// the other half are partial sums the peer needs: each CTA writes them into the
// peer's shared memory (distributed shared memory of the cluster), and after a
// cluster barrier adds the peer's partials for its own half before the
// monomial weights and the accumulator update. Two cluster barriers per
// iteration: one before writing into the peer's receive area (the peer has
// finished reading the previous iteration's) and one after (the writes are
// visible).
//
// S = 4: CTA rank r = 2q + h owns accumulator half h (both CTAs of a half keep
// the same copy and update it identically) and the gadget digits of subset q
// (q = 0: the first ceil(l/2), q = 1: the rest) of that half's rows. Per
// iteration it runs its half's backward NTT, its digits' NTTs and their
// multiply-accumulate into all C components. Step 1: the other half's
// components go to CTA r ^ 1 (area 1); after a barrier each CTA adds them to
// its own half's components, which now sum this digit subset's rows of both
// halves. Step 2: that sum goes to CTA r ^ 2 (area 2); after a second barrier
// each CTA adds the other subset's sum and has its half's full products. Two
// barriers suffice with two areas: area 1 is read between the two barriers of
// an iteration and written in the next iteration only after its second
// barrier; area 2 is read after the second barrier and written in the next
// iteration only after the next first barrier, which its reader reaches after
// reading.
//
// The residues are the single-block kernel's, so the output words are
// identical. All CTAs of a cluster run the same loop over the same ciphertexts
// and read the same LWE words (skipping the same a_i = 0 iterations), so they
// reach every barrier the same number of times.
#pragma once

#include <cooperative_groups.h>

#include "br_kernels.cuh"

namespace tp {

// Shared-memory plan of the S-block kernel, in words (LWE area budgeted at 1024
// words; the host adds the real size and checks the total). The key row stage
// is kept when it fits, then the twiddles.
// Exchange buffers of the NTTs: two (transforms alternate between them), or one
// where two do not fit beside the four-block kernel's receive areas (then every
// transform starts after a block barrier instead).
__host__ __device__ constexpr int br_split_xbufs(int logn, int variant, int s) {
    return ((size_t)(1 << logn) * (2 + 1 + (s == 4 ? 2 : 1) * br_rgsw_per_group(variant)) + 1024) * 8 <=
                   227u * 1024u
               ? 2
               : 1;
}
__host__ __device__ constexpr size_t br_pair_core_words(int logn, int variant, int s = 2) {
    // xbufs, acc half, receive area(s)
    return (size_t)(1 << logn) *
               (br_split_xbufs(logn, variant, s) + 1 + (s == 4 ? 2 : 1) * br_rgsw_per_group(variant)) +
           1024;
}
__host__ __device__ constexpr bool br_pair_key_prefetch(int logn, int variant, int s = 2) {
    return (br_pair_core_words(logn, variant, s) + (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant)) * 8 <=
           227u * 1024u;
}
__host__ __device__ constexpr bool br_pair_smem_twiddles(int logn, int variant, int loge, int s = 2) {
    return (br_pair_core_words(logn, variant, s) +
            (br_pair_key_prefetch(logn, variant, s) ? (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant) : 0) +
            2 * (size_t)br_twiddle_words(logn, loge)) * 8 <= 227u * 1024u;
}
__host__ __device__ constexpr size_t br_pair_smem_words(int logn, int variant, uint32_t n, int loge, int s = 2) {
    return (br_pair_smem_twiddles(logn, variant, loge, s) ? 2 * (size_t)br_twiddle_words(logn, loge) : 0) +
           br_pair_core_words(logn, variant, s) - 1024 +
           (br_pair_key_prefetch(logn, variant, s) ? (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant) : 0) +
           ((n + 2) & ~1u);
}
// The four-block kernel is built only where its core fits one SM's shared memory.
__host__ __device__ constexpr bool br_quad_fits(int logn, int variant) {
    return br_pair_core_words(logn, variant, 4) * 8 <= 227u * 1024u;
}

template <int LOGN, int VARIANT, int LOGE, int S>
__device__ __forceinline__ void br_split_body(const BrKernelParams& prm) {
    static_assert(S == 2 || S == 4, "two or four blocks per rotation");
    namespace cg = cooperative_groups;
    using SH = NttShape<LOGN, LOGE>;
    constexpr int N = SH::N;
    constexpr int T = SH::T;
    constexpr int E = SH::E;
    constexpr int G = br_rgsw_per_group(VARIANT);
    constexpr int C = 2 * G;
    constexpr uint32_t MASK2N = 2u * N - 1u;
    constexpr bool SIGNED = VARIANT != kCggiBinary;
    constexpr bool R4 = br_fused_radix4(LOGE, VARIANT, S);
    constexpr bool PF = br_pair_key_prefetch(LOGN, VARIANT, S);
    constexpr bool TW_SMEM = br_pair_smem_twiddles(LOGN, VARIANT, LOGE, S);

    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int h = rank & 1;   // accumulator half and gadget rows of this CTA
    const int q = rank >> 1;  // digit subset (S = 4)

    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* base = smem;
    const uint64_t* tw_f = prm.tw_fwd;
    const uint64_t* tw_i = prm.tw_inv;
    if constexpr (TW_SMEM) {
        constexpr int TWW = br_twiddle_words(LOGN, LOGE);
        for (int i = threadIdx.x; i < TWW; i += T) {
            base[i] = prm.tw_fwd[i];
            base[TWW + i] = prm.tw_inv[i];
        }
        tw_f = base;
        tw_i = base + TWW;
        base += 2 * TWW;
    }
    constexpr int XB = br_split_xbufs(LOGN, VARIANT, S);
    uint64_t* xbuf0 = base;
    uint64_t* xbuf1 = base + (XB - 1) * N;
    uint64_t* acc = base + XB * N;       // this CTA's half, [j*T + t], canonical, NTT domain
    uint64_t* recv = acc + N;            // area 1: partial sums for this half, [(g*E/2 + jp)*T + t] x 16 bytes
    uint64_t* recv2 = recv + G * N;      // area 2 (S = 4): the other digit subset's sums, same layout
    uint64_t* kst = recv + (S == 4 ? 2 : 1) * G * N;  // key row stage (C*N words)
    uint64_t* lwe_s = kst + (PF ? C * N : 0);
    uint64_t* peer_recv = cluster.map_shared_rank(recv, rank ^ 1);
    uint64_t* peer_recv2 = S == 4 ? cluster.map_shared_rank(recv2, rank ^ 2) : nullptr;

    const int t = threadIdx.x;
    const uint32_t n = prm.n;
    const uint32_t L = prm.digits;
    // this CTA's gadget digits of its half's rows: all (S = 2) or subset q (S = 4)
    const uint32_t d_begin = S == 4 && q ? (L + 1) / 2 : 0;
    const uint32_t d_end = S == 4 && !q ? (L + 1) / 2 : L;

    int sel = 0;
    // exchange buffer of the next transform; with one buffer, a block barrier first
    // (every warp has finished reading the previous transform's last exchange)
    auto xb = [&]() -> uint64_t* {
        if constexpr (XB == 1) __syncthreads();
        uint64_t* b = sel ? xbuf1 : xbuf0;
        sel ^= 1;
        return b;
    };

    const uint64_t clusters = gridDim.x / S;
    for (uint64_t b = blockIdx.x / S; b < prm.batch; b += clusters) {
        __syncthreads();  // previous ciphertext done with lwe_s / acc (and twiddles written)
        const uint64_t* lwe = prm.lwes + b * prm.lwe_stride;
        bool bad = false;
        for (uint32_t i = t; i <= n; i += T) {
            uint64_t v = lwe[i];
            bad |= v > MASK2N;
            lwe_s[i] = v & MASK2N;
        }
        if (bad && rank == 0) atomicOr(prm.err, 1u);
        __syncthreads();

        // Prologue on this half: acc_h = NTT(acc_in_h) * X^b
        {
            const uint64_t* ain = prm.accs + b * prm.acc_stride + (uint64_t)h * N;
            const uint32_t bb = (uint32_t)lwe_s[n];
            uint64_t x[1][E];
#pragma unroll
            for (int j = 0; j < E; ++j) x[0][j] = ain[t + j * T];
            ntt_forward_k<LOGN, 1, LOGE, R4, true>(x, t, xb(), tw_f);
#pragma unroll
            for (int j = 0; j < E; ++j)
                acc[j * T + t] = gl_mul(x[0][j], mono<LOGN>(prm.psi_pow, slot_exponent<LOGN>(E * t + j), bb));
        }

        const uint32_t step = VARIANT == kBmmpBinary ? 2 : 1;
#pragma unroll 1
        for (uint32_t i = 0; i < n; i += step) {
            uint32_t a0 = (uint32_t)lwe_s[i];
            uint32_t a1 = 0;
            if constexpr (VARIANT == kBmmpBinary) {
                a0 = (2u * N - a0) & MASK2N;
                a1 = (2u * N - (uint32_t)lwe_s[i + 1]) & MASK2N;
            } else {
                if (a0 == 0) continue;  // all CTAs read the same word: they skip together
            }
            const uint64_t* kit = prm.key + (uint64_t)(i / step) * (2ull * L * N * C);

            uint64_t o[C][E];
#pragma unroll
            for (int c = 0; c < C; ++c)
#pragma unroll
                for (int j = 0; j < E; ++j) o[c][j] = 0;

            // backward NTT of this half into corrected coefficients
            uint64_t cx[1][E];
#pragma unroll
            for (int j = 0; j < E; ++j) {
                cx[0][j] = acc[j * T + t];
                if constexpr (VARIANT == kCggiBinary)
                    cx[0][j] = gl_mul(cx[0][j],
                                      gl_sub(mono<LOGN>(prm.psi_pow, slot_exponent<LOGN>(E * t + j), 2u * N - a0), 1));
            }
#pragma unroll 1
            for (uint32_t d = d_begin; d < d_end; ++d) {
                const uint64_t* kr = kit + (uint64_t)(h * L + d) * (N * C);
                if constexpr (PF) {
#pragma unroll
                    for (int c = 0; c < C; ++c)
#pragma unroll
                        for (int jp = 0; jp < E / 2; ++jp) {
                            const int ko = ((c * (E / 2) + jp) * T + t) * 2;
                            cp_async16(kst + ko, kr + ko);
                        }
                    cp_async_commit();
                }
                if (d == d_begin) {
                    ntt_backward_unscaled_k<LOGN, 1, LOGE, R4>(cx, t, xb(), tw_i);
#pragma unroll
                    for (int j = 0; j < E; ++j) cx[0][j] = gl_add(gl_div_pow2<LOGN>(cx[0][j]), prm.corr);
                }
                uint64_t x[1][E];
                const uint32_t sh = prm.dshift[d];
                const uint64_t mk = prm.dmask[d];
                const uint64_t dl = prm.ddelta[d];
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    const uint64_t raw = (cx[0][j] >> sh) & mk;
                    x[0][j] = SIGNED ? gl_sub(raw, dl) : raw;
                }
                ntt_forward_k<LOGN, 1, LOGE, R4, true>(x, t, xb(), tw_f);
                if constexpr (PF) cp_async_wait_all();
#pragma unroll
                for (int c = 0; c < C; ++c)
#pragma unroll
                    for (int jp = 0; jp < E / 2; ++jp) {
                        const int ko = ((c * (E / 2) + jp) * T + t) * 2;
                        const ulonglong2 kv = PF ? *reinterpret_cast<const ulonglong2*>(kst + ko)
                                                 : __ldg(reinterpret_cast<const ulonglong2*>(kr + ko));
                        o[c][2 * jp] = gl_fma(o[c][2 * jp], x[0][2 * jp], kv.x);
                        o[c][2 * jp + 1] = gl_fma(o[c][2 * jp + 1], x[0][2 * jp + 1], kv.y);
                    }
            }

            // component 2g + h of this half / 2g + (h^1) of the peer's, selected without
            // indexing the register array by the (run-time) block rank
            auto mine = [&](int g, int j) -> uint64_t { return h ? o[2 * g + 1][j] : o[2 * g][j]; };
            auto theirs = [&](int g, int j) -> uint64_t { return h ? o[2 * g][j] : o[2 * g + 1][j]; };

            if constexpr (S == 2) {
                // hand the peer its half's partial sums
                cluster.sync();  // the peer has read the previous iteration's partials
#pragma unroll
                for (int g = 0; g < G; ++g)
#pragma unroll
                    for (int jp = 0; jp < E / 2; ++jp)
                        *reinterpret_cast<ulonglong2*>(peer_recv + ((g * (E / 2) + jp) * T + t) * 2) =
                            make_ulonglong2(theirs(g, 2 * jp), theirs(g, 2 * jp + 1));
                cluster.sync();  // the peer's partials for this half are in recv
            } else {
                // step 1: the other half's components to the CTA of that half with the same digits
#pragma unroll
                for (int g = 0; g < G; ++g)
#pragma unroll
                    for (int jp = 0; jp < E / 2; ++jp)
                        *reinterpret_cast<ulonglong2*>(peer_recv + ((g * (E / 2) + jp) * T + t) * 2) =
                            make_ulonglong2(theirs(g, 2 * jp), theirs(g, 2 * jp + 1));
                cluster.sync();  // area 1 holds the other half's products of this digit subset
            }
            // S = 4: this half's components summed over this CTA's digit subset of both halves' rows,
            // handed to the CTA of this half with the other digit subset
            uint64_t sm[S == 4 ? G : 1][E];
            if constexpr (S == 4) {
#pragma unroll
                for (int g = 0; g < G; ++g)
#pragma unroll
                    for (int jp = 0; jp < E / 2; ++jp) {
                        const ulonglong2 v =
                            *reinterpret_cast<const ulonglong2*>(recv + ((g * (E / 2) + jp) * T + t) * 2);
                        sm[g][2 * jp] = gl_add(mine(g, 2 * jp), v.x);
                        sm[g][2 * jp + 1] = gl_add(mine(g, 2 * jp + 1), v.y);
                        *reinterpret_cast<ulonglong2*>(peer_recv2 + ((g * (E / 2) + jp) * T + t) * 2) =
                            make_ulonglong2(sm[g][2 * jp], sm[g][2 * jp + 1]);
                    }
            }
            // this CTA's share of this half's products: its own rows (S = 2) or its subset's sum (S = 4)
            auto own = [&](int g, int j) -> uint64_t {
                if constexpr (S == 4) return sm[g][j];
                else return mine(g, j);
            };
            if constexpr (S == 4) cluster.sync();  // area 2 holds the other subset's sums
            uint64_t* const rv = S == 4 ? recv2 : recv;

            // accumulator update of this half (the single-block kernel's weights)
#pragma unroll
            for (int jp = 0; jp < E / 2; ++jp) {
                uint64_t pr[G][2];
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(rv + ((g * (E / 2) + jp) * T + t) * 2);
                    pr[g][0] = v.x;
                    pr[g][1] = v.y;
                }
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int j = 2 * jp + e;
                    const uint32_t ek = slot_exponent<LOGN>(E * t + j);
                    uint64_t u = acc[j * T + t];
                    if constexpr (VARIANT == kCggiBinary) {
                        u = gl_add(gl_add(u, own(0, j)), pr[0][e]);
                    } else if constexpr (VARIANT == kCggiTernary) {
                        const uint64_t mp = gl_sub(mono<LOGN>(prm.psi_pow, ek, 2u * N - a0), 1);
                        const uint64_t mn = gl_sub(mono<LOGN>(prm.psi_pow, ek, a0), 1);
                        u = gl_fma(gl_fma(u, own(0, j), mp), pr[0][e], mp);
                        u = gl_fma(gl_fma(u, own(1, j), mn), pr[1][e], mn);
                    } else {
                        const uint64_t m0 = mono<LOGN>(prm.psi_pow, ek, a0);
                        const uint64_t m1 = mono<LOGN>(prm.psi_pow, ek, a1);
                        const uint64_t m2 = mono<LOGN>(prm.psi_pow, ek, (a0 + a1) & MASK2N);
                        const uint64_t w0 = gl_sub(m0, 1);
                        const uint64_t w1 = gl_sub(m1, 1);
                        const uint64_t w2 = gl_add(gl_sub(gl_sub(m2, m0), m1), 1);
                        u = gl_fma(gl_fma(u, own(0, j), w0), pr[0][e], w0);
                        u = gl_fma(gl_fma(u, own(1, j), w1), pr[1][e], w1);
                        u = gl_fma(gl_fma(u, own(2, j), w2), pr[2][e], w2);
                    }
                    acc[j * T + t] = u;
                }
            }
        }

        // Epilogue: this half of the result (S = 4: written by the first digit subset's CTAs)
        if (S == 4 && q) continue;
        uint64_t* res = prm.out + b * (2ull * N) + (uint64_t)h * N;
        uint64_t x[1][E];
#pragma unroll
        for (int j = 0; j < E; ++j) x[0][j] = acc[j * T + t];
        if (prm.out_coef) {
            ntt_backward_unscaled_k<LOGN, 1, LOGE, R4>(x, t, xb(), tw_i);
#pragma unroll
            for (int j = 0; j < E; ++j) res[t + j * T] = gl_div_pow2<LOGN>(x[0][j]);
        } else {
#pragma unroll
            for (int c = 0; c < E / 2; ++c)
                *reinterpret_cast<ulonglong2*>(res + E * t + 2 * c) = make_ulonglong2(x[0][2 * c], x[0][2 * c + 1]);
        }
    }
    cluster.sync();  // no CTA leaves while a peer may still address its shared memory
}

template <int LOGN, int VARIANT, int LOGE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__((1 << LOGN) >> LOGE, br_min_blocks(LOGN, VARIANT, LOGE))
br_pair_kernel(const BrKernelParams prm) {
    br_split_body<LOGN, VARIANT, LOGE, 2>(prm);
}

template <int LOGN, int VARIANT, int LOGE>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__((1 << LOGN) >> LOGE, br_min_blocks(LOGN, VARIANT, LOGE))
br_quad_kernel(const BrKernelParams prm) {
    br_split_body<LOGN, VARIANT, LOGE, 4>(prm);
}

// Entry point of the S-block kernel for (N, variant), 4 coefficients per thread;
// nullptr for S = 4 where its shared-memory core does not fit.
template <int LOGN, int VARIANT>
const void* br_split_kernel_entry(int split) {
    if (split == 4) {
        if constexpr (br_quad_fits(LOGN, VARIANT)) return (const void*)br_quad_kernel<LOGN, VARIANT, 2>;
        else return nullptr;
    }
    return (const void*)br_pair_kernel<LOGN, VARIANT, 2>;
}

template <int LOGN>
const void* br_split_kernel_ptr(int variant, int split) {
    switch (variant) {
        case kCggiBinary: return br_split_kernel_entry<LOGN, kCggiBinary>(split);
        case kCggiTernary: return br_split_kernel_entry<LOGN, kCggiTernary>(split);
        default: return br_split_kernel_entry<LOGN, kBmmpBinary>(split);
    }
}

}  // namespace tp
