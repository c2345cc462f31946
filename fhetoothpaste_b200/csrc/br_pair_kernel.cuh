// Blind rotation with two thread blocks per ciphertext (a cluster of two CTAs on
// two SMs), for batches smaller than the number of SMs.
//
// The persistent kernel in br_kernels.cuh gives each ciphertext one block, so a
// batch of 1 or 37 leaves most SMs idle and each rotation takes n serial
// iterations on one SM. Here CTA h (h = 0: the A half, 1: the B half) of a pair
// owns accumulator half h and its l gadget rows: per iteration it runs the
// backward NTT of its half, the l digit NTTs and the multiply-accumulate of
// those rows into all C = 2G key components, i.e. half of the iteration's work.
// The components of the other half are partial sums the peer needs: each CTA
// writes them into the peer's shared memory (distributed shared memory of the
// cluster), and after a cluster barrier adds the peer's partials for its own
// half before the monomial weights and the accumulator update. The residues
// are the single-block kernel's, so the output words are identical.
//
// Per iteration two cluster barriers: one before writing into the peer's
// receive area (the peer has finished reading the previous iteration's) and one
// after (the writes are visible). Both CTAs of a pair run the same loop over the
// same ciphertexts, so they reach every barrier the same number of times.
#pragma once

#include <cooperative_groups.h>

#include "br_kernels.cuh"

namespace tp {

// Shared-memory plan of the pair kernel, in words (LWE area budgeted at 1024
// words; the host adds the real size and checks the total). The key row stage
// is kept when it fits, then the twiddles.
__host__ __device__ constexpr size_t br_pair_core_words(int logn, int variant) {
    return (size_t)(1 << logn) * (2 + 1 + br_rgsw_per_group(variant)) + 1024;  // xbufs, acc half, receive area
}
__host__ __device__ constexpr bool br_pair_key_prefetch(int logn, int variant) {
    return (br_pair_core_words(logn, variant) + (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant)) * 8 <=
           227u * 1024u;
}
__host__ __device__ constexpr bool br_pair_smem_twiddles(int logn, int variant, int loge) {
    return (br_pair_core_words(logn, variant) +
            (br_pair_key_prefetch(logn, variant) ? (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant) : 0) +
            2 * (size_t)br_twiddle_words(logn, loge)) * 8 <= 227u * 1024u;
}
__host__ __device__ constexpr size_t br_pair_smem_words(int logn, int variant, uint32_t n, int loge) {
    return (br_pair_smem_twiddles(logn, variant, loge) ? 2 * (size_t)br_twiddle_words(logn, loge) : 0) +
           (size_t)(1 << logn) * (2 + 1 + br_rgsw_per_group(variant)) +
           (br_pair_key_prefetch(logn, variant) ? (size_t)(1 << logn) * 2 * br_rgsw_per_group(variant) : 0) +
           ((n + 2) & ~1u);
}

template <int LOGN, int VARIANT, int LOGE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__((1 << LOGN) >> LOGE, br_min_blocks(LOGN, VARIANT, LOGE))
br_pair_kernel(const BrKernelParams prm) {
    namespace cg = cooperative_groups;
    using SH = NttShape<LOGN, LOGE>;
    constexpr int N = SH::N;
    constexpr int T = SH::T;
    constexpr int E = SH::E;
    constexpr int G = br_rgsw_per_group(VARIANT);
    constexpr int C = 2 * G;
    constexpr uint32_t MASK2N = 2u * N - 1u;
    constexpr bool SIGNED = VARIANT != kCggiBinary;
    constexpr bool R4 = br_fused_radix4(LOGE, VARIANT);
    constexpr bool PF = br_pair_key_prefetch(LOGN, VARIANT);
    constexpr bool TW_SMEM = br_pair_smem_twiddles(LOGN, VARIANT, LOGE);

    cg::cluster_group cluster = cg::this_cluster();
    const int h = (int)cluster.block_rank();  // accumulator half and gadget rows of this CTA

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
    uint64_t* xbuf0 = base;
    uint64_t* xbuf1 = base + N;
    uint64_t* acc = base + 2 * N;        // this CTA's half, [j*T + t], canonical, NTT domain
    uint64_t* recv = acc + N;            // peer's partial sums for this half, [(g*E/2 + jp)*T + t] x 16 bytes
    uint64_t* kst = recv + G * N;        // key row stage (C*N words)
    uint64_t* lwe_s = kst + (PF ? C * N : 0);
    uint64_t* peer_recv = cluster.map_shared_rank(recv, h ^ 1);

    const int t = threadIdx.x;
    const uint32_t n = prm.n;
    const uint32_t L = prm.digits;

    int sel = 0;
    auto xb = [&]() -> uint64_t* {
        uint64_t* b = sel ? xbuf1 : xbuf0;
        sel ^= 1;
        return b;
    };

    const uint64_t pairs = gridDim.x / 2;
    for (uint64_t b = blockIdx.x / 2; b < prm.batch; b += pairs) {
        __syncthreads();  // previous ciphertext done with lwe_s / acc (and twiddles written)
        const uint64_t* lwe = prm.lwes + b * prm.lwe_stride;
        bool bad = false;
        for (uint32_t i = t; i <= n; i += T) {
            uint64_t v = lwe[i];
            bad |= v > MASK2N;
            lwe_s[i] = v & MASK2N;
        }
        if (bad && h == 0) atomicOr(prm.err, 1u);
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
                if (a0 == 0) continue;  // both CTAs read the same word: they skip together
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
            for (uint32_t d = 0; d < L; ++d) {
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
                if (d == 0) {
                    ntt_backward_unscaled_k<LOGN, 1, LOGE, R4>(cx, t, xb(), tw_i);
#pragma unroll
                    for (int j = 0; j < E; ++j) cx[0][j] = gl_fma(prm.corr, cx[0][j], prm.n_inv);
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

            // hand the peer its half's partial sums
            cluster.sync();  // the peer has read the previous iteration's partials
#pragma unroll
            for (int g = 0; g < G; ++g)
#pragma unroll
                for (int jp = 0; jp < E / 2; ++jp)
                    *reinterpret_cast<ulonglong2*>(peer_recv + ((g * (E / 2) + jp) * T + t) * 2) =
                        make_ulonglong2(theirs(g, 2 * jp), theirs(g, 2 * jp + 1));
            cluster.sync();  // the peer's partials for this half are in recv

            // accumulator update of this half (the single-block kernel's weights)
#pragma unroll
            for (int jp = 0; jp < E / 2; ++jp) {
                uint64_t pr[G][2];
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(recv + ((g * (E / 2) + jp) * T + t) * 2);
                    pr[g][0] = v.x;
                    pr[g][1] = v.y;
                }
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int j = 2 * jp + e;
                    const uint32_t ek = slot_exponent<LOGN>(E * t + j);
                    uint64_t u = acc[j * T + t];
                    if constexpr (VARIANT == kCggiBinary) {
                        u = gl_add(gl_add(u, mine(0, j)), pr[0][e]);
                    } else if constexpr (VARIANT == kCggiTernary) {
                        const uint64_t mp = gl_sub(mono<LOGN>(prm.psi_pow, ek, 2u * N - a0), 1);
                        const uint64_t mn = gl_sub(mono<LOGN>(prm.psi_pow, ek, a0), 1);
                        u = gl_fma(gl_fma(u, mine(0, j), mp), pr[0][e], mp);
                        u = gl_fma(gl_fma(u, mine(1, j), mn), pr[1][e], mn);
                    } else {
                        const uint64_t m0 = mono<LOGN>(prm.psi_pow, ek, a0);
                        const uint64_t m1 = mono<LOGN>(prm.psi_pow, ek, a1);
                        const uint64_t m2 = mono<LOGN>(prm.psi_pow, ek, (a0 + a1) & MASK2N);
                        const uint64_t w0 = gl_sub(m0, 1);
                        const uint64_t w1 = gl_sub(m1, 1);
                        const uint64_t w2 = gl_add(gl_sub(gl_sub(m2, m0), m1), 1);
                        u = gl_fma(gl_fma(u, mine(0, j), w0), pr[0][e], w0);
                        u = gl_fma(gl_fma(u, mine(1, j), w1), pr[1][e], w1);
                        u = gl_fma(gl_fma(u, mine(2, j), w2), pr[2][e], w2);
                    }
                    acc[j * T + t] = u;
                }
            }
        }

        // Epilogue: this half of the result
        uint64_t* res = prm.out + b * (2ull * N) + (uint64_t)h * N;
        uint64_t x[1][E];
#pragma unroll
        for (int j = 0; j < E; ++j) x[0][j] = acc[j * T + t];
        if (prm.out_coef) {
            ntt_backward_unscaled_k<LOGN, 1, LOGE, R4>(x, t, xb(), tw_i);
#pragma unroll
            for (int j = 0; j < E; ++j) res[t + j * T] = gl_mul(x[0][j], prm.n_inv);
        } else {
#pragma unroll
            for (int c = 0; c < E / 2; ++c)
                *reinterpret_cast<ulonglong2*>(res + E * t + 2 * c) = make_ulonglong2(x[0][2 * c], x[0][2 * c + 1]);
        }
    }
    cluster.sync();  // neither CTA leaves while the peer may still address its shared memory
}

}  // namespace tp
