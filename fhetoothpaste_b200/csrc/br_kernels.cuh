// Batched blind rotation (CGGI binary / CGGI ternary / BMMP) for sm_100a.
//
// One thread block rotates one ciphertext at a time with T = N/E threads (E =
// 2^LOGE coefficients per thread, 8 or 4) and loops over the batch
// (persistent grid, a few blocks per SM). The RLWE
// accumulator [A | B] lives in shared memory, in the NTT domain, for all n
// CMux iterations. Per iteration the block runs the reference's CMux with the
// same residues (cggi_blind_rotation.cpp:313-472, bmmp_blind_rotation.cpp:354-419,
// mux_operator.cpp:30-294):
//   backward NTT of A and B -> gadget digits -> forward NTT of each digit ->
//   multiply-accumulate against the iteration's key rows -> monomial weights ->
//   accumulator update.
// Keys are streamed from HBM through L2: all blocks walk the iterations in the
// same order at about the same pace, so each key row is fetched from HBM about
// once per wave of blocks and served from L2 to the rest of the batch.
//
// Key layout on the device (built by key_relayout_kernel from the reference's
// m_brk): per iteration group `it` (an LWE index for CGGI, a pair for BMMP),
// per gadget row r (0..2l-1; rows < l multiply digits of A, rows >= l digits
// of B), the C = 2*G components (G RGSWs x {A, B} halves) of slot k = E*t +
// 2jp + e sit at  ((c*E/2 + jp)*T + t)*2 + e,  so each thread's 16-byte loads
// are contiguous across the warp.
#pragma once

#include <cooperative_groups.h>

#include "cluster_ntt.cuh"
#include "gl_arith.cuh"
#include "ntt_block.cuh"

namespace tp {

enum BrVariant : int { kCggiBinary = 0, kCggiTernary = 1, kBmmpBinary = 2 };

// RGSWs consumed per iteration group.
__host__ __device__ constexpr int br_rgsw_per_group(int variant) {
    return variant == kCggiBinary ? 1 : (variant == kCggiTernary ? 2 : 3);
}

struct BrKernelParams {
    const uint64_t* key;      // device layout, see above
    const uint64_t* tw_fwd;   // psi^brv(k) (k < N), then tw[i] tw[2i] (i < N/2)
    const uint64_t* tw_inv;   // psi^-brv(k), then the same products
    const uint64_t* psi_pow;  // 2N: psi^k
    const uint64_t* lwes;
    uint64_t lwe_stride;
    const uint64_t* accs;
    uint64_t acc_stride;
    uint64_t* out;
    uint64_t batch;
    uint32_t n;
    uint32_t digits;
    uint32_t out_coef;
    uint64_t n_inv;           // N^-1 mod p
    uint64_t corr;            // signed-decomposition corrector (canonical)
    uint32_t dshift[8];       // per-digit shift
    uint64_t dmask[8];        // per-digit mask
    uint64_t ddelta[8];       // per-digit offset subtracted (signed) or 0 (unsigned)
    unsigned int* err;        // bit 0: an LWE word was outside [0, 2N)
    uint32_t small_digits;    // every digit is at most 2^14 in magnitude: integer pass 0 (tile 4)
};

// Polynomials transformed together by the rotation kernel (the accumulator
// halves, the gadget digits in pairs when 2). Two measured slower (4.4k vs 6.0k
// ternary N = 2048 rotations/s): the doubled, fully unrolled transforms no longer
// fit the instruction cache, so the kernel transforms one polynomial at a time.
__host__ __device__ constexpr int br_ntt_width(int logn, int variant) {
    return (void)logn, (void)variant, 1;
}
// Twiddles live in shared memory unless the exchange buffers of the wide
// transforms leave no room for them (then they are read through L1).
__host__ __device__ constexpr bool br_smem_twiddles(int logn) { return logn <= 11; }

// Twiddle words per direction: psi^(+-brv(k)) for k < N, plus for the fused
// radix-4 passes the products tw[i] tw[2i] (i < N/2) at N + i.
__host__ __device__ constexpr int br_twiddle_words(int logn, int loge, bool r4 = true) {
    return loge == 2 && r4 ? (1 << logn) + (1 << (logn - 1)) : (1 << logn);
}

// Fused radix-4 NTT passes (three products and a shift per two levels, see
// ntt_block.cuh) for 4 coefficients per thread, by blocks per rotation. They
// trade IMAD work for ALU work. With the carry-form reduction (both integer
// pipes level) plain radix-2 butterflies are faster everywhere but in the BMMP
// four-block kernel, rotations/s: BMMP N = 2048 7808 vs 7615 (one block), 81.0
// vs 79.0 (two blocks, batch 1), 100.7 vs 102.4 (four blocks, batch 1); CGGI
// ternary N = 2048 7275 vs 6885, binary N = 1024 18.8k vs 17.5k. (With the
// earlier 16-instruction reduction radix-4 was faster for BMMP: 5570 vs 5438.)
__host__ __device__ constexpr bool br_fused_radix4(int loge, int variant, int blocks) {
    return loge == 2 && variant == kBmmpBinary && blocks == 4;
}

// Power-of-two levels of the later transform passes as shifts (ntt_block.cuh,
// pow2_block_pass) in every rotation kernel but the digit-staged CGGI ternary one
// at 2048 coefficients per CTA, where the same change measured slower although it
// spills no more (rotations/s, 4096 rotations, n = 630: 8695 on table twiddles,
// 8523 with both directions shifted, 8355 forward only, 7449 backward only; with its
// key loads grouped, 9085 on table twiddles against 8780 shifted). In
// the others it measured faster: CGGI binary N = 1024 digit-staged 20.58k ->
// 21.58k, row by row 19.38k -> 20.00k; CGGI ternary N = 2048 row by row 7861 ->
// 8014; BMMP N = 2048 9487 -> 9541; CGGI ternary N = 4096 2358 -> 2431.
__host__ __device__ constexpr bool br_table_passes(int variant, bool digit_staged, int logl) {
    return variant == kCggiTernary && digit_staged && logl == 11;
}

// Key rows staged in shared memory: each thread copies its own slots of the
// next gadget row with cp.async before the digit's transforms and reads them
// after, so the L2 latency of the key stream hides behind the NTTs. The stage
// needs C*N words and is used where it fits (not for ternary and BMMP at
// N = 4096). Keeping the accumulator in registers there to make room measured
// slower (ternary N = 4096: 1856 vs 1977 rotations/s; the spills cost more), and
// so did staging part of each row there (two components, the rest read from L2
// at use: ternary 1918 vs 1978; BMMP 2939 vs 2889, within run-to-run spread).
// Ring sizes above 4096 rotate on a cluster of 2^logs CTAs of 4096 coefficients and
// slots each (cluster_ntt.cuh): 2, 4, 8 and 16 CTAs for N = 8192 .. 65536. Fewer, larger
// CTAs measured faster than 2048 per CTA (rotations/s, n = 64: ternary N = 16384 5201 vs
// 4918 on 8 CTAs, N = 32768 2167 vs 1823 on 16, binary N = 16384 4819 vs 4315): the GPU
// keeps more SMs busy with small clusters (32 of 4 CTAs, 15 of 8, 7 of 16 resident) and a
// transform exchanges with fewer CTAs, which outweighs the 4096-coefficient plan's register
// spills. Every plan below is per CTA, in words of its local size, plus two receive areas
// of the distributed transform's exchange.
__host__ __device__ constexpr int br_cluster_logs(int logn) { return logn > 12 ? logn - 12 : 0; }

__host__ __device__ constexpr size_t br_base_words(int logn, int variant, int loge, int logs = 0, bool r4 = false) {
    return (size_t)(br_smem_twiddles(logn - logs)
                        ? 2 * br_twiddle_words(logn - logs, loge, r4 || br_fused_radix4(loge, variant, 1))
                        : 0) +
           (size_t)(1 << (logn - logs)) * (2 * br_ntt_width(logn, variant) + 2 + (logs ? 2 : 0)) +
           1024;  // LWE area budget for the plan; the host adds the real size
}
__host__ __device__ constexpr size_t br_stage_words(int logn, int variant, int logs = 0) {
    return (size_t)(1 << (logn - logs)) * 2 * br_rgsw_per_group(variant);
}
__host__ __device__ constexpr bool br_key_prefetch(int logn, int variant, int loge, int logs = 0, bool r4 = false) {
    return (br_base_words(logn, variant, loge, logs, r4) + br_stage_words(logn, variant, logs)) * 8 <= 227u * 1024u;
}

// Digit-staged multiply-accumulate (template parameter DL = the digit count l,
// 4 coefficients per thread): each iteration transforms all 2l gadget digits
// first, keeping rows 0..2l-2 in shared memory (each thread its own slots) and
// the last in registers, then sums every output word over the 2l rows exactly
// (WideAcc) and reduces it once, reading the key words straight from L2. No
// key row stage. A running canonical sum instead pays a reduction per row.
// Key loads of the digit-staged multiply-accumulate run ahead of their use either
// row by row, AH rows ahead through a ring of registers (AH > 0), or a whole
// (slot pair, component) group of 2l rows at a time, one group ahead (AH = 0).
// Measured (rotations/s, full waves, N = 2048): CGGI ternary 8185 (ring, 5 ahead),
// 7850 (8), 7274 (11), 7911 (groups); BMMP 9212 (groups) against 6204 and 6020
// for rings of 5 and 8; CGGI binary N = 1024 about equal (20.35k to 20.55k).
// Re-measured on the current kernel: CGGI ternary 9089 (groups), 8695 (ring, 5 ahead),
// 7799 (4), 8817 (6), 8340 (7), 8236 (8), with the fused radix-4 passes 8858 (groups),
// 8884 (6); binary N = 1024 21.55k (5), 21.50k (4), 21.49k (6), 21.39k (groups); BMMP
// 9546 (groups), 6174 (4), 6313 (6); CGGI ternary N = 1024 24.76k (5) against 24.63k
// (groups), N = 512 49.87k either way.
__host__ __device__ constexpr int br_ds_ahead(int variant, int logl) {
    return variant == kBmmpBinary ? 0 : (variant == kCggiTernary && logl >= 11 ? 0 : 5);
}
// Contexts start with radix-2 passes: with the digit-staged sums the fused radix-4 form
// measured slower (CGGI ternary N = 2048, l = 3: 8858 against 9089 rotations/s; binary
// N = 1024: 18.2k against 21.6k); tp_br_set_radix and the autotuner still offer it.

__host__ __device__ constexpr size_t br_digit_stage_words(int logn, int dl) {
    return dl > 0 ? (size_t)(2 * dl - 1) << logn : 0;
}

// Shared memory of one block, in words (local size NL = 2^(logn - logs)):
// twiddles (both directions, if kept there), two exchange areas of width*NL words,
// the accumulator (2 NL), the key row stage (C NL, if used) or the digit stage
// (DL > 0), two receive areas (2 NL, clusters only), the LWE vector (n+1, rounded
// up to an even count).
__host__ __device__ constexpr size_t br_smem_words(int logn, int variant, uint32_t n, int loge, int dl = 0,
                                                   int logs = 0, bool r4 = false) {
    return (size_t)(br_smem_twiddles(logn - logs)
                        ? 2 * br_twiddle_words(logn - logs, loge, r4 || br_fused_radix4(loge, variant, 1))
                        : 0) +
           (size_t)(1 << (logn - logs)) * (2 * br_ntt_width(logn, variant) + 2 + (logs ? 2 : 0)) +
           (dl > 0 ? br_digit_stage_words(logn - logs, dl)
                   : (br_key_prefetch(logn, variant, loge, logs, r4) ? br_stage_words(logn, variant, logs) : 0)) +
           ((n + 2) & ~1u);
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Exponent e_k = 2 brv(k) + 1 of slot k: NTT(X^a)[k] = psi^(e_k a mod 2N).
template <int LOGN>
__device__ __forceinline__ uint32_t slot_exponent(int k) {
    return 2u * (__brev((uint32_t)k) >> (32 - LOGN)) + 1u;
}

template <int LOGN>
__device__ __forceinline__ uint64_t mono(const uint64_t* __restrict__ psi_pow, uint32_t ek, uint32_t a) {
    return __ldg(psi_pow + ((ek * a) & (2u * (1u << LOGN) - 1u)));
}


// Coefficients per thread (log2) a context starts with; tp_br_set_tile and
// tp_br_autotune change it. 4 per thread measured faster than 8 for every
// variant and ring size (rotations/s, full waves: ternary N = 2048 7286 vs
// 6798, BMMP N = 2048 7658 vs 7099, binary N = 1024 18786 vs 17168, ternary
// N = 4096 2188 vs 1874): twice the warps per SM hide the integer pipes'
// dependency latency that 8 per thread left exposed. Re-measured on the current
// kernels at N = 4096 (rotations/s): ternary 2432 vs 1789, binary 4132 vs 4033,
// BMMP 2818 vs 2091.
__host__ __device__ constexpr int br_default_loge(int logn, int variant) {
    return (void)logn, (void)variant, 2;
}

// Resident blocks per SM the kernel is compiled for (register budget
// 65536 / (T * blocks)). With 8 coefficients per thread, from N = 2048 up one
// block per SM with the full register file measured faster than two blocks
// that spill (ternary N = 2048: 6.0k vs 5.3k rotations/s). With 4 per thread
// the budget is 128 registers (two blocks of N/4 threads up to N = 1024, one
// block of 512 threads at N = 2048).
__host__ __device__ constexpr int br_min_blocks(int logn, int variant, int loge) {
    return loge == 2 ? (logn <= 10 ? 2 : 1) : ((logn >= 11 || variant == kBmmpBinary) ? 1 : 2);
}

// LOGS > 0: one rotation per cluster of 2^LOGS CTAs (launched with that cluster
// size), each CTA holding the coefficients i = i' 2^LOGS + r and the slots
// r NL .. r NL + NL - 1 of the cluster's rank r (cluster_ntt.cuh); the
// multiply-accumulate, the update and the key words of a slot are local to its CTA.
// RADIX4: the transforms' radix-4 passes use the fused form (three products and a
// shift per two levels, ntt_block.cuh) instead of radix-2 butterflies: a runtime
// choice per context (tp_br_set_radix), built for one CTA per rotation.
template <int LOGN, int VARIANT, int LOGE, int DL = 0, int LOGS = 0, bool RADIX4 = false>
__global__ void __launch_bounds__((1 << (LOGN - LOGS)) >> LOGE, br_min_blocks(LOGN - LOGS, VARIANT, LOGE))
br_kernel(const BrKernelParams prm) {
    constexpr int LOGL = LOGN - LOGS;        // log2 of the coefficients / slots per CTA
    using SH = NttShape<LOGL, LOGE>;
    constexpr int N = 1 << LOGN;             // ring dimension
    constexpr int NL = SH::N;
    constexpr int T = SH::T;
    constexpr int E = SH::E;
    constexpr int G = br_rgsw_per_group(VARIANT);
    constexpr int C = 2 * G;                 // key components per slot
    constexpr int K = br_ntt_width(LOGN, VARIANT);  // polynomials per transform
    constexpr bool TW_SMEM = br_smem_twiddles(LOGL);
    constexpr uint32_t MASK2N = 2u * N - 1u;
    constexpr bool SIGNED = VARIANT != kCggiBinary;
    constexpr bool R4 = RADIX4 || br_fused_radix4(LOGE, VARIANT, 1);
    static_assert(!RADIX4 || LOGE == 2, "the fused radix-4 passes need 4 coefficients per thread");
    constexpr bool DS = DL > 0;              // digit-staged multiply-accumulate (prm.digits == DL)
    constexpr bool PF = !DS && br_key_prefetch(LOGN, VARIANT, LOGE, LOGS, R4);
    static_assert(!DS || (LOGE == 2 && K == 1), "the digit stage runs with 4 coefficients per thread");
    static_assert(LOGS == 0 || (LOGE == 2 && K == 1 && !R4), "clusters run radix-2 with 4 coefficients per thread");
    constexpr int NF = (R4 ? kNttRadix4 : 0) | (br_table_passes(VARIANT, DS, LOGL) ? kNttTablePasses : 0);

    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* base = smem;
    const uint64_t* tw_f = prm.tw_fwd;
    const uint64_t* tw_i = prm.tw_inv;
    if constexpr (TW_SMEM) {
        constexpr int TWW = br_twiddle_words(LOGL, LOGE, R4);  // the first NL words of the N-point tables
        for (int i = threadIdx.x; i < TWW; i += T) {
            base[i] = prm.tw_fwd[i];
            base[TWW + i] = prm.tw_inv[i];
        }
        tw_f = base;
        tw_i = base + TWW;
        base += 2 * TWW;
    }
    uint64_t* xbuf0 = base;
    uint64_t* xbuf1 = base + K * NL;
    uint64_t* acc = base + 2 * K * NL;       // [(h*E + j)*T + t], canonical, NTT domain
    uint64_t* kst = acc + 2 * NL;            // key row stage, this CTA's part of one row (C*NL words)
    // digit stage (DS): row r < 2L-1 of this thread's slot pair jp at xs + r*NL + (jp*T + t)*2
    uint64_t* xs = acc + 2 * NL;
    uint64_t* recv0 = kst + (PF ? C * NL : (DS ? (2 * DL - 1) * NL : 0));  // cluster exchange areas
    uint64_t* recv1 = recv0 + NL;
    uint64_t* lwe_s = recv0 + (LOGS ? 2 * NL : 0);
    int cr = 0;                              // rank in the cluster
    if constexpr (LOGS > 0) {
        cr = (int)cooperative_groups::this_cluster().block_rank();
        cooperative_groups::this_cluster().sync();  // every CTA of the cluster running before remote stores
    }
    const uint32_t sbase = (uint32_t)cr << LOGL;  // first slot of this CTA

    const int t = threadIdx.x;
    const uint32_t n = prm.n;
    const uint32_t L = prm.digits;
    // slot j of accumulator half h of this thread
    auto acc_ld = [&](int h, int j) -> uint64_t { return acc[(h * E + j) * T + t]; };
    auto acc_st = [&](int h, int j, uint64_t v) { acc[(h * E + j) * T + t] = v; };

    int sel = 0;
    auto xb = [&]() -> uint64_t* {
        uint64_t* b = sel ? xbuf1 : xbuf0;
        sel ^= 1;
        return b;
    };
    int rsel = 0;
    auto recv_next = [&]() -> uint64_t* {
        uint64_t* b = rsel ? recv1 : recv0;
        rsel ^= 1;
        return b;
    };
    // the cluster halves of a forward / backward transform (nothing for one CTA)
    auto fwd_tail = [&](uint64_t (&v)[E]) {
        if constexpr (LOGS > 0)
            cluster_fwd_tail<LOGN, LOGS, true>(reinterpret_cast<uint64_t(&)[4]>(v), t, cr, recv_next(),
                                               (1 << LOGS) > 4 ? xb() : nullptr, prm.tw_fwd);
    };
    auto inv_head = [&](uint64_t (&v)[E]) {
        if constexpr (LOGS > 0)
            cluster_inv_head<LOGN, LOGS>(reinterpret_cast<uint64_t(&)[4]>(v), t, cr, recv_next(),
                                         (1 << LOGS) > 4 ? xb() : nullptr, prm.tw_inv);
    };

    for (uint64_t b = blockIdx.x >> LOGS; b < prm.batch; b += gridDim.x >> LOGS) {
        __syncthreads();  // previous ciphertext done with lwe_s / acc (and twiddles written)
        const uint64_t* lwe = prm.lwes + b * prm.lwe_stride;
        bool bad = false;
        for (uint32_t i = t; i <= n; i += T) {
            uint64_t v = lwe[i];
            bad |= v > MASK2N;
            lwe_s[i] = v & MASK2N;
        }
        if (bad && cr == 0) atomicOr(prm.err, 1u);
        __syncthreads();

        // Prologue: acc = NTT(acc_in) * X^b   (cggi_blind_rotation.cpp:242,333-358)
        {
            const uint64_t* ain = prm.accs + b * prm.acc_stride;
            const uint32_t bb = (uint32_t)lwe_s[n];
#pragma unroll 1
            for (int h0 = 0; h0 < 2; h0 += K) {
                uint64_t x[K][E];
#pragma unroll
                for (int p = 0; p < K; ++p)
#pragma unroll
                    for (int j = 0; j < E; ++j) x[p][j] = ain[(h0 + p) * N + ((uint32_t)(t + j * T) << LOGS) + cr];
                ntt_forward_k<LOGL, K, LOGE, NF, true>(x, t, xb(), tw_f);
                fwd_tail(x[0]);
#pragma unroll
                for (int p = 0; p < K; ++p)
#pragma unroll
                    for (int j = 0; j < E; ++j)
                        acc_st(h0 + p, j,
                               gl_mul(x[p][j], mono<LOGN>(prm.psi_pow, slot_exponent<LOGN>(sbase + E * t + j), bb)));
            }
        }

        const uint32_t step = VARIANT == kBmmpBinary ? 2 : 1;
#pragma unroll 1
        for (uint32_t i = 0; i < n; i += step) {
            uint32_t a0 = (uint32_t)lwe_s[i];
            uint32_t a1 = 0;
            if constexpr (VARIANT == kBmmpBinary) {
                a0 = (2u * N - a0) & MASK2N;                         // X^{-a} (bmmp_blind_rotation.cpp:403-404)
                a1 = (2u * N - (uint32_t)lwe_s[i + 1]) & MASK2N;
            } else {
                if (a0 == 0) continue;                               // cggi_blind_rotation.cpp:369-370
            }
            // this CTA's part of the group's key rows (row stride C*N, part offset C*NL*cr)
            const uint64_t* kit = prm.key + (uint64_t)(i / step) * (2ull * L * N * C) + (uint64_t)cr * (C * NL);

            // MAC accumulators (canonical: every update is a gl_fma); the digit-staged
            // form sums per slot pair after the digit loop instead
            uint64_t o[DS ? 1 : C][DS ? 1 : E];
            if constexpr (!DS) {
#pragma unroll
                for (int c = 0; c < C; ++c)
#pragma unroll
                    for (int j = 0; j < E; ++j) o[c][j] = 0;
            }

            // Backward NTT of an accumulator half into corrected coefficients. Binary
            // CGGI decomposes (X^{-a} - 1) * acc (mux_operator.cpp:144-150); the other
            // variants decompose acc itself (mux_operator.cpp:174-177, 219-224).
            uint64_t cx[2][E];
            auto load_half = [&](uint64_t (&dst)[E], int h) {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    dst[j] = acc_ld(h, j);
                    if constexpr (VARIANT == kCggiBinary)
                        dst[j] = gl_mul(dst[j], gl_sub(mono<LOGN>(prm.psi_pow, slot_exponent<LOGN>(sbase + E * t + j),
                                                                  2u * N - a0), 1));
                }
            };
            // times 1/N (a shift: N^-1 = 2^-log2 N), plus the signed-digit corrector
            // (gadget_decomp.h:169-173)
            auto finish_half = [&](uint64_t (&v)[E]) {
#pragma unroll
                for (int j = 0; j < E; ++j) v[j] = gl_add(gl_div_pow2<LOGN>(v[j]), prm.corr);
            };
            if constexpr (K == 2) {
                load_half(cx[0], 0);
                load_half(cx[1], 1);
                ntt_backward_unscaled_k<LOGL, 2, LOGE, NF>(cx, t, xb(), tw_i);
                finish_half(cx[0]);
                finish_half(cx[1]);
            }
            uint64_t x[K][E];  // digit transform of the row last processed
#pragma unroll 1
            for (uint32_t r = 0; r < 2 * L; r += K) {
                if constexpr (PF && K == 1) {
                    // this thread's slots of key row r; read back by this thread only
                    const uint64_t* kr = kit + (uint64_t)r * (N * C);
#pragma unroll
                    for (int c = 0; c < C; ++c)
#pragma unroll
                        for (int jp = 0; jp < E / 2; ++jp) {
                            const int ko = ((c * (E / 2) + jp) * T + t) * 2;
                            cp_async16(kst + ko, kr + ko);
                        }
                    cp_async_commit();
                }
                if constexpr (K == 1) {
                    if (r == 0 || r == L) {
                        uint64_t (&c1)[1][E] = reinterpret_cast<uint64_t(&)[1][E]>(cx[0]);
                        load_half(cx[0], r == 0 ? 0 : 1);
                        inv_head(cx[0]);
                        ntt_backward_unscaled_k<LOGL, 1, LOGE, NF>(c1, t, xb(), tw_i);
                        finish_half(cx[0]);
                    }
                }
                bool pass0_done = false;
                if constexpr (LOGE == 2 && K == 1) {
                    if (prm.small_digits) {
                        // digits as small signed integers, levels 0 and 1 in integer arithmetic
                        const uint32_t d = r < L ? r : r - L;
                        const uint32_t sh = prm.dshift[d];
                        const uint64_t mk = prm.dmask[d];
                        const int64_t dl = SIGNED ? (int64_t)prm.ddelta[d] : 0;
                        int64_t dv[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) dv[j] = (int64_t)((cx[0][j] >> sh) & mk) - dl;
                        ntt_pass0_small(dv, reinterpret_cast<uint64_t(&)[4]>(x[0]));
                        pass0_done = true;
                    }
                }
                if (!pass0_done) {
#pragma unroll
                    for (int p = 0; p < K; ++p) {
                        const uint32_t rr = r + p;
                        const bool hb = K == 2 && rr >= L;          // digit of the B half
                        const uint32_t d = rr < L ? rr : rr - L;
                        const uint32_t sh = prm.dshift[d];
                        const uint64_t mk = prm.dmask[d];
                        const uint64_t dl = prm.ddelta[d];
#pragma unroll
                        for (int j = 0; j < E; ++j) {
                            const uint64_t c = hb ? cx[K - 1][j] : cx[0][j];
                            const uint64_t raw = (c >> sh) & mk;
                            x[p][j] = SIGNED ? gl_sub(raw, dl) : raw;
                        }
                    }
                    fwd_pass_math<LOGL, 0, K, LOGE, NF, true>(x, t, tw_f);
                }
                ntt_forward_after_pass0<LOGL, K, LOGE, NF, true>(x, t, xb(), tw_f);
                fwd_tail(x[0]);
                if constexpr (DS) {
                    // rows before the last wait in the stage (this thread's own slots: no barrier)
                    if (r + 1 < 2 * L) {
#pragma unroll
                        for (int jp = 0; jp < E / 2; ++jp)
                            *reinterpret_cast<ulonglong2*>(xs + r * NL + (jp * T + t) * 2) =
                                make_ulonglong2(x[0][2 * jp], x[0][2 * jp + 1]);
                    }
                } else {
                    if constexpr (PF && K == 1) cp_async_wait_all();
#pragma unroll
                    for (int p = 0; p < K; ++p) {
                        const uint64_t* kr = kit + (uint64_t)(r + p) * (N * C);
#pragma unroll
                        for (int c = 0; c < C; ++c) {
#pragma unroll
                            for (int jp = 0; jp < E / 2; ++jp) {
                                const int ko = ((c * (E / 2) + jp) * T + t) * 2;
                                const ulonglong2 kv = (PF && K == 1)
                                                          ? *reinterpret_cast<const ulonglong2*>(kst + ko)
                                                          : __ldg(reinterpret_cast<const ulonglong2*>(kr + ko));
                                o[c][2 * jp] = gl_fma(o[c][2 * jp], x[p][2 * jp], kv.x);
                                o[c][2 * jp + 1] = gl_fma(o[c][2 * jp + 1], x[p][2 * jp + 1], kv.y);
                            }
                        }
                    }
                }
            }

            // Accumulator update of slot j from its C key-component sums oj[c].
            auto update = [&](int j, const uint64_t* oj) {
                const uint32_t ek = slot_exponent<LOGN>(sbase + E * t + j);
                uint64_t ua = acc_ld(0, j);
                uint64_t ub = acc_ld(1, j);
                if constexpr (VARIANT == kCggiBinary) {
                    // acc += ExtProd (mux_operator.cpp:151)
                    ua = gl_add(ua, oj[0]);
                    ub = gl_add(ub, oj[1]);
                } else if constexpr (VARIANT == kCggiTernary) {
                    // acc += (X^{-a}-1) ExtProd(lo) + (X^{a}-1) ExtProd(hi) (mux_operator.cpp:188-200)
                    const uint64_t mp = gl_sub(mono<LOGN>(prm.psi_pow, ek, 2u * N - a0), 1);
                    const uint64_t mn = gl_sub(mono<LOGN>(prm.psi_pow, ek, a0), 1);
                    ua = gl_fma(gl_fma(ua, oj[0], mp), oj[2], mn);
                    ub = gl_fma(gl_fma(ub, oj[1], mp), oj[3], mn);
                } else {
                    // weights X^{a0}-1, X^{a1}-1, X^{a0+a1}-X^{a0}-X^{a1}+1
                    // (bmmp_blind_rotation.cpp:280-323; MultiMux mux_operator.cpp:274-291)
                    const uint64_t m0 = mono<LOGN>(prm.psi_pow, ek, a0);
                    const uint64_t m1 = mono<LOGN>(prm.psi_pow, ek, a1);
                    const uint64_t m2 = mono<LOGN>(prm.psi_pow, ek, (a0 + a1) & MASK2N);
                    const uint64_t w0 = gl_sub(m0, 1);
                    const uint64_t w1 = gl_sub(m1, 1);
                    const uint64_t w2 = gl_add(gl_sub(gl_sub(m2, m0), m1), 1);
                    ua = gl_fma(gl_fma(gl_fma(ua, oj[0], w0), oj[2], w1), oj[4], w2);
                    ub = gl_fma(gl_fma(gl_fma(ub, oj[1], w0), oj[3], w1), oj[5], w2);
                }
                acc_st(0, j, ua);
                acc_st(1, j, ub);
            };

            if constexpr (DS) {
                // Every slot's C sums over the 2L rows, exact, one reduction each: for slot
                // pair jp and key component c, the thread's 16 bytes of row r sit at
                // ((c*E/2 + jp)*T + t)*2 of that row. The loads run ahead of their use in one
                // of two schedules (br_ds_ahead).
                constexpr int R2 = 2 * (DL > 0 ? DL : 1);
                constexpr int AH = br_ds_ahead(VARIANT, LOGL);
                auto kaddr = [&](int jp, int c, int r) {
                    return reinterpret_cast<const ulonglong2*>(kit + (uint64_t)r * (N * C) +
                                                               ((c * (E / 2) + jp) * T + t) * 2);
                };
                auto row_x = [&](int jp, int r) -> ulonglong2 {
                    return r < R2 - 1 ? *reinterpret_cast<const ulonglong2*>(xs + r * NL + (jp * T + t) * 2)
                                      : make_ulonglong2(x[0][2 * jp], x[0][2 * jp + 1]);
                };
                if constexpr (AH > 0) {
                    // steps st = (jp*C + c)*2L + r, each row's key requested AH steps ahead
                    // through a ring of AH+1 register pairs
                    constexpr int NS = (E / 2) * C * R2;
                    ulonglong2 ring[AH + 1];
#pragma unroll
                    for (int st = 0; st < AH && st < NS; ++st)
                        ring[st] = __ldg(kaddr(st / (C * R2), (st / R2) % C, st % R2));
                    WideAcc s0, s1;
                    uint64_t oj[2][C];
#pragma unroll
                    for (int st = 0; st < NS; ++st) {
                        if (st + AH < NS) {
                            const int sa = st + AH;
                            ring[sa % (AH + 1)] = __ldg(kaddr(sa / (C * R2), (sa / R2) % C, sa % R2));
                        }
                        const int jp = st / (C * R2), c = (st / R2) % C, r = st % R2;
                        const ulonglong2 kv = ring[st % (AH + 1)];
                        if (r == 0) {
                            wide_zero(s0);
                            wide_zero(s1);
                        }
                        const ulonglong2 xv = row_x(jp, r);
                        wide_mad(s0, xv.x, kv.x);
                        wide_mad(s1, xv.y, kv.y);
                        if (r == R2 - 1) {
                            oj[0][c] = wide_reduce(s0);
                            oj[1][c] = wide_reduce(s1);
                            if (c == C - 1) {
                                update(2 * jp, oj[0]);
                                update(2 * jp + 1, oj[1]);
                            }
                        }
                    }
                } else {
                    // groups g = jp*C + c: all 2L rows of a group requested together, one group
                    // ahead of their use
                    constexpr int NG = C * (E / 2);
                    ulonglong2 kv[2][R2];
                    auto kload = [&](int g, ulonglong2 (&k)[R2]) {
#pragma unroll
                        for (int r = 0; r < R2; ++r) k[r] = __ldg(kaddr(g / C, g % C, r));
                    };
                    kload(0, kv[0]);
#pragma unroll
                    for (int jp = 0; jp < E / 2; ++jp) {
                        uint64_t oj[2][C];
#pragma unroll
                        for (int c = 0; c < C; ++c) {
                            const int g = jp * C + c;
                            if (g + 1 < NG) kload(g + 1, kv[(g + 1) & 1]);
                            WideAcc s0, s1;
                            wide_zero(s0);
                            wide_zero(s1);
#pragma unroll
                            for (int r = 0; r < R2; ++r) {
                                const ulonglong2 xv = row_x(jp, r);
                                wide_mad(s0, xv.x, kv[g & 1][r].x);
                                wide_mad(s1, xv.y, kv[g & 1][r].y);
                            }
                            oj[0][c] = wide_reduce(s0);
                            oj[1][c] = wide_reduce(s1);
                        }
                        update(2 * jp, oj[0]);
                        update(2 * jp + 1, oj[1]);
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < E; ++j) {
                    uint64_t oj[C];
#pragma unroll
                    for (int c = 0; c < C; ++c) oj[c] = o[c][j];
                    update(j, oj);
                }
            }
        }

        // Epilogue (cggi_blind_rotation.cpp:258-261).
        uint64_t* res = prm.out + b * (2ull * N);
#pragma unroll 1
        for (int h0 = 0; h0 < 2; h0 += K) {
            uint64_t x[K][E];
#pragma unroll
            for (int p = 0; p < K; ++p)
#pragma unroll
                for (int j = 0; j < E; ++j) x[p][j] = acc_ld(h0 + p, j);
            if (prm.out_coef) {
                inv_head(x[0]);
                ntt_backward_unscaled_k<LOGL, K, LOGE, NF>(x, t, xb(), tw_i);
#pragma unroll
                for (int p = 0; p < K; ++p)
#pragma unroll
                    for (int j = 0; j < E; ++j)
                        res[(h0 + p) * N + ((uint32_t)(t + j * T) << LOGS) + cr] = gl_div_pow2<LOGN>(x[p][j]);
            } else {
#pragma unroll
                for (int p = 0; p < K; ++p)
#pragma unroll
                    for (int c = 0; c < E / 2; ++c)
                        *reinterpret_cast<ulonglong2*>(res + (h0 + p) * N + sbase + E * t + 2 * c) =
                            make_ulonglong2(x[p][2 * c], x[p][2 * c + 1]);
            }
        }
    }
}

}  // namespace tp
