// Element-wise kernels of the LWE -> RGSW scheme switch (C ABI unit only);
// lib/src/operators/lwe_to_rgsw_conversion.cpp:168-225.
#pragma once

#include "gl_arith.cuh"

namespace tp {

// Lev row d of ciphertext b, scaled by N^-1 for the trace that follows
// (trace_evaluation.cpp:143): X^{-d*bs} (R_b + (0, tp)), where R_b is the
// rotation output in coefficients and tp the test polynomial added to its B
// half (lwe_to_rgsw_conversion.cpp:180). The rotation reads [A, -A, B, -B] at
// offset d*bs (lines 188-200).
// N = 2^logn and D = 2^logd (D divides N, so it is a power of two too): index
// arithmetic by shifts and masks.
__global__ void ss_rows_kernel(uint64_t* __restrict__ rows, const uint64_t* __restrict__ rot,
                               const uint64_t* __restrict__ tp, uint64_t batch, uint32_t logd, uint32_t logn,
                               uint32_t bs, uint64_t n_inv) {
    const uint32_t N = 1u << logn;
    const uint64_t total = batch << (logd + logn + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(w & (N - 1));
        const uint32_t h = (uint32_t)((w >> logn) & 1);
        const uint64_t row = w >> (logn + 1);
        const uint32_t d = (uint32_t)(row & ((1u << logd) - 1));
        const uint64_t b = row >> logd;
        uint32_t src = k + d * bs;
        const bool neg = src >= N;
        if (neg) src -= N;
        uint64_t v = rot[b * 2ull * N + (uint64_t)h * N + src];
        if (h) v = gl_add(v, tp[src]);
        if (neg) v = gl_neg(v);
        rows[w] = gl_mul(v, n_inv);
    }
}

// out_b = [lev_left rows | lev_right rows]: right row d = the traced row T (NTT
// domain); left row d = [T.B - O.A, -O.B] with O = -KS_{s^2 -> s}(INTT(T.A))
// (lines 208-224: the converter subtracts into a zero row, the result is
// negated, then T.B is added to its A half).
__global__ void ss_assemble_kernel(uint64_t* __restrict__ out, const uint64_t* __restrict__ rows,
                                   const uint64_t* __restrict__ sq, uint64_t batch, uint32_t logd, uint32_t logn) {
    const uint32_t N = 1u << logn, D = 1u << logd;
    const uint64_t total = batch << (logd + logn + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(w & (2ull * N - 1));
        const uint64_t row = w >> (logn + 1);
        const uint32_t d = (uint32_t)(row & (D - 1));
        const uint64_t b = row >> logd;
        const uint64_t* t = rows + row * 2ull * N;
        const uint64_t* o = sq + row * 2ull * N;
        uint64_t* ob = out + b * 4ull * N * D;
        ob[2ull * N * D + (uint64_t)d * 2 * N + k] = t[k];
        ob[(uint64_t)d * 2 * N + k] = k < N ? gl_sub(t[N + k], o[k]) : gl_neg(o[k]);
    }
}

}  // namespace tp
