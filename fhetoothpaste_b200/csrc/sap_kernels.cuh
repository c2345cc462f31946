// Element-wise kernels of the SAP digit decomposition (C ABI unit only);
// lib/src/operators/sap_decomposer.cpp. The heavy steps (blind rotations, the
// truncation tree's automorphism key switches, NTTs, the reset's key switch)
// run on the library's rotation, key-switch and NTT kernels.
#pragma once

#include "gl_arith.cuh"

namespace tp {

// The reference's IntLog2 (math_utils.cpp:11-25): ceil(log2 x), 0 for x <= 1.
__device__ __forceinline__ uint32_t ref_int_log2(uint64_t x) { return x <= 1 ? 0u : 64u - __clzll(x - 1); }

// Per LWE: copy of the input and the input modulus read from the words
// themselves (lines 409-416: 2^IntLog2(a_0), doubled once for each later word it
// does not exceed).
__global__ void sap_init_kernel(uint64_t* __restrict__ copy, uint64_t* __restrict__ modulus,
                                const uint64_t* __restrict__ in, uint64_t batch, uint32_t n) {
    const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const uint64_t* x = in + b * (n + 1ull);
    uint64_t* c = copy + b * (n + 1ull);
    uint64_t M = 1ull << ref_int_log2(x[0]);
    c[0] = x[0];
    for (uint32_t i = 1; i <= n; ++i) {
        const uint64_t v = x[i];
        if (M <= v) M <<= 1;
        c[i] = v;
    }
    modulus[b] = M;
}

// The starting accumulators (0, Q/2N) in coefficients (lines 389-392).
__global__ void sap_acc_init_kernel(uint64_t* __restrict__ acc, uint64_t batch, uint32_t logn) {
    const uint64_t N = 1ull << logn, total = batch << (logn + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x)
        acc[w] = (w & (2 * N - 1)) == N ? kP / (2 * N) : 0;
}

// One digit step on every LWE (lines 421-430): sub = copy mod radix, copy >>=
// log radix, M >>= log radix, then the perturbations sub_n += radix*beta (mod 2N)
// and copy_n -= beta (mod M, the reference's SubUIntMod). flags[b]: bit 0 = the
// LWE is still decomposing at this step, bit 1 = its accumulator is reset after it.
__global__ void sap_digit_kernel(uint64_t* __restrict__ copy, uint64_t* __restrict__ sub,
                                 uint64_t* __restrict__ modulus, uint8_t* __restrict__ flags, uint64_t batch,
                                 uint32_t n, uint32_t N, uint32_t log_radix, uint64_t beta, uint64_t step,
                                 uint64_t restart) {
    const uint64_t per = n + 1ull;
    const uint64_t total = batch * per;
    const uint64_t mask = (1ull << log_radix) - 1;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / per, i = w % per;
        uint64_t s = copy[w] & mask;
        uint64_t c = copy[w] >> log_radix;
        if (i == n) {
            const uint64_t M0 = modulus[b];
            const uint64_t M = M0 >> log_radix;
            s = (s + (beta << log_radix)) % (2ull * N);
            c = c >= beta ? c - beta : c + M - beta;
            const bool active = M0 > 1;
            const bool reset = active && (step + 1) % restart == 0 && M != 0;
            flags[b] = (uint8_t)((active ? 1 : 0) | (reset ? 2 : 0));
            if (active) modulus[b] = M;
        }
        sub[w] = s;
        copy[w] = c;
    }
}

// dst = src (.) poly * scale over both halves of every RLWE (NTT domain).
__global__ void sap_mul_poly_kernel(uint64_t* __restrict__ dst, uint64_t dst_stride, const uint64_t* __restrict__ src,
                                    const uint64_t* __restrict__ poly, uint64_t scale, uint64_t batch, uint32_t logn) {
    const uint64_t N = 1ull << logn, total = batch << (logn + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> (logn + 1), k = w & (2 * N - 1);
        dst[b * dst_stride + k] = gl_mul(gl_mul(src[w], poly[k & (N - 1)]), scale);
    }
}

// SampleExtract(0) of RLWE b (coefficients) into digit `step` of LWE b's output
// (lines 443-445), for the LWEs still decomposing.
__global__ void sap_extract_kernel(uint64_t* __restrict__ out, uint64_t out_stride, uint64_t step,
                                   const uint64_t* __restrict__ rlwe, const uint8_t* __restrict__ flags,
                                   uint64_t batch, uint32_t N) {
    const uint64_t per = N + 1ull;
    const uint64_t total = batch * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / per, i = w % per;
        if (!(flags[b] & 1)) continue;
        const uint64_t* src = rlwe + b * 2ull * N;
        const uint64_t v = i == 0 ? src[0] : (i < N ? gl_neg(src[N - i]) : src[N]);
        out[b * out_stride + step * per + i] = v;
    }
}

// acc_b <- fresh_b where LWE b is reset at this step.
__global__ void sap_select_kernel(uint64_t* __restrict__ acc, const uint64_t* __restrict__ fresh,
                                  const uint8_t* __restrict__ flags, uint64_t batch, uint32_t logn) {
    const uint64_t total = batch << (logn + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        if (flags[w >> (logn + 1)] & 2) acc[w] = fresh[w];
    }
}

// End of HomTrunc (lines 253-263), in coefficients: acc_b = sum_e X^brev(e) * leaf_{b,e}
// over the 2^L leaves of LWE b's tree (leaf e at words e*2N of its tree).
__global__ void sap_leaf_sum_kernel(uint64_t* __restrict__ acc, const uint64_t* __restrict__ tree, uint64_t batch,
                                    uint32_t logn, uint32_t L) {
    const uint32_t N = 1u << logn;
    const uint64_t total = batch << (logn + 1);
    const uint32_t leaves = 1u << L;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> (logn + 1);
        const uint32_t k = (uint32_t)(w & (2ull * N - 1));
        const uint32_t h = k >> logn, m = k & (N - 1);
        const uint64_t* t = tree + b * (uint64_t)leaves * 2 * N + (uint64_t)h * N;
        uint64_t sum = 0;
        for (uint32_t e = 0; e < leaves; ++e) {
            const uint32_t r = L ? (__brev(e) >> (32 - L)) : 0;
            const uint64_t* leaf = t + (uint64_t)e * 2 * N;
            sum = m >= r ? gl_add(sum, leaf[m - r]) : gl_sub(sum, leaf[m + N - r]);
        }
        acc[w] = sum;
    }
}

}  // namespace tp
