// Packing set-up and LWE -> LWE key switching (launched by the C ABI unit only).
#pragma once

#include "gl_arith.cuh"

namespace tp {

// L0Setup of every packing input (lwe_to_rlwe_packing.cpp:238-251), written in
// the packing tree's element order: node c of pack p takes input
// (len-1) ^ brv_{log len}(c) (lwe_to_rlwe_packing.cpp:143).
__global__ void pack_l0_kernel(uint64_t* __restrict__ nodes, const uint64_t* __restrict__ in, uint64_t packs,
                               uint32_t len, uint32_t log_len, uint32_t logn, uint64_t n_inv) {
    const uint64_t N = 1ull << logn;
    const uint64_t total = packs * len * 2 * N;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = w % (2 * N);
        const uint64_t c = (w / (2 * N)) % len;
        const uint64_t p = w / (2 * N * len);
        const uint32_t src = (len - 1) ^ (log_len ? (__brev((uint32_t)c) >> (32 - log_len)) : 0u);
        const uint64_t* lwe = in + (p * len + src) * (N + 1);
        uint64_t v;
        if (k == 0) v = lwe[0];
        else if (k < N) v = gl_neg(lwe[N - k]);
        else if (k == N) v = lwe[N];
        else v = 0;
        nodes[w] = gl_mul(v, n_inv);
    }
}

// ---------------------------------------------------------------------------
// LWE -> LWE key switching (lib/src/operators/lwe_conversion.cpp:205-239), q = p:
//   out[n_out] = in[n_in]; out[k] -= sum_{i,j} digit_j(in[i]) * ksk[i][j][k]
// A block owns 16 ciphertexts x 128 output words; digits of a chunk of input
// coefficients are staged in shared memory, key words stream through L1/L2.
// ---------------------------------------------------------------------------
struct LweKsParams {
    const uint64_t* ksk;      // reference layout: [i][j][n_out + 1]
    const uint64_t* in;       // batch x (n_in + 1)
    uint64_t* out;            // batch x (n_out + 1)
    uint64_t batch;
    uint32_t n_in, n_out, digits;
    uint64_t corr;
    uint32_t dshift[8];
    uint64_t dmask[8];
    uint64_t ddelta[8];
};

constexpr int kLweKsRows = 16;     // ciphertexts per block
constexpr int kLweKsCols = 128;    // output words per block (= threads)
constexpr int kLweKsChunk = 32;    // input coefficients staged per round

__global__ void __launch_bounds__(kLweKsCols) lwe_ks_kernel(const LweKsParams prm) {
    __shared__ uint64_t dig[kLweKsRows][kLweKsChunk * 8];
    const int t = threadIdx.x;
    const uint64_t row0 = (uint64_t)blockIdx.y * kLweKsRows;
    const uint32_t col = blockIdx.x * kLweKsCols + t;
    const uint32_t width = prm.n_out + 1;
    const uint32_t L = prm.digits;
    uint64_t acc[kLweKsRows];
#pragma unroll
    for (int r = 0; r < kLweKsRows; ++r) acc[r] = 0;
    for (uint32_t i0 = 0; i0 < prm.n_in; i0 += kLweKsChunk) {
        const uint32_t ni = min((uint32_t)kLweKsChunk, prm.n_in - i0);
        __syncthreads();
        for (uint32_t e = t; e < kLweKsRows * ni; e += kLweKsCols) {
            const uint32_t r = e / ni, ii = e % ni;
            uint64_t x = 0;
            if (row0 + r < prm.batch) x = gl_add(prm.in[(row0 + r) * (prm.n_in + 1) + i0 + ii], prm.corr);
            for (uint32_t j = 0; j < L; ++j)
                dig[r][ii * L + j] = row0 + r < prm.batch ? gl_sub((x >> prm.dshift[j]) & prm.dmask[j], prm.ddelta[j]) : 0;
        }
        __syncthreads();
        if (col < width) {
            for (uint32_t ij = 0; ij < ni * L; ++ij) {
                const uint64_t kv = __ldg(prm.ksk + (uint64_t)(i0 * L + ij) * width + col);
#pragma unroll
                for (int r = 0; r < kLweKsRows; ++r) acc[r] = gl_fma_lazy(acc[r], dig[r][ij], kv);
            }
        }
    }
    if (col < width) {
#pragma unroll
        for (int r = 0; r < kLweKsRows; ++r) {
            const uint64_t row = row0 + r;
            if (row >= prm.batch) break;
            uint64_t* o = prm.out + row * width;
            const uint64_t base = col == prm.n_out ? prm.in[row * (prm.n_in + 1) + prm.n_in] : o[col];
            o[col] = gl_sub(base, gl_canon(acc[r]));
        }
    }
}

}  // namespace tp
