// Packing set-up and LWE -> LWE key switching (launched by the C ABI unit only).
#pragma once

#include "gl_arith.cuh"

namespace tp {

// The two consecutive words k, k + 1 (k even) of a packing leaf, L0Setup
// (lwe_to_rlwe_packing.cpp:238-251) of the LWE at `lwe`: A = (a0, -a_{N-1}, ..,
// -a_1) and B = (b, 0, .., 0), times N^-1.
__device__ __forceinline__ ulonglong2 pack_l0_pair(const uint64_t* __restrict__ lwe, uint64_t k, uint64_t N,
                                                   uint64_t n_inv) {
    uint64_t v0 = 0, v1 = 0;
    if (k == 0) v0 = lwe[0];
    else if (k < N) v0 = gl_neg(lwe[N - k]);
    else if (k == N) v0 = lwe[N];
    if (k + 1 < N) v1 = gl_neg(lwe[N - k - 1]);
    return make_ulonglong2(gl_mul(v0, n_inv), gl_mul(v1, n_inv));
}

// L0Setup of every packing input, written in the packing tree's element order:
// node c of pack p takes input (len-1) ^ brv_{log len}(c) (lwe_to_rlwe_packing.cpp:143).
// Each thread writes 16-byte word pairs; N and len are powers of two, so the
// indices are shifts and masks.
__global__ void pack_l0_kernel(uint64_t* __restrict__ nodes, const uint64_t* __restrict__ in, uint64_t packs,
                               uint32_t len, uint32_t log_len, uint32_t logn, uint64_t n_inv) {
    const uint64_t N = 1ull << logn;
    const uint64_t pairs = (packs * len) << logn;  // 2N words per node
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < pairs;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = (q << 1) & (2 * N - 1);
        const uint64_t node = q >> logn;
        const uint32_t c = (uint32_t)(node & (len - 1));
        const uint64_t p = node >> log_len;
        const uint32_t src = (len - 1) ^ (log_len ? (__brev(c) >> (32 - log_len)) : 0u);
        reinterpret_cast<ulonglong2*>(nodes)[q] = pack_l0_pair(in + (p * len + src) * (N + 1), k, N, n_inv);
    }
}

// L0Setup of the inputs of a consecutive packing (lwe_to_rlwe_packing.cpp:260-393):
// node s of pack p is the tree leaf whose input index is src[s] < len.
__global__ void pack_l0_idx_kernel(uint64_t* __restrict__ nodes, const uint64_t* __restrict__ in,
                                   const uint32_t* __restrict__ src, uint64_t packs, uint32_t count, uint32_t len,
                                   uint32_t logn, uint64_t n_inv) {
    const uint64_t N = 1ull << logn;
    const uint64_t pairs = (packs * count) << logn;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < pairs;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = (q << 1) & (2 * N - 1);
        const uint64_t node = q >> logn;
        const uint64_t p = node / count, c = node - p * count;
        reinterpret_cast<ulonglong2*>(nodes)[q] = pack_l0_pair(in + (p * len + src[c]) * (N + 1), k, N, n_inv);
    }
}

// out = in * factor (mod p), element-wise (out may equal in).
__global__ void scale_kernel(uint64_t* __restrict__ out, const uint64_t* __restrict__ in, uint64_t count,
                             uint64_t factor) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < count;
         w += (uint64_t)gridDim.x * blockDim.x)
        out[w] = gl_mul(in[w], factor);
}

// ---------------------------------------------------------------------------
// LWE -> LWE key switching (lib/src/operators/lwe_conversion.cpp:205-239), q = p:
//   out[n_out] = in[n_in]; out[k] -= sum_{i,j} digit_j(in[i]) * ksk[i][j][k]
// A block owns 16 ciphertexts x 128 output words; digits of a chunk of input
// coefficients are staged in shared memory, key words stream through L1/L2.
// ---------------------------------------------------------------------------
struct LweKsParams {
    const uint64_t* ksk;      // reference layout: [i][j][n_out + 1]
    const uint64_t* in;       // batch x (n_in + 1); or, with rlwe_in, batch x 2N RLWEs (coefficients)
    uint64_t* out;            // batch x (n_out + 1)
    uint64_t batch;
    uint32_t n_in, n_out, digits;
    uint32_t rlwe_in;         // 1: input row = SampleExtract(index 0) of an RLWE with N = n_in
    uint32_t ms_log2;         // k > 0: write floor(out * 2^k / p) into a fresh output (PBS epilogue)
    const uint64_t* cterm;    // per output word: sum_j ddelta[j] * sum_i ksk[i][j][col] mod p
    uint64_t corr;
    uint32_t dshift[8];
    uint64_t dmask[8];
    uint64_t ddelta[8];
};

constexpr int kLweKsRows = 16;     // ciphertexts per block
constexpr int kLweKsCols = 128;    // output words per block (= threads)
constexpr int kLweKsChunk = 32;    // input coefficients staged per round

// floor(v 2^k / p) for 1 <= k <= 32: v 2^k = hi 2^64 + lo and v 2^k - hi p =
// lo + hi (2^32 - 1) lies in [0, 2p), so the quotient is hi or hi + 1. This is
// also the reference's long-double FLOOR switch (modulus_switching.cpp:43-48):
// with p = 1 (mod 2^k) every quotient q is at least q/p away from the integer
// above it, more than half a 64-bit-mantissa ulp, so rounding the quotient to
// long double never carries it over an integer.
__device__ __forceinline__ uint64_t ms_floor_pow2(uint64_t v, uint32_t k) {
    const uint64_t hi = v >> (64 - k), lo = v << k;
    const uint64_t m = (hi << 32) - hi;
    const uint64_t r = lo + m;
    return hi + ((r < lo || r >= kP) ? 1u : 0u);
}

// ModulusSwitch from p to 2^k, 1 <= k <= 32, of any 64-bit word, with the
// reference's result (modulus_switching.cpp:36-93): x = RN64(v 2^k / p) in x87
// long double (64-bit significand, ties to even), then floorl / ceill / roundl,
// then minus 2^k where that reaches 2^k. Computed exactly with integers: with
// v 2^k = a p + r (0 <= r < p, a <= 2^k) and b the bit length of a, x lies in a's
// binade, so x = a + F 2^-s with s = 64 - b and F = RN(r 2^s / p) (no ties: p is
// odd and prime). Then
//   FLOOR: a (F never reaches 2^s: p = 1 mod 2^k keeps p - r >= a + 1);
//   CEIL:  a when r = 0 or F = 0 (a >= 1 and r <= p >> (s+1)), else a + 1;
//   ROUND: a + 1 when F >= 2^(s-1), i.e. r >= ceil((p - (p >> s)) / 2); for a = 0
//          the binade below 1/2 has half-ulp 2^-66 and the test is 2r >= p (s = 65).
// type: 0 ROUND, 1 FLOOR, 2 CEIL.
__device__ __forceinline__ uint64_t ms_pow2(uint64_t v, uint32_t k, int type) {
    const uint64_t hi = v >> (64 - k), lo = v << k;
    const uint64_t t = lo + ((hi << 32) - hi);  // lo + hi (2^32 - 1), 65 bits
    const bool carry = t < lo;
    uint64_t a = hi, r = t;
    if (carry || t >= kP) {
        a = hi + 1;
        r = t - kP;  // mod 2^64: the 65-bit t minus p, below p
    }
    uint64_t res = a;
    if (r != 0 && type != 1) {
        const int b = a ? 64 - __clzll((long long)a) : 0;
        const int sh = a ? 64 - b : 65;
        if (type == 2) {
            const uint64_t lim = sh + 1 >= 64 ? 0 : (kP >> (sh + 1));
            res = (a && r <= lim) ? a : a + 1;
        } else {
            const uint64_t tail = sh >= 64 ? 0 : (kP >> sh);
            res = r >= (kP - tail + 1) / 2 ? a + 1 : a;
        }
    }
    const uint64_t top = 1ull << k;
    return res >= top ? res - top : res;
}

__global__ void ms_pow2_kernel(uint64_t* __restrict__ vec, uint64_t count, uint32_t k, int type) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
        vec[i] = ms_pow2(vec[i], k, type);
}

// Input word i (< n_in) and the body word of ciphertext row `row`: an LWE row, or
// SampleExtract at index 0 of an RLWE [A | B] (a_0 = A[0], a_i = -A[N - i], b = B[0]).
__device__ __forceinline__ uint64_t lwe_ks_in_word(const LweKsParams& prm, uint64_t row, uint32_t i) {
    if (!prm.rlwe_in) return prm.in[row * (prm.n_in + 1) + i];
    const uint64_t* r = prm.in + row * 2ull * prm.n_in;
    return i == 0 ? r[0] : gl_neg(r[prm.n_in - i]);
}
__device__ __forceinline__ uint64_t lwe_ks_in_body(const LweKsParams& prm, uint64_t row) {
    return prm.rlwe_in ? prm.in[row * 2ull * prm.n_in + prm.n_in] : prm.in[row * (prm.n_in + 1) + prm.n_in];
}

// a (128-bit, four 32-bit limbs) += raw * k exactly, raw < 2^32: two 32x64-bit
// partial products folded into the limbs' carry chains.
__device__ __forceinline__ void mac_raw(uint32_t (&a)[4], uint32_t raw, uint64_t k) {
    asm("mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
        "madc.hi.cc.u32 %1, %4, %5, %1;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "mad.lo.cc.u32 %1, %4, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %6, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3])
        : "r"(raw), "r"(lo32(k)), "r"(hi32(k)));
}

// The signed digits are d_ij = raw_ij - ddelta[j] with raw_ij in [0, 2^beta), so
//   sum_ij d_ij k_ij = sum_ij raw_ij k_ij - sum_j ddelta[j] (sum_i k_ij)   (mod p).
// The kernel accumulates the first sum exactly in 128 bits (no reduction per
// term: n_in * l terms below 2^94 each) and takes off the second, which depends
// only on the key and the output word (cterm, computed at key upload).
__global__ void __launch_bounds__(kLweKsCols) lwe_ks_kernel(const LweKsParams prm) {
    __shared__ uint32_t dig[kLweKsRows][kLweKsChunk * 8];
    const int t = threadIdx.x;
    const uint64_t row0 = (uint64_t)blockIdx.y * kLweKsRows;
    const uint32_t col = blockIdx.x * kLweKsCols + t;
    const uint32_t width = prm.n_out + 1;
    const uint32_t L = prm.digits;
    uint32_t acc[kLweKsRows][4];
#pragma unroll
    for (int r = 0; r < kLweKsRows; ++r)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[r][w] = 0;
    for (uint32_t i0 = 0; i0 < prm.n_in; i0 += kLweKsChunk) {
        const uint32_t ni = min((uint32_t)kLweKsChunk, prm.n_in - i0);
        __syncthreads();
        for (uint32_t e = t; e < kLweKsRows * ni; e += kLweKsCols) {
            const uint32_t r = e / ni, ii = e % ni;
            uint64_t x = 0;
            if (row0 + r < prm.batch) x = gl_add(lwe_ks_in_word(prm, row0 + r, i0 + ii), prm.corr);
            for (uint32_t j = 0; j < L; ++j)
                dig[r][ii * L + j] = row0 + r < prm.batch ? (uint32_t)((x >> prm.dshift[j]) & prm.dmask[j]) : 0u;
        }
        __syncthreads();
        if (col < width) {
            for (uint32_t ij = 0; ij < ni * L; ++ij) {
                const uint64_t kv = __ldg(prm.ksk + (uint64_t)(i0 * L + ij) * width + col);
#pragma unroll
                for (int r = 0; r < kLweKsRows; ++r) mac_raw(acc[r], dig[r][ij], kv);
            }
        }
    }
    if (col < width) {
        const uint64_t ct = prm.cterm[col];
#pragma unroll
        for (int r = 0; r < kLweKsRows; ++r) {
            const uint64_t row = row0 + r;
            if (row >= prm.batch) break;
            const uint64_t sum = gl_sub(gl_reduce128(acc[r][0], acc[r][1], acc[r][2], acc[r][3]), ct);
            uint64_t* o = prm.out + row * width;
            if (prm.ms_log2) {
                const uint64_t base = col == prm.n_out ? lwe_ks_in_body(prm, row) : 0;
                o[col] = ms_floor_pow2(gl_sub(base, sum), prm.ms_log2);
            } else {
                const uint64_t base = col == prm.n_out ? lwe_ks_in_body(prm, row) : o[col];
                o[col] = gl_sub(base, sum);
            }
        }
    }
}

// cterm[col] = sum_j ddelta[j] * (sum_i ksk[i][j][col]) mod p. Block (32, Y): threadIdx.x
// picks the column of a 32-column tile (coalesced key reads), threadIdx.y a slice of the
// input index i; each thread forms sum_j ddelta[j] * (its slice's sum) and the Y partials
// are added in shared memory (the constant is linear in the sums, so the words equal a
// serial sum's).
constexpr int kCtermSlices = 16;
__global__ void __launch_bounds__(32 * kCtermSlices) lwe_ks_cterm_kernel(uint64_t* __restrict__ cterm,
                                                                         const LweKsParams prm) {
    __shared__ uint64_t part[kCtermSlices][32];
    const uint32_t width = prm.n_out + 1;
    const uint32_t col = blockIdx.x * 32 + threadIdx.x;
    uint64_t total = 0;
    if (col < width) {
        for (uint32_t j = 0; j < prm.digits; ++j) {
            uint64_t s = 0;
            for (uint32_t i = threadIdx.y; i < prm.n_in; i += kCtermSlices)
                s = gl_add(s, gl_canon(prm.ksk[((uint64_t)i * prm.digits + j) * width + col]));
            total = gl_add(total, gl_mul(s, gl_canon(prm.ddelta[j])));
        }
    }
    part[threadIdx.y][threadIdx.x] = total;
    __syncthreads();
    if (threadIdx.y == 0 && col < width) {
        uint64_t sum = part[0][threadIdx.x];
        for (int y = 1; y < kCtermSlices; ++y) sum = gl_add(sum, part[y][threadIdx.x]);
        cterm[col] = sum;
    }
}

}  // namespace tp
