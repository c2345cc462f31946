// Element-wise kernels launched by the C ABI unit only (key re-layout,
// SampleExtract).
#pragma once

#include "gl_arith.cuh"

namespace tp {

// Reference m_brk layout -> device layout, one word per thread.
// Reference: word (it, g, r, h, k) at ((it*G + g)*2l + r)*2N + h*N + k
// (MakeRGSW rows, base_crypto.cpp:90-95; per-iteration RGSW order,
// cggi_blind_rotation.cpp:277,306-309 and bmmp_blind_rotation.cpp:241-258).
__global__ void key_relayout_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t groups,
                                    uint32_t G, uint32_t rows, uint32_t logn) {
    const uint64_t N = 1ull << logn;
    const uint64_t T = N / 8;
    const uint64_t per_group = (uint64_t)G * rows * 2 * N;
    const uint64_t total = groups * per_group;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t it = w / per_group;
        uint64_t rem = w % per_group;
        const uint64_t r = rem / (2 * G * N);
        rem %= 2 * G * N;
        // rem = ((c*4 + jp)*T + t)*2 + e
        const uint64_t e = rem & 1;
        const uint64_t tt = (rem >> 1) % T;
        const uint64_t cj = (rem >> 1) / T;
        const uint64_t jp = cj % 4, c = cj / 4;
        const uint64_t g = c >> 1, h = c & 1;
        const uint64_t k = 8 * tt + 2 * jp + e;
        dst[w] = src[((it * G + g) * rows + r) * 2 * N + h * N + k];
    }
}

// SampleExtract at index 0 (lib/include/static/sample_extraction.h:20-36):
// out[0] = A[0], out[i] = -A[N - i] (i = 1..N-1), out[N] = B[0].
__global__ void sample_extract0_kernel(uint64_t* __restrict__ out, const uint64_t* __restrict__ rlwe, uint64_t batch,
                                       uint32_t N) {
    const uint64_t per = (uint64_t)N + 1;
    const uint64_t total = batch * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / per, i = w % per;
        const uint64_t* src = rlwe + b * 2ull * N;
        uint64_t v;
        if (i == 0) v = src[0];
        else if (i < N) v = gl_neg(src[N - i]);
        else v = src[N];
        out[w] = v;
    }
}

// Element-wise arithmetic check (tp_debug_arith).
__global__ void debug_arith_kernel(int op, uint64_t count, uint64_t* __restrict__ out, const uint64_t* __restrict__ a,
                                   const uint64_t* __restrict__ b, const uint64_t* __restrict__ c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = 0;
        switch (op) {
            case 0: r = gl_add(a[i], b[i]); break;
            case 1: r = gl_sub(a[i], b[i]); break;
            case 2: r = gl_mul(a[i], b[i]); break;
            case 3: r = gl_canon(gl_fma_lazy(c[i], a[i], b[i])); break;
            case 4: r = gl_canon(gl_reduce128_lazy(lo32(a[i]), hi32(a[i]), lo32(b[i]), hi32(b[i]))); break;
            default: r = gl_canon(a[i]); break;
        }
        out[i] = r;
    }
}

// INT32 peak probes: independent chains of 64x64->128 products (mul_wide,
// exactly as the kernels issue them) or of 32-bit mad.lo.
template <int MODE>
__global__ void int_peak_kernel(uint64_t* out, uint64_t seed, int iters) {
    uint64_t a[8], b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        a[j] = (seed * (threadIdx.x + 1 + j) + j) % kP;
        b[j] = (a[j] ^ 0x9E3779B97F4A7C15ull) % kP;
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (MODE == 0) {
                uint32_t r0, r1, r2, r3;
                mul_wide(a[j], b[j], r0, r1, r2, r3);
                a[j] = pack64(r0 ^ r2, r1 ^ r3);
            } else {
                uint32_t x = lo32(a[j]), y = lo32(b[j]), z = hi32(a[j]);
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(y), "r"(z));
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(z) : "r"(y), "r"(x));
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(y), "r"(z));
                asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(z) : "r"(y), "r"(x));
                a[j] = pack64(x, z);
            }
        }
    }
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s ^= a[j] ^ b[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace tp
