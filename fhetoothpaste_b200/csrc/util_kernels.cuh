// Element-wise kernels launched by the C ABI unit only (key re-layout,
// SampleExtract).
#pragma once

#include "gl_arith.cuh"

namespace tp {

// Device position of key word (group it, gadget row r, component c = 2g + h,
// slot k) for a rotation kernel with 2^loge coefficients per thread: slot
// k = E*t + 2jp + e sits at ((c*E/2 + jp)*T + t)*2 + e inside the (it, r) row.
// A cluster of 2^logs CTAs (ring sizes above 4096) splits each row into 2^logs
// parts of 2G * NL words, NL = N >> logs: slot k belongs to part k / NL and
// takes the same position inside it as slot k mod NL of an NL-slot row.
__device__ __forceinline__ uint64_t key_device_pos(uint64_t it, uint64_t r, uint64_t c, uint64_t k, uint32_t G,
                                                   uint32_t rows, uint32_t logn, uint32_t loge, uint32_t logs = 0) {
    const uint64_t N = 1ull << logn;
    const uint64_t NL = N >> logs;
    const uint64_t E = 1ull << loge;
    const uint64_t T = NL >> loge;
    const uint64_t part = k / NL, kl = k % NL;
    const uint64_t t = kl >> loge, jp = (kl & (E - 1)) >> 1, e = kl & 1;
    return (it * rows + r) * 2 * G * N + part * (2 * G * NL) + ((c * (E / 2) + jp) * T + t) * 2 + e;
}

// Reference m_brk layout ((it*G + g)*rows + r)*2N + h*N + k  ->  device layout.
// Words k, k + 1 (k even) stay neighbours in the device layout, so each thread
// moves 16-byte pairs; the polynomial index is a shift, the small row and group
// counts 32-bit divisions.
__global__ void key_relayout_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t groups,
                                    uint32_t G, uint32_t rows, uint32_t logn, uint32_t loge, uint32_t logs = 0) {
    const uint64_t N = 1ull << logn;
    const uint64_t pairs = (groups * G * rows) << logn;  // 2N words per (it, g, r)
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < pairs;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t w = q << 1;
        const uint64_t k = w & (N - 1);
        const uint64_t poly = w >> logn;                 // (ig * rows + r) * 2 + h
        const uint32_t h = (uint32_t)(poly & 1);
        const uint32_t rig = (uint32_t)(poly >> 1);      // ig * rows + r
        const uint32_t r = rig % rows, ig = rig / rows;
        const uint32_t g = ig % G, it = ig / G;
        reinterpret_cast<ulonglong2*>(dst)[key_device_pos(it, r, 2 * g + h, k, G, rows, logn, loge, logs) >> 1] =
            reinterpret_cast<const ulonglong2*>(src)[q];
    }
}

// Device layout for one coefficients-per-thread count -> another (same key),
// 16-byte pairs as above.
__global__ void key_retile_kernel(uint64_t* __restrict__ dst, const uint64_t* __restrict__ src, uint64_t groups,
                                  uint32_t G, uint32_t rows, uint32_t logn, uint32_t loge_src, uint32_t loge_dst) {
    const uint64_t N = 1ull << logn;
    const uint64_t pairs = (groups * G * rows) << logn;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < pairs;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t w = q << 1;
        const uint64_t k = w & (N - 1);
        const uint32_t poly = (uint32_t)(w >> logn);     // (it * rows + r) * 2G + c
        const uint32_t c = poly % (2 * G), rit = poly / (2 * G);
        const uint32_t r = rit % rows, it = rit / rows;
        reinterpret_cast<ulonglong2*>(dst)[key_device_pos(it, r, c, k, G, rows, logn, loge_dst) >> 1] =
            reinterpret_cast<const ulonglong2*>(src)[key_device_pos(it, r, c, k, G, rows, logn, loge_src) >> 1];
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
            case 3: r = gl_fma(c[i], a[i], b[i]); break;
            case 4: r = gl_canon(gl_reduce128(lo32(a[i]), hi32(a[i]), lo32(b[i]), hi32(b[i]))); break;
            case 6: r = gl_reduce128(lo32(a[i]), hi32(a[i]), lo32(b[i]), hi32(b[i])); break;
            case 7: r = gl_canon(gl_add_lazy(a[i], b[i])); break;
            case 8: r = gl_canon(gl_add(a[i], b[i])); break;
            case 9: r = gl_canon(gl_sub(a[i], b[i])); break;
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
