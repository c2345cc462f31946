// Standalone batched NTT kernel.
#pragma once

#include "gl_arith.cuh"
#include "ntt_block.cuh"

namespace tp {

// count polynomials, polynomial p at in + p*in_stride / out + p*out_stride;
// block b handles polynomials b, b + gridDim.x, ...
// Shared memory: twiddles (N) + two exchange buffers (2N).
template <int LOGN, bool FORWARD>
__global__ void __launch_bounds__((1 << LOGN) / 8) ntt_batch_kernel(uint64_t* out, const uint64_t* in, uint64_t count,
                                                                     const uint64_t* tw, uint64_t n_inv,
                                                                     uint64_t in_stride, uint64_t out_stride) {
    using SH = NttShape<LOGN>;
    constexpr int N = SH::N;
    constexpr int T = SH::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* tws = smem;
    uint64_t* buf[2] = {smem + N, smem + 2 * N};
    const int t = threadIdx.x;
    for (int i = t; i < N; i += T) tws[i] = tw[i];
    __syncthreads();
    int sel = 0;
    for (uint64_t p = blockIdx.x; p < count; p += gridDim.x) {
        const uint64_t* src = in + p * in_stride;
        uint64_t* dst = out + p * out_stride;
        uint64_t x[8];
        if constexpr (FORWARD) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = src[t + j * T];
            __syncthreads();  // in-place: every read of src before any write of dst
            ntt_forward<LOGN>(x, t, buf[sel], tws);
            sel ^= 1;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                *reinterpret_cast<ulonglong2*>(dst + 8 * t + 2 * c) = make_ulonglong2(x[2 * c], x[2 * c + 1]);
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(src + 8 * t + 2 * c);
                x[2 * c] = v.x;
                x[2 * c + 1] = v.y;
            }
            __syncthreads();
            ntt_backward_unscaled<LOGN>(x, t, buf[sel], tws);
            sel ^= 1;
#pragma unroll
            for (int j = 0; j < 8; ++j) dst[t + j * T] = gl_div_pow2<LOGN>(x[j]);
        }
    }
}

}  // namespace tp
