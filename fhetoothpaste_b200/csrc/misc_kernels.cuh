// Standalone batched NTT kernels.
#pragma once

#include "cluster_ntt.cuh"
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

// N > 4096: one polynomial per cluster of 2^LOGS CTAs (cluster_ntt.cuh layouts),
// 4 coefficients per thread, NL / 4 threads per CTA. Shared memory: the first NL
// words of the table, two exchange buffers and two receive areas (5 NL words).
// In place is safe: every CTA's reads of a polynomial precede the transform's
// cluster barrier, every write follows it.
template <int LOGN, bool FORWARD, int LOGS>
__global__ void __launch_bounds__((1 << (LOGN - LOGS)) / 4) ntt_cluster_kernel(
    uint64_t* out, const uint64_t* in, uint64_t count, const uint64_t* tw, uint64_t n_inv, uint64_t in_stride,
    uint64_t out_stride) {
    using CS = ClusterShape<LOGN, LOGS>;
    constexpr int NL = CS::NL;
    constexpr int T = CS::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* tws = smem;
    uint64_t* buf[2] = {smem + NL, smem + 2 * NL};
    uint64_t* recv[2] = {smem + 3 * NL, smem + 4 * NL};
    const int t = threadIdx.x;
    const int r = (int)cooperative_groups::this_cluster().block_rank();
    for (int i = t; i < NL; i += T) tws[i] = tw[i];
    cooperative_groups::this_cluster().sync();  // tables written; every CTA running before remote stores
    int sel = 0, rsel = 0;
    for (uint64_t p = blockIdx.x >> LOGS; p < count; p += gridDim.x >> LOGS) {
        const uint64_t* src = in + p * in_stride;
        uint64_t* dst = out + p * out_stride;
        uint64_t x[1][4];
        if constexpr (FORWARD) {
            // coefficient i' S + r, i' = t + j T
#pragma unroll
            for (int j = 0; j < 4; ++j) x[0][j] = src[((uint32_t)(t + j * T) << LOGS) + (uint32_t)r];
            ntt_forward_k<LOGN - LOGS, 1, 2>(x, t, buf[sel], tws);
            sel ^= 1;
            uint64_t* fb = nullptr;
            if constexpr (CS::S > 4) {
                fb = buf[sel];
                sel ^= 1;
            }
            cluster_fwd_tail<LOGN, LOGS, false>(x[0], t, r, recv[rsel], fb, tw);
            rsel ^= 1;
            *reinterpret_cast<ulonglong2*>(dst + r * NL + 4 * t) = make_ulonglong2(x[0][0], x[0][1]);
            *reinterpret_cast<ulonglong2*>(dst + r * NL + 4 * t + 2) = make_ulonglong2(x[0][2], x[0][3]);
        } else {
            const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(src + r * NL + 4 * t);
            const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(src + r * NL + 4 * t + 2);
            x[0][0] = a.x;
            x[0][1] = a.y;
            x[0][2] = b.x;
            x[0][3] = b.y;
            uint64_t* fb = nullptr;
            if constexpr (CS::S > 4) {
                fb = buf[sel];
                sel ^= 1;
            }
            cluster_inv_head<LOGN, LOGS>(x[0], t, r, recv[rsel], fb, tw);
            rsel ^= 1;
            ntt_backward_unscaled_k<LOGN - LOGS, 1, 2>(x, t, buf[sel], tws);
            sel ^= 1;
#pragma unroll
            for (int j = 0; j < 4; ++j) dst[((uint32_t)(t + j * T) << LOGS) + (uint32_t)r] = gl_div_pow2<LOGN>(x[0][j]);
        }
    }
    (void)n_inv;
}

}  // namespace tp
