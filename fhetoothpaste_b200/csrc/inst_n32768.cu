// Kernel instantiations for N = 32768: one rotation per cluster of 16 CTAs
// (cluster_ntt.cuh), 4 coefficients per thread, for the rotation and the key-switching
// modes; compiled as a separate unit so
// the ring sizes build in parallel.
#include "br_kernels.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_15(int variant, int loge, int dl, bool r4) {
    if (r4) return nullptr;  // fused radix-4 rotation kernels are built for N = 1024 .. 4096
    if (loge != 2 || (dl != 0 && dl != 3 && dl != 4)) return nullptr;
    switch (variant) {
        case kCggiBinary:
            return dl == 0 ? (const void*)br_kernel<15, kCggiBinary, 2, 0, 4>
                           : (dl == 3 ? (const void*)br_kernel<15, kCggiBinary, 2, 3, 4>
                                      : (const void*)br_kernel<15, kCggiBinary, 2, 4, 4>);
        case kCggiTernary:
            return dl == 0 ? (const void*)br_kernel<15, kCggiTernary, 2, 0, 4>
                           : (dl == 3 ? (const void*)br_kernel<15, kCggiTernary, 2, 3, 4>
                                      : (const void*)br_kernel<15, kCggiTernary, 2, 4, 4>);
        default:
            return dl == 0 ? (const void*)br_kernel<15, kBmmpBinary, 2, 0, 4>
                           : (dl == 3 ? (const void*)br_kernel<15, kBmmpBinary, 2, 3, 4>
                                      : (const void*)br_kernel<15, kBmmpBinary, 2, 4, 4>);
    }
}

const void* ks_kernel_ptr_15(int mode, int loge) {
    if (loge != 2) return nullptr;  // clusters run with 4 coefficients per thread
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<15, kKsRlwe, 2, 4>;
        case kKsAuto: return (const void*)ks_kernel<15, kKsAuto, 2, 4>;
        case kKsMerge: return (const void*)ks_kernel<15, kKsMerge, 2, 4>;
        case kKsTrace: return (const void*)ks_kernel<15, kKsTrace, 2, 4>;
        default: return (const void*)ks_kernel<15, kKsSplit, 2, 4>;
    }
}

const void* ntt_kernel_ptr_15(bool forward) {
    return forward ? (const void*)ntt_cluster_kernel<15, true, 4>
                   : (const void*)ntt_cluster_kernel<15, false, 4>;
}

}  // namespace tp
