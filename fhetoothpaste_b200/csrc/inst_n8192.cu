// Kernel instantiations for N = 8192: one rotation per cluster of 4 CTAs
// (cluster_ntt.cuh), 4 coefficients per thread, for the rotation and the key-switching
// modes; compiled as a separate unit so
// the ring sizes build in parallel.
#include "br_kernels.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

static_assert(br_cluster_logs(13) == 2, "cluster size of this unit");

const void* br_kernel_ptr_13(int variant, int loge, int dl, bool r4) {
    if (r4) return nullptr;  // fused radix-4 rotation kernels are built for N = 1024 .. 4096
    if (loge != 2 || (dl != 0 && dl != 3 && dl != 4)) return nullptr;
    switch (variant) {
        case kCggiBinary:
            return dl == 0 ? (const void*)br_kernel<13, kCggiBinary, 2, 0, 2>
                           : (dl == 3 ? (const void*)br_kernel<13, kCggiBinary, 2, 3, 2>
                                      : (const void*)br_kernel<13, kCggiBinary, 2, 4, 2>);
        case kCggiTernary:
            return dl == 0 ? (const void*)br_kernel<13, kCggiTernary, 2, 0, 2>
                           : (dl == 3 ? (const void*)br_kernel<13, kCggiTernary, 2, 3, 2>
                                      : (const void*)br_kernel<13, kCggiTernary, 2, 4, 2>);
        default:
            return dl == 0 ? (const void*)br_kernel<13, kBmmpBinary, 2, 0, 2>
                           : (dl == 3 ? (const void*)br_kernel<13, kBmmpBinary, 2, 3, 2>
                                      : (const void*)br_kernel<13, kBmmpBinary, 2, 4, 2>);
    }
}

const void* ks_kernel_ptr_13(int mode, int loge) {
    if (loge != 2) return nullptr;  // clusters run with 4 coefficients per thread
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<13, kKsRlwe, 2, 2>;
        case kKsAuto: return (const void*)ks_kernel<13, kKsAuto, 2, 2>;
        case kKsMerge: return (const void*)ks_kernel<13, kKsMerge, 2, 2>;
        case kKsTrace: return (const void*)ks_kernel<13, kKsTrace, 2, 2>;
        default: return (const void*)ks_kernel<13, kKsSplit, 2, 2>;
    }
}

const void* ntt_kernel_ptr_13(bool forward) {
    return forward ? (const void*)ntt_cluster_kernel<13, true, 2>
                   : (const void*)ntt_cluster_kernel<13, false, 2>;
}

}  // namespace tp
