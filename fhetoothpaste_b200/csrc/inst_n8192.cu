// Kernel instantiations for N = 8192: one rotation per cluster of 2 CTAs of 4096
// coefficients each (cluster_ntt.cuh; 1024 threads per CTA, 4 coefficients per
// thread), for the rotation (row-by-row multiply-accumulate: the digit stage does not
// fit beside 4096 coefficients) and the key-switching modes; compiled as a separate
// unit so the ring sizes build in parallel.
#include "br_kernels.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

static_assert(br_cluster_logs(13) == 1, "cluster size of this unit");

const void* br_kernel_ptr_13(int variant, int loge, int dl, bool r4) {
    if (r4 || loge != 2 || dl != 0) return nullptr;
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<13, kCggiBinary, 2, 0, 1>;
        case kCggiTernary: return (const void*)br_kernel<13, kCggiTernary, 2, 0, 1>;
        default: return (const void*)br_kernel<13, kBmmpBinary, 2, 0, 1>;
    }
}

const void* ks_kernel_ptr_13(int mode, int loge) {
    if (loge != 2) return nullptr;  // clusters run with 4 coefficients per thread
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<13, kKsRlwe, 2, 1>;
        case kKsAuto: return (const void*)ks_kernel<13, kKsAuto, 2, 1>;
        case kKsMerge: return (const void*)ks_kernel<13, kKsMerge, 2, 1>;
        case kKsTrace: return (const void*)ks_kernel<13, kKsTrace, 2, 1>;
        default: return (const void*)ks_kernel<13, kKsSplit, 2, 1>;
    }
}

const void* ntt_kernel_ptr_13(bool forward) {
    return forward ? (const void*)ntt_cluster_kernel<13, true, 1>
                   : (const void*)ntt_cluster_kernel<13, false, 1>;
}

}  // namespace tp
