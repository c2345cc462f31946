// Kernel instantiations for N = 32768: one rotation per cluster of 8 CTAs of 4096
// coefficients each (cluster_ntt.cuh; 1024 threads per CTA, 4 coefficients per
// thread), for the rotation (row-by-row multiply-accumulate: the digit stage does not
// fit beside 4096 coefficients) and the key-switching modes; compiled as a separate
// unit so the ring sizes build in parallel.
#include "br_kernels.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

static_assert(br_cluster_logs(15) == 3, "cluster size of this unit");

const void* br_kernel_ptr_15(int variant, int loge, int dl, bool r4) {
    if (r4 || loge != 2 || dl != 0) return nullptr;
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<15, kCggiBinary, 2, 0, 3>;
        case kCggiTernary: return (const void*)br_kernel<15, kCggiTernary, 2, 0, 3>;
        default: return (const void*)br_kernel<15, kBmmpBinary, 2, 0, 3>;
    }
}

const void* ks_kernel_ptr_15(int mode, int loge) {
    if (loge != 2) return nullptr;  // clusters run with 4 coefficients per thread
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<15, kKsRlwe, 2, 3>;
        case kKsAuto: return (const void*)ks_kernel<15, kKsAuto, 2, 3>;
        case kKsMerge: return (const void*)ks_kernel<15, kKsMerge, 2, 3>;
        case kKsTrace: return (const void*)ks_kernel<15, kKsTrace, 2, 3>;
        default: return (const void*)ks_kernel<15, kKsSplit, 2, 3>;
    }
}

const void* ntt_kernel_ptr_15(bool forward) {
    return forward ? (const void*)ntt_cluster_kernel<15, true, 3>
                   : (const void*)ntt_cluster_kernel<15, false, 3>;
}

}  // namespace tp
