// Kernel instantiations for N = 4096 (compiled as a separate unit so the
// ring sizes build in parallel).
#include "br_kernels.cuh"
#include "br_pair_kernel.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_12(int variant, int loge, int dl, bool r4) {
    if (r4) {  // fused radix-4 passes, 4 coefficients per thread
        if (loge != 2 || dl != 0) return nullptr;
        if (variant == kCggiBinary) return (const void*)br_kernel<12, kCggiBinary, 2, 0, 0, true>;
        if (variant == kCggiTernary) return (const void*)br_kernel<12, kCggiTernary, 2, 0, 0, true>;
        if (variant == kBmmpBinary) return (const void*)br_kernel<12, kBmmpBinary, 2, 0, 0, true>;
        return nullptr;
    }
    if (dl != 0) return nullptr;  // the digit stage does not fit one SM's shared memory at this N
    if (loge == 2) {
        switch (variant) {
            case kCggiBinary: return (const void*)br_kernel<12, kCggiBinary, 2>;
            case kCggiTernary: return (const void*)br_kernel<12, kCggiTernary, 2>;
            default: return (const void*)br_kernel<12, kBmmpBinary, 2>;
        }
    }
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<12, kCggiBinary, 3>;
        case kCggiTernary: return (const void*)br_kernel<12, kCggiTernary, 3>;
        default: return (const void*)br_kernel<12, kBmmpBinary, 3>;
    }
}

const void* br_pair_kernel_ptr_12(int variant, int split) { return br_split_kernel_ptr<12>(variant, split); }

const void* ntt_kernel_ptr_12(bool forward) {
    return forward ? (const void*)ntt_batch_kernel<12, true> : (const void*)ntt_batch_kernel<12, false>;
}

const void* ks_kernel_ptr_12(int mode, int loge) {
    if (loge == 2) {
        switch (mode) {
            case kKsRlwe: return (const void*)ks_kernel<12, kKsRlwe, 2>;
            case kKsAuto: return (const void*)ks_kernel<12, kKsAuto, 2>;
            case kKsMerge: return (const void*)ks_kernel<12, kKsMerge, 2>;
            case kKsTrace: return (const void*)ks_kernel<12, kKsTrace, 2>;
            default: return (const void*)ks_kernel<12, kKsSplit, 2>;
        }
    }
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<12, kKsRlwe, 3>;
        case kKsAuto: return (const void*)ks_kernel<12, kKsAuto, 3>;
        case kKsMerge: return (const void*)ks_kernel<12, kKsMerge, 3>;
        case kKsTrace: return (const void*)ks_kernel<12, kKsTrace, 3>;
        default: return (const void*)ks_kernel<12, kKsSplit, 3>;
    }
}

}  // namespace tp
