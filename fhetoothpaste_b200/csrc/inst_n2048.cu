// Kernel instantiations for N = 2048 (compiled as a separate unit so the
// ring sizes build in parallel).
#include "br_kernels.cuh"
#include "br_pair_kernel.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_11(int variant, int loge, int dl, bool r4) {
    if (r4) {  // fused radix-4 passes, 4 coefficients per thread
        if (loge != 2 || !(dl == 0 || dl == 3 || dl == 4)) return nullptr;
        if (variant == kCggiBinary)
            return dl == 0 ? (const void*)br_kernel<11, kCggiBinary, 2, 0, 0, true>
                           : (dl == 3 ? (const void*)br_kernel<11, kCggiBinary, 2, 3, 0, true>
                                      : (const void*)br_kernel<11, kCggiBinary, 2, 4, 0, true>);
        if (variant == kCggiTernary)
            return dl == 0 ? (const void*)br_kernel<11, kCggiTernary, 2, 0, 0, true>
                           : (dl == 3 ? (const void*)br_kernel<11, kCggiTernary, 2, 3, 0, true>
                                      : (const void*)br_kernel<11, kCggiTernary, 2, 4, 0, true>);
        if (variant == kBmmpBinary)
            return dl == 0 ? (const void*)br_kernel<11, kBmmpBinary, 2, 0, 0, true>
                           : (dl == 3 ? (const void*)br_kernel<11, kBmmpBinary, 2, 3, 0, true>
                                      : (const void*)br_kernel<11, kBmmpBinary, 2, 4, 0, true>);
        return nullptr;
    }
    if (dl == 3 || dl == 4) {  // digit-staged multiply-accumulate, 4 coefficients per thread
        if (loge != 2) return nullptr;
        switch (variant) {
            case kCggiBinary: return dl == 3 ? (const void*)br_kernel<11, kCggiBinary, 2, 3>
                                             : (const void*)br_kernel<11, kCggiBinary, 2, 4>;
            case kCggiTernary: return dl == 3 ? (const void*)br_kernel<11, kCggiTernary, 2, 3>
                                              : (const void*)br_kernel<11, kCggiTernary, 2, 4>;
            default: return dl == 3 ? (const void*)br_kernel<11, kBmmpBinary, 2, 3>
                                    : (const void*)br_kernel<11, kBmmpBinary, 2, 4>;
        }
    }
    if (dl != 0) return nullptr;
    if (loge == 2) {
        switch (variant) {
            case kCggiBinary: return (const void*)br_kernel<11, kCggiBinary, 2>;
            case kCggiTernary: return (const void*)br_kernel<11, kCggiTernary, 2>;
            default: return (const void*)br_kernel<11, kBmmpBinary, 2>;
        }
    }
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<11, kCggiBinary, 3>;
        case kCggiTernary: return (const void*)br_kernel<11, kCggiTernary, 3>;
        default: return (const void*)br_kernel<11, kBmmpBinary, 3>;
    }
}

const void* br_pair_kernel_ptr_11(int variant, int split) { return br_split_kernel_ptr<11>(variant, split); }

const void* ntt_kernel_ptr_11(bool forward) {
    return forward ? (const void*)ntt_batch_kernel<11, true> : (const void*)ntt_batch_kernel<11, false>;
}

const void* ks_kernel_ptr_11(int mode, int loge) {
    if (loge == 2) {
        switch (mode) {
            case kKsRlwe: return (const void*)ks_kernel<11, kKsRlwe, 2>;
            case kKsAuto: return (const void*)ks_kernel<11, kKsAuto, 2>;
            case kKsMerge: return (const void*)ks_kernel<11, kKsMerge, 2>;
            case kKsTrace: return (const void*)ks_kernel<11, kKsTrace, 2>;
            default: return (const void*)ks_kernel<11, kKsSplit, 2>;
        }
    }
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<11, kKsRlwe, 3>;
        case kKsAuto: return (const void*)ks_kernel<11, kKsAuto, 3>;
        case kKsMerge: return (const void*)ks_kernel<11, kKsMerge, 3>;
        case kKsTrace: return (const void*)ks_kernel<11, kKsTrace, 3>;
        default: return (const void*)ks_kernel<11, kKsSplit, 3>;
    }
}

}  // namespace tp
