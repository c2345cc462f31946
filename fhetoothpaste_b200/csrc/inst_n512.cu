// Kernel instantiations for N = 512 (compiled as a separate unit so the
// ring sizes build in parallel).
#include "br_kernels.cuh"
#include "br_pair_kernel.cuh"
#include "dispatch.h"
#include "ks_kernels.cuh"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_9(int variant, int loge, int dl, bool r4) {
    if (r4) return nullptr;  // fused radix-4 rotation kernels are built for N = 1024 .. 4096
    if (dl == 3 || dl == 4) {  // digit-staged multiply-accumulate, 4 coefficients per thread
        if (loge != 2) return nullptr;
        switch (variant) {
            case kCggiBinary: return dl == 3 ? (const void*)br_kernel<9, kCggiBinary, 2, 3>
                                             : (const void*)br_kernel<9, kCggiBinary, 2, 4>;
            case kCggiTernary: return dl == 3 ? (const void*)br_kernel<9, kCggiTernary, 2, 3>
                                              : (const void*)br_kernel<9, kCggiTernary, 2, 4>;
            default: return dl == 3 ? (const void*)br_kernel<9, kBmmpBinary, 2, 3>
                                    : (const void*)br_kernel<9, kBmmpBinary, 2, 4>;
        }
    }
    if (dl != 0) return nullptr;
    if (loge == 2) {
        switch (variant) {
            case kCggiBinary: return (const void*)br_kernel<9, kCggiBinary, 2>;
            case kCggiTernary: return (const void*)br_kernel<9, kCggiTernary, 2>;
            default: return (const void*)br_kernel<9, kBmmpBinary, 2>;
        }
    }
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<9, kCggiBinary, 3>;
        case kCggiTernary: return (const void*)br_kernel<9, kCggiTernary, 3>;
        default: return (const void*)br_kernel<9, kBmmpBinary, 3>;
    }
}

const void* br_pair_kernel_ptr_9(int variant, int split) { return br_split_kernel_ptr<9>(variant, split); }

const void* ntt_kernel_ptr_9(bool forward) {
    return forward ? (const void*)ntt_batch_kernel<9, true> : (const void*)ntt_batch_kernel<9, false>;
}

const void* ks_kernel_ptr_9(int mode, int loge) {
    if (loge == 2) {
        switch (mode) {
            case kKsRlwe: return (const void*)ks_kernel<9, kKsRlwe, 2>;
            case kKsAuto: return (const void*)ks_kernel<9, kKsAuto, 2>;
            case kKsMerge: return (const void*)ks_kernel<9, kKsMerge, 2>;
            case kKsTrace: return (const void*)ks_kernel<9, kKsTrace, 2>;
            default: return (const void*)ks_kernel<9, kKsSplit, 2>;
        }
    }
    switch (mode) {
        case kKsRlwe: return (const void*)ks_kernel<9, kKsRlwe, 3>;
        case kKsAuto: return (const void*)ks_kernel<9, kKsAuto, 3>;
        case kKsMerge: return (const void*)ks_kernel<9, kKsMerge, 3>;
        case kKsTrace: return (const void*)ks_kernel<9, kKsTrace, 3>;
        default: return (const void*)ks_kernel<9, kKsSplit, 3>;
    }
}

}  // namespace tp
