// Kernel instantiations for N = 512 (compiled as a separate unit so the
// ring sizes build in parallel).
#include "br_kernels.cuh"
#include "dispatch.h"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_9(int variant) {
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<9, kCggiBinary>;
        case kCggiTernary: return (const void*)br_kernel<9, kCggiTernary>;
        default: return (const void*)br_kernel<9, kBmmpBinary>;
    }
}

const void* ntt_kernel_ptr_9(bool forward) {
    return forward ? (const void*)ntt_batch_kernel<9, true> : (const void*)ntt_batch_kernel<9, false>;
}

}  // namespace tp
