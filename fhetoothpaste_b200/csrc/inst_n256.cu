// Kernel instantiations for N = 256 (compiled as a separate unit so the
// ring sizes build in parallel).
#include "br_kernels.cuh"
#include "dispatch.h"
#include "misc_kernels.cuh"

namespace tp {

const void* br_kernel_ptr_8(int variant) {
    switch (variant) {
        case kCggiBinary: return (const void*)br_kernel<8, kCggiBinary>;
        case kCggiTernary: return (const void*)br_kernel<8, kCggiTernary>;
        default: return (const void*)br_kernel<8, kBmmpBinary>;
    }
}

const void* ntt_kernel_ptr_8(bool forward) {
    return forward ? (const void*)ntt_batch_kernel<8, true> : (const void*)ntt_batch_kernel<8, false>;
}

}  // namespace tp
