// Kernel lookup across the per-ring-size compilation units.
#pragma once

namespace tp {

const void* br_kernel_ptr_7(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_7(bool forward);
const void* br_kernel_ptr_8(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_8(bool forward);
const void* br_kernel_ptr_9(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_9(bool forward);
const void* br_kernel_ptr_10(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_10(bool forward);
const void* br_kernel_ptr_11(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_11(bool forward);
const void* br_kernel_ptr_12(int variant, int loge, int dl, bool r4);
const void* br_kernel_ptr_13(int variant, int loge, int dl, bool r4);
const void* br_kernel_ptr_14(int variant, int loge, int dl, bool r4);
const void* br_kernel_ptr_15(int variant, int loge, int dl, bool r4);
const void* br_kernel_ptr_16(int variant, int loge, int dl, bool r4);
const void* ntt_kernel_ptr_12(bool forward);
const void* ntt_kernel_ptr_13(bool forward);  // cluster kernels (ntt_cluster_kernel)
const void* ntt_kernel_ptr_14(bool forward);
const void* ntt_kernel_ptr_15(bool forward);
const void* ntt_kernel_ptr_16(bool forward);
const void* br_pair_kernel_ptr_7(int variant, int split);
const void* br_pair_kernel_ptr_8(int variant, int split);
const void* br_pair_kernel_ptr_9(int variant, int split);
const void* br_pair_kernel_ptr_10(int variant, int split);
const void* br_pair_kernel_ptr_11(int variant, int split);
const void* br_pair_kernel_ptr_12(int variant, int split);
const void* ks_kernel_ptr_7(int mode, int loge);
const void* ks_kernel_ptr_8(int mode, int loge);
const void* ks_kernel_ptr_9(int mode, int loge);
const void* ks_kernel_ptr_10(int mode, int loge);
const void* ks_kernel_ptr_11(int mode, int loge);
const void* ks_kernel_ptr_12(int mode, int loge);
const void* ks_kernel_ptr_13(int mode, int loge);
const void* ks_kernel_ptr_14(int mode, int loge);
const void* ks_kernel_ptr_15(int mode, int loge);
const void* ks_kernel_ptr_16(int mode, int loge);

// One-block rotation kernel (one cluster of CTAs per rotation above N = 4096, N up to 65536);
// dl = 0: multiply-accumulate row by row, dl = 3 or 4: the digit-staged form for
// that digit count; r4: the fused radix-4 passes (N = 1024 .. 4096, 4 coefficients
// per thread) (nullptr where not built).
inline const void* br_kernel_lookup(int logn, int variant, int loge, int dl = 0, bool r4 = false) {
    switch (logn) {
        case 7: return br_kernel_ptr_7(variant, loge, dl, r4);
        case 8: return br_kernel_ptr_8(variant, loge, dl, r4);
        case 9: return br_kernel_ptr_9(variant, loge, dl, r4);
        case 10: return br_kernel_ptr_10(variant, loge, dl, r4);
        case 11: return br_kernel_ptr_11(variant, loge, dl, r4);
        case 12: return br_kernel_ptr_12(variant, loge, dl, r4);
        case 13: return br_kernel_ptr_13(variant, loge, dl, r4);
        case 14: return br_kernel_ptr_14(variant, loge, dl, r4);
        case 15: return br_kernel_ptr_15(variant, loge, dl, r4);
        case 16: return br_kernel_ptr_16(variant, loge, dl, r4);
        default: return nullptr;
    }
}

// Two- or four-CTA (cluster) rotation kernel, 4 coefficients per thread
// (nullptr for four where it does not fit).
inline const void* br_pair_kernel_lookup(int logn, int variant, int split) {
    switch (logn) {
        case 7: return br_pair_kernel_ptr_7(variant, split);
        case 8: return br_pair_kernel_ptr_8(variant, split);
        case 9: return br_pair_kernel_ptr_9(variant, split);
        case 10: return br_pair_kernel_ptr_10(variant, split);
        case 11: return br_pair_kernel_ptr_11(variant, split);
        case 12: return br_pair_kernel_ptr_12(variant, split);
        default: return nullptr;
    }
}

inline const void* ntt_kernel_lookup(int logn, bool forward) {
    switch (logn) {
        case 7: return ntt_kernel_ptr_7(forward);
        case 8: return ntt_kernel_ptr_8(forward);
        case 9: return ntt_kernel_ptr_9(forward);
        case 10: return ntt_kernel_ptr_10(forward);
        case 11: return ntt_kernel_ptr_11(forward);
        case 12: return ntt_kernel_ptr_12(forward);
        case 13: return ntt_kernel_ptr_13(forward);
        case 14: return ntt_kernel_ptr_14(forward);
        case 15: return ntt_kernel_ptr_15(forward);
        case 16: return ntt_kernel_ptr_16(forward);
        default: return nullptr;
    }
}

inline const void* ks_kernel_lookup(int logn, int mode, int loge) {
    switch (logn) {
        case 7: return ks_kernel_ptr_7(mode, loge);
        case 8: return ks_kernel_ptr_8(mode, loge);
        case 9: return ks_kernel_ptr_9(mode, loge);
        case 10: return ks_kernel_ptr_10(mode, loge);
        case 11: return ks_kernel_ptr_11(mode, loge);
        case 12: return ks_kernel_ptr_12(mode, loge);
        case 13: return ks_kernel_ptr_13(mode, loge);
        case 14: return ks_kernel_ptr_14(mode, loge);
        case 15: return ks_kernel_ptr_15(mode, loge);
        case 16: return ks_kernel_ptr_16(mode, loge);
        default: return nullptr;
    }
}

}  // namespace tp
