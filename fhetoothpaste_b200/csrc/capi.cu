// C ABI of the blind-rotation engine (include/toothpaste_gpu.h): contexts,
// key upload, launches, error reporting.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "toothpaste_gpu.h"
#include "br_kernels.cuh"
#include "br_pair_kernel.cuh"
#include "dispatch.h"
#include "br_launch.h"
#include "misc_kernels.cuh"
#include "util_kernels.cuh"
#include "ks_kernels.cuh"
#include "ks_util_kernels.cuh"
#include "sap_kernels.cuh"
#include "ss_kernels.cuh"

#include <atomic>

// Kernels this library has launched in the process (tp_kernel_launches). Launches
// made while a stream is being captured into one of the library's graphs are not
// executed then; they are counted when the graph is replayed instead.
namespace tp {
static std::atomic<uint64_t> g_launches{0};
static thread_local int t_capturing = 0;
static void note_launch() {
    if (!t_capturing) g_launches.fetch_add(1, std::memory_order_relaxed);
}
}  // namespace tp

extern "C" uint64_t tp_kernel_launches(void) { return tp::g_launches.load(std::memory_order_relaxed); }

namespace {

using u128 = unsigned __int128;
constexpr uint64_t kP = 0xFFFFFFFF00000001ull;

thread_local std::string g_err;

tp_status fail(tp_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

#define TP_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? TP_ERR_OOM : TP_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                   \
    } while (0)

// ---- host Goldilocks arithmetic (tables only) ----
uint64_t hmul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % kP); }
uint64_t hpow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= kP;
    while (e) {
        if (e & 1) r = hmul(r, b);
        b = hmul(b, b);
        e >>= 1;
    }
    return r;
}
uint64_t hinv(uint64_t a) { return hpow(a, kP - 2); }
uint32_t brv(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}
int ilog2(uint64_t x) {
    int r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}

// Per-(device, N) tables: forward/inverse twiddles psi^(+-brv(k)) and psi^k, k < 2N.
struct Tables {
    int device = -1;
    int logn = 0;
    uint64_t* tw_fwd = nullptr;
    uint64_t* tw_inv = nullptr;
    uint64_t* psi_pow = nullptr;
    uint64_t n_inv = 0;
};

std::mutex g_tab_mu;
std::vector<Tables*> g_tables;

tp_status get_tables(int device, int logn, const Tables** out) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    for (auto* t : g_tables)
        if (t->device == device && t->logn == logn) {
            *out = t;
            return TP_OK;
        }
    const uint64_t N = 1ull << logn;
    // psi = 7^((p-1)/2N) (lib/src/backend/solinas.cpp:176)
    const uint64_t psi = hpow(7, (kP - 1) >> (logn + 1));
    const uint64_t psi_inv = hinv(psi);
    // twiddles psi^(+-brv(k)), k < N, followed by the radix-4 products tw[i] tw[2i], i < N/2
    std::vector<uint64_t> pw(2 * N), pwi(N), tf(N + N / 2, 0), ti(N + N / 2, 0);
    pw[0] = 1;
    for (uint64_t i = 1; i < 2 * N; ++i) pw[i] = hmul(pw[i - 1], psi);
    pwi[0] = 1;
    for (uint64_t i = 1; i < N; ++i) pwi[i] = hmul(pwi[i - 1], psi_inv);
    for (uint64_t k = 0; k < N; ++k) {
        tf[k] = pw[brv((uint32_t)k, logn)];
        ti[k] = pwi[brv((uint32_t)k, logn)];
    }
    for (uint64_t i = 1; i < N / 2; ++i) {
        tf[N + i] = hmul(tf[i], tf[2 * i]);
        ti[N + i] = hmul(ti[i], ti[2 * i]);
    }
    // The radix-4 kernels multiply by the first levels' twiddles as shifts:
    // psi^(N/2) = 2^48, psi^(N/4) = 2^120 (and their inverses 2^144, 2^72).
    if (tf[1] != hpow(2, 48) || tf[2] != hpow(2, 120) || ti[1] != hpow(2, 144) || ti[2] != hpow(2, 72))
        return fail(TP_ERR_PARAM, "unexpected NTT roots of unity (shift twiddles do not apply)");
    auto* t = new Tables();
    t->device = device;
    t->logn = logn;
    t->n_inv = hinv(N);
    cudaError_t e = cudaMalloc(&t->tw_fwd, tf.size() * 8);
    if (e == cudaSuccess) e = cudaMalloc(&t->tw_inv, ti.size() * 8);
    if (e == cudaSuccess) e = cudaMalloc(&t->psi_pow, 2 * N * 8);
    if (e == cudaSuccess) e = cudaMemcpy(t->tw_fwd, tf.data(), tf.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->tw_inv, ti.data(), ti.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->psi_pow, pw.data(), 2 * N * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(t->tw_fwd);
        cudaFree(t->tw_inv);
        cudaFree(t->psi_pow);
        delete t;
        return fail(e == cudaErrorMemoryAllocation ? TP_ERR_OOM : TP_ERR_CUDA, "table upload: %s",
                    cudaGetErrorString(e));
    }
    g_tables.push_back(t);
    *out = t;
    return TP_OK;
}

int sm_count(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v > 0 ? v : 1;
}

// Signed-digit constants of SignedGadgetDecomposeRepNTT on a 64-bit modulus
// (lib/include/static/gadget_decomp.h:16-28,156-205).
void signed_digit_consts(int beta, uint32_t digits, uint64_t& corr, uint32_t* dshift, uint64_t* dmask,
                         uint64_t* ddelta) {
    const int max_digits = (64 + beta - 1) / beta;
    uint64_t c = 0;
    int64_t shift = 64 - beta;
    while (shift > 0) {
        c += 1ull << (shift + beta - 1);
        shift -= beta;
    }
    const uint64_t least = 1ull << (shift + beta - 1);
    c += least;
    corr = c % kP;
    int64_t sh = 64 - beta;
    uint64_t mask = (1ull << beta) - 1;
    for (uint32_t d = 0; d < digits; ++d) {
        uint64_t delta = 1ull << (beta - 1);
        if ((int)d == max_digits - 1) {
            delta = least;
            sh = 0;
            mask = (delta << 1) - 1;
        }
        dshift[d] = (uint32_t)sh;
        dmask[d] = mask;
        ddelta[d] = delta;
        sh -= beta;
    }
}

uint32_t inv_mod_2n(uint32_t t, uint32_t two_n) {
    for (uint32_t x = 1; x < two_n; x += 2)
        if ((uint64_t)x * t % two_n == 1) return x;
    return 0;
}

}  // namespace

struct tp_br_ctx {
    tp_br_params prm{};
    int device = 0;
    int logn = 0;
    int G = 1;                    // RGSWs per iteration group
    uint64_t groups = 0;          // iteration groups (n, or n/2 for BMMP)
    uint64_t key_words = 0;
    const Tables* tab = nullptr;
    uint64_t* key = nullptr;      // device layout
    bool key_ready = false;
    unsigned int* err = nullptr;  // device error word
    tp::BrKernelParams kp{};
    int loge = 3;                 // log2 coefficients per thread of the active tile
    const void* kernels[4] = {};  // by loge (2, 3)
    int grid_caps[4] = {};        // resident blocks on the device, by loge
    size_t smem[4] = {};          // dynamic shared memory bytes, by loge
    int logs = 0;                 // log2 of the CTAs of one rotation's cluster (N > 4096), else 0
    int split = 1;                // thread blocks per rotation (2, 4: cluster kernels, tile 4 only)
    int mac = 0;                  // multiply-accumulate form of the one-block kernel at tile 4 (TP_MAC_*)
    const void* ds_kernel = nullptr;  // digit-staged one-block kernel (digits 3 or 4, N <= 2048)
    size_t ds_smem = 0;
    int ds_cap = 0;               // its resident blocks on the device (0: unavailable)
    int radix = 2;                // NTT passes of the one-block kernel at tile 4: 2 or 4 (fused radix-4)
    struct Form {
        const void* k = nullptr;
        size_t smem = 0;
        int cap = 0;
    };
    Form r4_row, r4_ds;           // the fused radix-4 one-block kernels (row by row, digit-staged)
    const void* pair_kernel = nullptr;
    size_t pair_smem = 0;
    int pair_cap = 0;             // resident two-CTA clusters on the device (0: unavailable)
    const void* quad_kernel = nullptr;
    size_t quad_smem = 0;
    int quad_cap = 0;             // resident four-CTA clusters on the device (0: unavailable)
    // workspace for host-pointer calls
    uint64_t* ws = nullptr;
    uint64_t ws_words = 0;
    std::mutex mu;                // serializes host-pointer calls on one context
};

// Ring sizes above 4096: one rotation per cluster of 2^logs CTAs. Sets up the
// row-by-row kernel (the default) and, for 3 or 4 digits where it fits, the
// digit-staged one; 4 coefficients per thread, no split kernels.
static tp_status br_setup_cluster(tp_br_ctx* c) {
    const int S = 1 << c->logs;
    const uint32_t T = c->prm.ring_dim >> (c->logs + 2);
    auto probe = [&](const void* k, size_t smem, int* cap) -> bool {
        if (!k || smem > 227u * 1024u) return false;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess && S > 8) e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        int clusters = 0;
        if (e == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr = {};
            attr.id = cudaLaunchAttributeClusterDimension;
            attr.val.clusterDim.x = (unsigned)S;
            attr.val.clusterDim.y = 1;
            attr.val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)S * (unsigned)sm_count(c->device));
            cfg.blockDim = dim3(T);
            cfg.dynamicSmemBytes = smem;
            cfg.attrs = &attr;
            cfg.numAttrs = 1;
            e = cudaOccupancyMaxActiveClusters(&clusters, k, &cfg);
        }
        if (e != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            return false;
        }
        *cap = clusters;
        return true;
    };
    const void* k = tp::br_kernel_lookup(c->logn, c->prm.variant, 2, 0);
    const size_t smem = tp::br_smem_words(c->logn, c->prm.variant, c->prm.lwe_dim, 2, 0, c->logs) * 8;
    int cap = 0;
    if (!probe(k, smem, &cap))
        return fail(TP_ERR_PARAM, "the %d-CTA cluster rotation kernel does not fit (N=%u, n=%u, smem=%zu) on device %d",
                    S, c->prm.ring_dim, c->prm.lwe_dim, smem, c->device);
    c->kernels[2] = k;
    c->smem[2] = smem;
    c->grid_caps[2] = cap;
    c->loge = 2;
    if (c->prm.digits == 3 || c->prm.digits == 4) {
        const void* kd = tp::br_kernel_lookup(c->logn, c->prm.variant, 2, (int)c->prm.digits);
        const size_t sd =
            tp::br_smem_words(c->logn, c->prm.variant, c->prm.lwe_dim, 2, (int)c->prm.digits, c->logs) * 8;
        int capd = 0;
        if (probe(kd, sd, &capd)) {
            // selectable, not the default (with 2048 coefficients per CTA the row-by-row form
            // measured faster on a cluster: N = 8192, ternary n = 1024, 670 vs 600 rotations/s);
            // the clusters of 4096 coefficients per CTA built now have no digit-staged kernel
            c->ds_kernel = kd;
            c->ds_smem = sd;
            c->ds_cap = capd;
        }
    }
    return TP_OK;
}

extern "C" {

const char* tp_last_error(void) { return g_err.c_str(); }

const char* tp_version(void) { return "toothpaste-b200 0.1 (sm_100a)"; }

tp_status tp_br_create(const tp_br_params* p, int device, tp_br_ctx** out) {
    if (!p || !out) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (p->modulus != kP) return fail(TP_ERR_PARAM, "modulus must be the Goldilocks prime 2^64-2^32+1");
    if (p->variant < 0 || p->variant > 2) return fail(TP_ERR_PARAM, "unknown variant %d", p->variant);
    const uint64_t N = p->ring_dim;
    if (N < 128 || N > 65536 || (N & (N - 1)))
        return fail(TP_ERR_PARAM, "ring_dim must be a power of two in [128, 65536]");
    if (p->lwe_dim == 0) return fail(TP_ERR_PARAM, "lwe_dim must be positive");
    if (p->variant == TP_BR_BMMP_BINARY && (p->lwe_dim % 2)) return fail(TP_ERR_PARAM, "BMMP needs an even lwe_dim");
    if (p->basis < 2 || (p->basis & (p->basis - 1))) return fail(TP_ERR_PARAM, "basis must be a power of two");
    const int beta = ilog2(p->basis);
    if (beta > 30) return fail(TP_ERR_PARAM, "basis above 2^30 is not supported");
    const int max_digits = (64 + beta - 1) / beta;
    if (p->digits < 1 || p->digits > 8 || (int)p->digits > max_digits)
        return fail(TP_ERR_PARAM, "digits must be in [1, min(8, ceil(64/beta))]");

    auto* c = new tp_br_ctx();
    c->prm = *p;
    c->device = device;
    c->logn = ilog2(N);
    c->logs = tp::br_cluster_logs(c->logn);
    c->G = tp::br_rgsw_per_group(p->variant);
    c->groups = p->variant == TP_BR_BMMP_BINARY ? p->lwe_dim / 2 : p->lwe_dim;
    c->key_words = c->groups * (uint64_t)c->G * 4 * N * p->digits;

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete c;
        return fail(TP_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    }
    tp_status s = get_tables(device, c->logn, &c->tab);
    if (s != TP_OK) {
        delete c;
        return s;
    }
    e = cudaMalloc(&c->err, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(c->err, 0, sizeof(unsigned int));
    if (e != cudaSuccess) {
        delete c;
        return fail(TP_ERR_CUDA, "error word: %s", cudaGetErrorString(e));
    }

    // Decomposition constants.
    tp::BrKernelParams& kp = c->kp;
    kp.tw_fwd = c->tab->tw_fwd;
    kp.tw_inv = c->tab->tw_inv;
    kp.psi_pow = c->tab->psi_pow;
    kp.n = p->lwe_dim;
    kp.digits = p->digits;
    kp.n_inv = c->tab->n_inv;
    kp.err = c->err;
    if (p->variant == TP_BR_CGGI_BINARY) {
        // unsigned digits, first shift beta*(ceil(64/beta)-1) (mux_operator.cpp:23-26,46-69)
        const int first = beta * (max_digits - 1);
        for (uint32_t d = 0; d < p->digits; ++d) {
            kp.dshift[d] = (uint32_t)(first - (int)d * beta);
            kp.dmask[d] = (1ull << beta) - 1;
            kp.ddelta[d] = 0;
        }
        kp.corr = 0;
    } else {
        // signed digits (gadget_decomp.h:16-28,156-205)
        uint64_t corr = 0;
        int64_t shift = 64 - beta;
        while (shift > 0) {
            corr += 1ull << (shift + beta - 1);
            shift -= beta;
        }
        const uint64_t least = 1ull << (shift + beta - 1);
        corr += least;
        kp.corr = corr % kP;
        int64_t sh = 64 - beta;
        uint64_t mask = (1ull << beta) - 1;
        for (uint32_t d = 0; d < p->digits; ++d) {
            uint64_t delta = 1ull << (beta - 1);
            if ((int)d == max_digits - 1) {
                delta = least;
                sh = 0;
                mask = (delta << 1) - 1;
            }
            kp.dshift[d] = (uint32_t)sh;
            kp.dmask[d] = mask;
            kp.ddelta[d] = delta;
            sh -= beta;
        }
    }

    // Digits small enough for the integer pass 0 of the digit transforms: signed digits lie in
    // [-2^(beta-1), 2^(beta-1)), unsigned in [0, 2^beta); the pass is exact up to 2^14.
    kp.small_digits = (p->variant == TP_BR_CGGI_BINARY ? beta <= 14 : beta <= 15) ? 1u : 0u;
    if (c->logs > 0) {
        tp_status cs = br_setup_cluster(c);
        if (cs != TP_OK) {
            cudaFree(c->err);
            delete c;
            return cs;
        }
        *out = c;
        return TP_OK;
    }
    for (int lg = 2; lg <= 3; ++lg) {
        const void* k = tp::br_kernel_lookup(c->logn, p->variant, lg);
        const size_t smem = tp::br_smem_words(c->logn, p->variant, p->lwe_dim, lg) * 8;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, (int)(N >> lg), smem);
        if (e != cudaSuccess || per_sm < 1) {
            cudaFree(c->err);
            delete c;
            return fail(TP_ERR_PARAM, "blind-rotation kernel does not fit (N=%llu, n=%u, smem=%zu, %d per thread): %s",
                        (unsigned long long)N, p->lwe_dim, smem, 1 << lg,
                        e == cudaSuccess ? "no resident block" : cudaGetErrorString(e));
        }
        c->kernels[lg] = k;
        c->smem[lg] = smem;
        c->grid_caps[lg] = per_sm * sm_count(device);
    }
    c->loge = tp::br_default_loge(c->logn, p->variant);
    if (p->digits == 3 || p->digits == 4) {
        // digit-staged kernel: optional, a parameter set it does not fit keeps the row-by-row form
        const void* k = tp::br_kernel_lookup(c->logn, p->variant, 2, (int)p->digits);
        const size_t smem = tp::br_smem_words(c->logn, p->variant, p->lwe_dim, 2, (int)p->digits) * 8;
        int per_sm = 0;
        cudaError_t de = k && smem <= 227u * 1024u
                             ? cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                             : cudaErrorInvalidValue;
        if (de == cudaSuccess) de = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, (int)(N >> 2), smem);
        if (de == cudaSuccess && per_sm > 0) {
            c->ds_kernel = k;
            c->ds_smem = smem;
            c->ds_cap = per_sm * sm_count(device);
            c->mac = TP_MAC_DIGIT_STAGED;
        } else if (k) {
            cudaGetLastError();  // clear the optional probe's error
        }
    }
    // fused radix-4 forms at tile 4: optional (built for N = 1024 .. 4096, where they fit)
    for (int dl : {0, (int)p->digits}) {
        if (dl != 0 && dl != 3 && dl != 4) continue;
        const void* k = tp::br_kernel_lookup(c->logn, p->variant, 2, dl, true);
        const size_t smem = tp::br_smem_words(c->logn, p->variant, p->lwe_dim, 2, dl, 0, true) * 8;
        int per_sm = 0;
        cudaError_t re = k && smem <= 227u * 1024u
                             ? cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                             : cudaErrorInvalidValue;
        if (re == cudaSuccess) re = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, (int)(N >> 2), smem);
        if (re == cudaSuccess && per_sm > 0) {
            auto& f = dl == 0 ? c->r4_row : c->r4_ds;
            f.k = k;
            f.smem = smem;
            f.cap = per_sm * sm_count(device);
        } else if (k) {
            cudaGetLastError();
        }
    }
    for (int split = 2; split <= 4; split += 2) {
        // two- and four-CTA cluster kernels; optional: a parameter set one does not fit keeps its cap 0
        const void* k = tp::br_pair_kernel_lookup(c->logn, p->variant, split);
        const size_t smem = tp::br_pair_smem_words(c->logn, p->variant, p->lwe_dim, 2, split) * 8;
        int clusters = 0;
        cudaError_t pe = k ? cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                           : cudaErrorInvalidValue;
        if (pe == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)split * (unsigned)sm_count(device));
            cfg.blockDim = dim3((unsigned)(N >> 2));
            cfg.dynamicSmemBytes = smem;
            pe = cudaOccupancyMaxActiveClusters(&clusters, k, &cfg);
        }
        if (pe == cudaSuccess && clusters > 0) {
            (split == 2 ? c->pair_kernel : c->quad_kernel) = k;
            (split == 2 ? c->pair_smem : c->quad_smem) = smem;
            (split == 2 ? c->pair_cap : c->quad_cap) = clusters;
        } else if (k) {
            cudaGetLastError();  // clear the optional probe's error
        }
    }
    *out = c;
    return TP_OK;
}

tp_status tp_br_destroy(tp_br_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    cudaFree(c->key);
    cudaFree(c->err);
    cudaFree(c->ws);
    delete c;
    return TP_OK;
}

uint64_t tp_br_key_words(const tp_br_ctx* c) { return c ? c->key_words : 0; }

tp_status tp_br_upload_key(tp_br_ctx* c, const uint64_t* brk, uint64_t words) {
    if (!c || !brk) return fail(TP_ERR_PARAM, "null argument");
    if (words != c->key_words)
        return fail(TP_ERR_LAYOUT, "key has %llu words, context expects %llu", (unsigned long long)words,
                    (unsigned long long)c->key_words);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    if (!c->key) TP_CUDA(cudaMalloc(&c->key, c->key_words * 8));
    const uint64_t N = c->prm.ring_dim;
    const uint64_t per_group = (uint64_t)c->G * 4 * N * c->prm.digits;
    // stage at most ~128 MB of the reference layout at a time
    uint64_t chunk = (128ull << 20) / (per_group * 8);
    if (chunk < 1) chunk = 1;
    if (chunk > c->groups) chunk = c->groups;
    uint64_t* stage = nullptr;
    TP_CUDA(cudaMalloc(&stage, chunk * per_group * 8));
    tp_status st = TP_OK;
    for (uint64_t g0 = 0; g0 < c->groups && st == TP_OK; g0 += chunk) {
        const uint64_t ng = std::min(chunk, c->groups - g0);
        cudaError_t e = cudaMemcpy(stage, brk + g0 * per_group, ng * per_group * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            const uint64_t total = ng * per_group;
            const int threads = 256;
            const uint64_t blocks = std::min<uint64_t>((total + threads - 1) / threads, 65535);
            tp::key_relayout_kernel<<<(unsigned)blocks, threads>>>(c->key + g0 * per_group, stage, ng, c->G,
                                                                    2 * c->prm.digits, c->logn, c->loge, c->logs);
            tp::note_launch();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) st = fail(TP_ERR_CUDA, "key upload: %s", cudaGetErrorString(e));
    }
    cudaFree(stage);
    if (st == TP_OK) c->key_ready = true;
    return st;
}

tp_status tp_br_blind_rotate_batch(tp_br_ctx* c, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                   uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef,
                                   void* stream) {
    return tp::br_batch_launch(c, batch, results, lwes, lwe_stride, accs, acc_stride, out_coef, stream, 0);
}

// Moves the resident key to the layout of another tile (2x key memory while it runs).
static tp_status br_retile(tp_br_ctx* c, int loge) {
    if (loge == c->loge) return TP_OK;
    if (c->logs > 0) return fail(TP_ERR_PARAM, "cluster rotations run with 4 coefficients per thread only");
    if (c->key_ready) {
        uint64_t* nk = nullptr;
        TP_CUDA(cudaMalloc(&nk, c->key_words * 8));
        const uint64_t blocks = std::min<uint64_t>((c->key_words + 255) / 256, 65535);
        tp::key_retile_kernel<<<(unsigned)blocks, 256>>>(nk, c->key, c->groups, c->G, 2 * c->prm.digits, c->logn,
                                                          c->loge, loge);
        tp::note_launch();
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            cudaFree(nk);
            return fail(TP_ERR_CUDA, "key re-tiling: %s", cudaGetErrorString(e));
        }
        cudaFree(c->key);
        c->key = nk;
    }
    c->loge = loge;
    return TP_OK;
}

tp_status tp_br_set_tile(tp_br_ctx* c, uint32_t coef_per_thread) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (coef_per_thread != 4 && coef_per_thread != 8) return fail(TP_ERR_PARAM, "coefficients per thread must be 4 or 8");
    std::lock_guard<std::mutex> lk(c->mu);
    if (coef_per_thread == 8 && c->split > 1)
        return fail(TP_ERR_STATE, "the %d-block kernel runs with 4 coefficients per thread; set the split to 1 first",
                    c->split);
    if (coef_per_thread == 8 && c->logs > 0)
        return fail(TP_ERR_PARAM, "ring dimension %u rotates on a CTA cluster with 4 coefficients per thread only",
                    c->prm.ring_dim);
    TP_CUDA(cudaSetDevice(c->device));
    return br_retile(c, coef_per_thread == 4 ? 2 : 3);
}

uint32_t tp_br_get_tile(const tp_br_ctx* c) { return c ? 1u << c->loge : 0u; }

tp_status tp_br_set_split(tp_br_ctx* c, uint32_t blocks_per_rotation) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (blocks_per_rotation != 1 && blocks_per_rotation != 2 && blocks_per_rotation != 4)
        return fail(TP_ERR_PARAM, "blocks per rotation must be 1, 2 or 4");
    std::lock_guard<std::mutex> lk(c->mu);
    if (blocks_per_rotation > 1) {
        if ((blocks_per_rotation == 2 ? c->pair_cap : c->quad_cap) == 0)
            return fail(TP_ERR_PARAM, "the %u-block kernel does not fit this parameter set on this device",
                        blocks_per_rotation);
        if (c->loge != 2)
            return fail(TP_ERR_STATE, "the %u-block kernel runs with 4 coefficients per thread; set the tile first",
                        blocks_per_rotation);
    }
    c->split = (int)blocks_per_rotation;
    return TP_OK;
}

uint32_t tp_br_get_split(const tp_br_ctx* c) { return c ? (uint32_t)c->split : 0u; }

tp_status tp_br_set_mac_form(tp_br_ctx* c, uint32_t form) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (form != TP_MAC_ROWWISE && form != TP_MAC_DIGIT_STAGED)
        return fail(TP_ERR_PARAM, "unknown multiply-accumulate form %u", form);
    std::lock_guard<std::mutex> lk(c->mu);
    if (form == TP_MAC_DIGIT_STAGED && !c->ds_kernel)
        return fail(TP_ERR_PARAM, "the digit-staged kernel is not built for this parameter set on this device "
                                  "(digits 3 or 4, N <= 2048, shared memory permitting)");
    c->mac = (int)form;
    return TP_OK;
}

uint32_t tp_br_get_mac_form(const tp_br_ctx* c) { return c ? (uint32_t)c->mac : 0u; }

tp_status tp_br_set_radix(tp_br_ctx* c, uint32_t radix) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (radix != 2 && radix != 4) return fail(TP_ERR_PARAM, "radix must be 2 or 4");
    std::lock_guard<std::mutex> lk(c->mu);
    if (radix == 4 && !c->r4_row.k)
        return fail(TP_ERR_PARAM, "fused radix-4 rotation kernels are not built for this parameter set "
                                  "(N = 1024 .. 4096, shared memory permitting)");
    c->radix = (int)radix;
    return TP_OK;
}

uint32_t tp_br_get_radix(const tp_br_ctx* c) { return c ? (uint32_t)c->radix : 0u; }

tp_status tp_br_autotune(tp_br_ctx* c, uint64_t batch, uint32_t* best_coef_per_thread, double* best_rotations_per_s) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (batch == 0) return fail(TP_ERR_PARAM, "empty batch");
    const uint64_t N = c->prm.ring_dim, n = c->prm.lwe_dim;
    const uint64_t cap = (uint64_t)std::max(std::max(c->grid_caps[2], c->grid_caps[3]), c->pair_cap);  // >= quad_cap
    const uint64_t tb = std::min<uint64_t>(batch, 2 * cap);  // at most two waves per trial
    std::vector<uint64_t> lw(tb * (n + 1));
    uint64_t z = 0x5eedull;
    for (auto& w : lw) {  // splitmix64 words in [0, 2N): timing does not depend on the values
        uint64_t x = (z += 0x9E3779B97F4A7C15ull);
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        w = (x ^ (x >> 31)) & (2 * N - 1);
    }
    TP_CUDA(cudaSetDevice(c->device));
    uint64_t *d_lwe = nullptr, *d_acc = nullptr, *d_res = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    tp_status s = TP_OK;
    double best_rate = 0.0;
    int best = c->loge;
    auto cleanup = [&]() {
        cudaFree(d_lwe);
        cudaFree(d_acc);
        cudaFree(d_res);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    };
    cudaError_t e = cudaMalloc(&d_lwe, lw.size() * 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_acc, 2 * N * 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_res, tb * 2 * N * 8);
    if (e == cudaSuccess) e = cudaMemcpy(d_lwe, lw.data(), lw.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_acc, 0, 2 * N * 8);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cleanup();
        return fail(TP_ERR_CUDA, "autotune set-up: %s", cudaGetErrorString(e));
    }
    std::lock_guard<std::mutex> lk(c->mu);
    int best_split = c->split;
    int best_mac = c->mac;
    int best_radix = c->radix;
    // tile (coefficients per thread), blocks per rotation, multiply-accumulate form, NTT radix
    struct Cand { int loge, split, mac, radix; };
    const Cand cands[] = {{3, 1, TP_MAC_ROWWISE, 2},      {2, 1, TP_MAC_ROWWISE, 2}, {2, 1, TP_MAC_DIGIT_STAGED, 2},
                          {2, 1, TP_MAC_ROWWISE, 4},      {2, 1, TP_MAC_DIGIT_STAGED, 4},
                          {2, 2, TP_MAC_ROWWISE, 2},      {2, 4, TP_MAC_ROWWISE, 2}};
    for (const Cand& cd : cands) {
        if ((cd.split == 2 && c->pair_cap == 0) || (cd.split == 4 && c->quad_cap == 0)) continue;
        if (cd.mac == TP_MAC_DIGIT_STAGED && !c->ds_kernel) continue;
        if (cd.radix == 4 && !(cd.mac == TP_MAC_DIGIT_STAGED ? c->r4_ds.k : c->r4_row.k)) continue;
        if (cd.loge != 2 && c->logs > 0) continue;  // clusters: 4 coefficients per thread
        s = br_retile(c, cd.loge);
        if (s != TP_OK) break;
        c->split = cd.split;
        c->mac = cd.mac;
        c->radix = cd.radix;
        for (int rep = 0; rep < 3 && s == TP_OK; ++rep) {  // one warm-up, two timed
            if (rep == 1) cudaEventRecord(e0, st);
            s = tp_br_blind_rotate_batch(c, tb, d_res, d_lwe, n + 1, d_acc, 0, 0, st);
        }
        if (s != TP_OK) break;
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            s = fail(TP_ERR_CUDA, "autotune timing: %s", cudaGetErrorString(e));
            break;
        }
        const double rate = 2.0 * tb / (ms * 1e-3);
        if (rate > best_rate) {
            best_rate = rate;
            best = cd.loge;
            best_split = cd.split;
            best_mac = cd.mac;
            best_radix = cd.radix;
        }
    }
    c->split = 1;
    if (s == TP_OK) s = br_retile(c, best);
    if (s == TP_OK) {
        c->split = best_split;
        c->mac = best_mac;
        c->radix = best_radix;
    }
    cleanup();
    if (s != TP_OK) return s;
    if (best_coef_per_thread) *best_coef_per_thread = 1u << best;
    if (best_rotations_per_s) *best_rotations_per_s = best_rate;
    return TP_OK;
}

tp_status tp_br_check(tp_br_ctx* c, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    TP_CUDA(cudaSetDevice(c->device));
    TP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    unsigned int flags = 0;
    TP_CUDA(cudaMemcpy(&flags, c->err, sizeof flags, cudaMemcpyDeviceToHost));
    TP_CUDA(cudaMemset(c->err, 0, sizeof flags));
    if (flags & 1u) return fail(TP_ERR_PARAM, "an LWE word was outside [0, 2N); it was reduced mod 2N");
    return TP_OK;
}

static tp_status ensure_ws(tp_br_ctx* c, uint64_t words) {
    if (c->ws_words >= words) return TP_OK;
    cudaFree(c->ws);
    c->ws = nullptr;
    c->ws_words = 0;
    TP_CUDA(cudaMalloc(&c->ws, words * 8));
    c->ws_words = words;
    return TP_OK;
}

tp_status tp_br_blind_rotate_batch_host(tp_br_ctx* c, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                        uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef,
                                        void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (batch == 0) return TP_OK;
    if (!results || !lwes || !accs) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->prm.ring_dim, n = c->prm.lwe_dim;
    if (lwe_stride < n + 1) return fail(TP_ERR_PARAM, "lwe_stride below n+1");
    if (acc_stride != 0 && acc_stride < 2 * N) return fail(TP_ERR_PARAM, "acc_stride below 2N");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    const uint64_t lw = (batch * (n + 1) + 1) & ~1ull;
    const uint64_t aw = acc_stride ? batch * 2 * N : 2 * N;
    const uint64_t rw = batch * 2 * N;
    tp_status s = ensure_ws(c, lw + aw + rw);
    if (s != TP_OK) return s;
    uint64_t* d_res = c->ws;
    uint64_t* d_acc = c->ws + rw;
    uint64_t* d_lwe = c->ws + rw + aw;
    cudaStream_t st = (cudaStream_t)stream;
    TP_CUDA(cudaMemcpy2DAsync(d_lwe, (n + 1) * 8, lwes, lwe_stride * 8, (n + 1) * 8, batch, cudaMemcpyHostToDevice, st));
    if (acc_stride)
        TP_CUDA(cudaMemcpy2DAsync(d_acc, 2 * N * 8, accs, acc_stride * 8, 2 * N * 8, batch, cudaMemcpyHostToDevice, st));
    else
        TP_CUDA(cudaMemcpyAsync(d_acc, accs, 2 * N * 8, cudaMemcpyHostToDevice, st));
    s = tp_br_blind_rotate_batch(c, batch, d_res, d_lwe, n + 1, d_acc, acc_stride ? 2 * N : 0, out_coef, stream);
    if (s != TP_OK) return s;
    TP_CUDA(cudaMemcpyAsync(results, d_res, rw * 8, cudaMemcpyDeviceToHost, st));
    TP_CUDA(cudaStreamSynchronize(st));
    return TP_OK;
}

tp_status tp_br_blind_rotate(tp_br_ctx* c, uint64_t* result, const uint64_t* lwe, const uint64_t* acc, int out_coef) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    tp_status s = tp_br_blind_rotate_batch_host(c, 1, result, lwe, (uint64_t)c->prm.lwe_dim + 1, acc,
                                                2ull * c->prm.ring_dim, out_coef, nullptr);
    if (s != TP_OK) return s;
    return tp_br_check(c, nullptr);
}

tp_status tp_sample_extract_batch(uint32_t ring_dim, uint64_t batch, uint64_t* out, const uint64_t* rlwe,
                                  void* stream) {
    if (ring_dim < 2 || (ring_dim & (ring_dim - 1))) return fail(TP_ERR_PARAM, "ring_dim must be a power of two");
    if (batch == 0) return TP_OK;
    if (!out || !rlwe) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t total = batch * ((uint64_t)ring_dim + 1);
    const int threads = 256;
    const uint64_t blocks = std::min<uint64_t>((total + threads - 1) / threads, 65535);
    tp::sample_extract0_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(out, rlwe, batch, ring_dim);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

struct tp_graph {
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    uint64_t kernels = 0;  // kernel nodes of the graph: launches per replay
};

static uint64_t graph_kernel_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    uint64_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}

tp_status tp_br_batch_graph_create(tp_br_ctx* c, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                   uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef,
                                   uint64_t* extract_out, tp_graph** out) {
    if (!c || !out) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (batch == 0) return fail(TP_ERR_PARAM, "empty batch");
    if (extract_out && !out_coef) return fail(TP_ERR_PARAM, "SampleExtract needs coefficient-domain results");
    TP_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = nullptr;
    TP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(s);
        return fail(TP_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    ++tp::t_capturing;
    tp_status st = tp_br_blind_rotate_batch(c, batch, results, lwes, lwe_stride, accs, acc_stride, out_coef, s);
    if (st == TP_OK && extract_out) st = tp_sample_extract_batch(c->prm.ring_dim, batch, extract_out, results, s);
    --tp::t_capturing;
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);  // always ends the capture, also after a failed launch
    cudaStreamDestroy(s);
    if (st != TP_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    auto* gr = new tp_graph();
    gr->device = c->device;
    gr->kernels = graph_kernel_nodes(g);
    e = cudaGraphInstantiate(&gr->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        delete gr;
        return fail(TP_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
    }
    *out = gr;
    return TP_OK;
}

tp_status tp_graph_launch(tp_graph* g, void* stream) {
    if (!g) return fail(TP_ERR_PARAM, "null graph");
    TP_CUDA(cudaSetDevice(g->device));
    TP_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    if (!tp::t_capturing) tp::g_launches.fetch_add(g->kernels, std::memory_order_relaxed);
    return TP_OK;
}

tp_status tp_graph_destroy(tp_graph* g) {
    if (!g) return TP_OK;
    cudaSetDevice(g->device);
    cudaGraphExecDestroy(g->exec);
    delete g;
    return TP_OK;
}

tp_status tp_debug_arith(int op, uint64_t count, uint64_t* out, const uint64_t* a, const uint64_t* b,
                         const uint64_t* c, void* stream) {
    if (op < 0 || op > 9) return fail(TP_ERR_PARAM, "unknown op %d", op);
    if (count == 0) return TP_OK;
    if (!out || !a || !b || !c) return fail(TP_ERR_PARAM, "null buffer");
    const int threads = 256;
    const uint64_t blocks = std::min<uint64_t>((count + threads - 1) / threads, 65535);
    tp::debug_arith_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(op, count, out, a, b, c);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

tp_status tp_measure_int_peak(int device, double* products_per_s, double* imad_per_s) {
    if (!products_per_s || !imad_per_s) return fail(TP_ERR_PARAM, "null argument");
    TP_CUDA(cudaSetDevice(device));
    const int threads = 256, per_sm = 8, iters = 2048;
    const int blocks = sm_count(device) * per_sm;
    uint64_t* out = nullptr;
    TP_CUDA(cudaMalloc(&out, (size_t)blocks * threads * 8));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms[2] = {0, 0};
    for (int mode = 0; mode < 2; ++mode) {
        for (int rep = 0; rep < 3; ++rep) {  // last repetition is timed
            cudaEventRecord(e0);
            if (mode == 0) tp::int_peak_kernel<0><<<blocks, threads>>>(out, 12345, iters);
            else tp::int_peak_kernel<1><<<blocks, threads>>>(out, 12345, iters);
            tp::note_launch();
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms[mode], e0, e1);
        }
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "peak probe: %s", cudaGetErrorString(e));
    const double ops = (double)blocks * threads * iters * 8;
    *products_per_s = ops / (ms[0] * 1e-3);
    *imad_per_s = 4 * ops / (ms[1] * 1e-3);
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Key switching contexts: RLWE -> RLWE, automorphism, packing
// ---------------------------------------------------------------------------
struct tp_ks_ctx {
    int kind = 0;                 // 0 RLWE KS, 1 automorphism, 2 packing
    int device = 0;
    int logn = 0;
    uint32_t N = 0;
    uint32_t digits = 0;
    uint32_t index = 0;           // automorphism index (kind 1)
    uint64_t basis = 0;
    int nkeys = 1;                // packing: logN keys, index 2^j + 1, j = 1..logN
    uint64_t key_words = 0;
    const Tables* tab = nullptr;
    uint64_t* key = nullptr;
    bool key_ready = false;
    tp::KsKernelParams kp{};
    size_t smem = 0;
    int loge = 2;                 // log2 coefficients per thread: 2 (4) or 3 (8)
    int per_sm[2][tp::kKsModes] = {};
    int logs = 0;                 // log2 CTAs per item's cluster (N > 4096), else 0
    int cluster_cap[tp::kKsModes] = {};  // resident clusters per mode (logs > 0)
    uint64_t* work = nullptr;     // packing tree nodes
    uint64_t work_words = 0;
    // PackConsecutively plan for consec_len inputs: leaf inputs, then each level's node pairs
    uint64_t consec_len = 0;
    uint32_t* consec_plan = nullptr;
    std::vector<uint64_t> consec_off;  // per level: offset into the plan (words)
    std::vector<uint32_t> consec_cnt;  // per level: nodes of one pack
    uint64_t* zero = nullptr;          // 2N zero words
    std::mutex mu;
};

static tp_status ks_create(int kind, uint32_t ring_dim, uint64_t basis, uint32_t digits, uint32_t index, int device,
                           tp_ks_ctx** out) {
    if (!out) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (ring_dim < 128 || ring_dim > 65536 || (ring_dim & (ring_dim - 1)))
        return fail(TP_ERR_PARAM, "ring_dim must be a power of two in [128, 65536]");
    if (basis < 2 || (basis & (basis - 1))) return fail(TP_ERR_PARAM, "basis must be a power of two");
    const int beta = ilog2(basis);
    if (beta > 30) return fail(TP_ERR_PARAM, "basis above 2^30 is not supported");
    const int max_digits = (64 + beta - 1) / beta;
    if (digits < 1 || digits > 8 || (int)digits > max_digits)
        return fail(TP_ERR_PARAM, "digits must be in [1, min(8, ceil(64/beta))]");
    if (kind == 1 && (index % 2 == 0 || index >= 2 * ring_dim))
        return fail(TP_ERR_PARAM, "automorphism index must be odd and below 2N");
    auto* c = new tp_ks_ctx();
    c->kind = kind;
    c->device = device;
    c->basis = basis;
    c->N = ring_dim;
    c->logn = ilog2(ring_dim);
    c->digits = digits;
    c->index = index;
    c->nkeys = kind == 2 ? c->logn : 1;
    c->loge = 2;  // 4 per thread: faster than 8 in every mode and ring size measured
    c->logs = tp::br_cluster_logs(c->logn);
    c->key_words = (uint64_t)c->nkeys * digits * 2 * ring_dim;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete c;
        return fail(TP_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    }
    tp_status s = get_tables(device, c->logn, &c->tab);
    if (s != TP_OK) {
        delete c;
        return s;
    }
    tp::KsKernelParams& kp = c->kp;
    kp.tw_fwd = c->tab->tw_fwd;
    kp.tw_inv = c->tab->tw_inv;
    kp.digits = digits;
    kp.n_inv = c->tab->n_inv;
    signed_digit_consts(beta, digits, kp.corr, kp.dshift, kp.dmask, kp.ddelta);
    c->smem = tp::ks_smem_words((int)ring_dim, 1 << c->logs) * 8;
    if (c->logs > 0) {
        // one item per cluster of 2^logs CTAs, 4 coefficients per thread
        const int S = 1 << c->logs;
        for (int mode = 0; mode < tp::kKsModes; ++mode) {
            const void* k = tp::ks_kernel_lookup(c->logn, mode, 2);
            e = k ? cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem)
                  : cudaErrorInvalidValue;
            if (e == cudaSuccess && S > 8) e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            int clusters = 0;
            if (e == cudaSuccess) {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute attr = {};
                attr.id = cudaLaunchAttributeClusterDimension;
                attr.val.clusterDim.x = (unsigned)S;
                attr.val.clusterDim.y = 1;
                attr.val.clusterDim.z = 1;
                cfg.gridDim = dim3((unsigned)S * (unsigned)sm_count(device));
                cfg.blockDim = dim3(ring_dim >> (c->logs + 2));
                cfg.dynamicSmemBytes = c->smem;
                cfg.attrs = &attr;
                cfg.numAttrs = 1;
                e = cudaOccupancyMaxActiveClusters(&clusters, k, &cfg);
            }
            if (e != cudaSuccess || clusters < 1) {
                delete c;
                return fail(TP_ERR_CUDA, "key-switch cluster kernel set-up (N=%u): %s", ring_dim,
                            e == cudaSuccess ? "no resident cluster" : cudaGetErrorString(e));
            }
            c->cluster_cap[mode] = clusters;
        }
        *out = c;
        return TP_OK;
    }
    for (int loge = 2; loge <= 3; ++loge) {
        for (int mode = 0; mode < tp::kKsModes; ++mode) {
            const void* k = tp::ks_kernel_lookup(c->logn, mode, loge);
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->per_sm[loge - 2][mode], k, ring_dim >> loge,
                                                                  c->smem);
            if (e != cudaSuccess || c->per_sm[loge - 2][mode] < 1) {
                delete c;
                return fail(TP_ERR_CUDA, "key-switch kernel set-up: %s", cudaGetErrorString(e));
            }
        }
    }
    *out = c;
    return TP_OK;
}

tp_status tp_rlwe_ks_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, int device, tp_ks_ctx** out) {
    return ks_create(0, ring_dim, basis, digits, 0, device, out);
}

tp_status tp_auto_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, uint32_t index, int device,
                         tp_ks_ctx** out) {
    return ks_create(1, ring_dim, basis, digits, index, device, out);
}

tp_status tp_pack_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, int device, tp_ks_ctx** out) {
    return ks_create(2, ring_dim, basis, digits, 0, device, out);
}

tp_status tp_ks_destroy(tp_ks_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    cudaFree(c->key);
    cudaFree(c->work);
    cudaFree(c->consec_plan);
    cudaFree(c->zero);
    delete c;
    return TP_OK;
}

uint64_t tp_ks_key_words(const tp_ks_ctx* c) { return c ? c->key_words : 0; }

tp_status tp_ks_upload_key(tp_ks_ctx* c, const uint64_t* ksk, uint64_t words) {
    if (!c || !ksk) return fail(TP_ERR_PARAM, "null argument");
    if (words != c->key_words)
        return fail(TP_ERR_LAYOUT, "key has %llu words, context expects %llu", (unsigned long long)words,
                    (unsigned long long)c->key_words);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    if (!c->key) TP_CUDA(cudaMalloc(&c->key, c->key_words * 8));
    uint64_t* stage = nullptr;
    TP_CUDA(cudaMalloc(&stage, c->key_words * 8));
    cudaError_t e = cudaMemcpy(stage, ksk, c->key_words * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        // each key: l rows of [A | B] (the reference's m_ksk) -> [row][c][jp][t][2]
        const uint64_t total = c->key_words;
        const uint64_t blocks = std::min<uint64_t>((total + 255) / 256, 65535);
        tp::key_relayout_kernel<<<(unsigned)blocks, 256>>>(c->key, stage, c->nkeys, 1, c->digits, c->logn,
                                                            c->loge, c->logs);
        tp::note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(stage);
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "key upload: %s", cudaGetErrorString(e));
    c->key_ready = true;
    return TP_OK;
}

static tp_status ks_launch(tp_ks_ctx* c, int mode, const tp::KsKernelParams& kp, cudaStream_t st) {
    tp::KsKernelParams p = kp;
    void* args[] = {&p};
    if (c->logs > 0) {
        // one item per cluster of 2^logs CTAs
        const uint64_t clusters = std::min<uint64_t>(kp.items, (uint64_t)c->cluster_cap[mode]);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr = {};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = 1u << c->logs;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)(clusters << c->logs));
        cfg.blockDim = dim3(c->N >> (c->logs + 2));
        cfg.dynamicSmemBytes = c->smem;
        cfg.stream = st;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        TP_CUDA(cudaLaunchKernelExC(&cfg, tp::ks_kernel_lookup(c->logn, mode, 2), args));
        tp::note_launch();
        return TP_OK;
    }
    const uint64_t grid =
        std::min<uint64_t>(kp.items, (uint64_t)c->per_sm[c->loge - 2][mode] * sm_count(c->device));
    TP_CUDA(cudaLaunchKernel(tp::ks_kernel_lookup(c->logn, mode, c->loge), dim3((unsigned)grid),
                             dim3(c->N >> c->loge), args, c->smem, st));
    tp::note_launch();
    return TP_OK;
}

tp_status tp_ks_set_tile(tp_ks_ctx* c, uint32_t coef_per_thread) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (coef_per_thread != 4 && coef_per_thread != 8) return fail(TP_ERR_PARAM, "tile must be 4 or 8");
    const int loge = coef_per_thread == 4 ? 2 : 3;
    std::lock_guard<std::mutex> lk(c->mu);
    if (loge == c->loge) return TP_OK;
    if (c->logs > 0) return fail(TP_ERR_PARAM, "ring sizes above 4096 run on clusters with 4 coefficients per thread");
    TP_CUDA(cudaSetDevice(c->device));
    if (c->key_ready) {
        uint64_t* nk = nullptr;
        TP_CUDA(cudaMalloc(&nk, c->key_words * 8));
        const uint64_t blocks = std::min<uint64_t>((c->key_words + 255) / 256, 65535);
        tp::key_retile_kernel<<<(unsigned)blocks, 256>>>(nk, c->key, c->nkeys, 1, c->digits, c->logn, c->loge, loge);
        tp::note_launch();
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            cudaFree(nk);
            return fail(TP_ERR_CUDA, "key re-tiling: %s", cudaGetErrorString(e));
        }
        cudaFree(c->key);
        c->key = nk;
    }
    c->loge = loge;
    return TP_OK;
}

uint32_t tp_ks_get_tile(const tp_ks_ctx* c) { return c ? 1u << c->loge : 0; }

tp_status tp_rlwe_ks_batch(tp_ks_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in, void* stream) {
    if (!c || c->kind != 0) return fail(TP_ERR_PARAM, "not an RLWE key-switching context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    TP_CUDA(cudaSetDevice(c->device));
    tp::KsKernelParams kp = c->kp;
    kp.key = c->key;
    kp.in = in;
    kp.out = out;
    kp.items = batch;
    kp.in_stride = kp.out_stride = 2ull * c->N;
    return ks_launch(c, tp::kKsRlwe, kp, (cudaStream_t)stream);
}

tp_status tp_auto_eval_batch(tp_ks_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in, void* stream) {
    if (!c || c->kind != 1) return fail(TP_ERR_PARAM, "not an automorphism context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    if (out == in) return fail(TP_ERR_PARAM, "automorphism output must not alias its input");
    TP_CUDA(cudaSetDevice(c->device));
    tp::KsKernelParams kp = c->kp;
    kp.key = c->key;
    kp.in = in;
    kp.out = out;
    kp.items = batch;
    kp.in_stride = kp.out_stride = 2ull * c->N;
    kp.auto_index = c->index;
    kp.auto_index_inv = inv_mod_2n(c->index, 2 * c->N);
    return ks_launch(c, tp::kKsAuto, kp, (cudaStream_t)stream);
}

// Trace steps j = j_hi down to j_lo over `items` RLWEs (coefficient domain, in
// place, `stride` words apart): x <- x + INTT(AutoKS_{2^j+1}(x)) with the
// packing context's key for index 2^j + 1 (lwe_to_rlwe_packing.cpp:228-234,
// trace_evaluation.cpp:145-153).
static tp_status ks_trace_steps(tp_ks_ctx* c, uint64_t items, uint64_t* data, uint64_t stride, int j_hi, int j_lo,
                                cudaStream_t st) {
    const uint64_t N = c->N;
    const uint64_t kw = (uint64_t)c->digits * 2 * N;
    tp::KsKernelParams kp = c->kp;
    for (int j = j_hi; j >= j_lo; --j) {
        kp.key = c->key + (uint64_t)(j - 1) * kw;
        kp.in = data;
        kp.out = data;
        kp.items = items;
        kp.in_stride = kp.out_stride = stride;
        kp.right_offset = 0;
        kp.auto_index = (1u << j) + 1;
        kp.auto_index_inv = inv_mod_2n(kp.auto_index, 2 * (uint32_t)N);
        kp.shift = 0;
        tp_status s = ks_launch(c, tp::kKsTrace, kp, st);
        if (s != TP_OK) return s;
    }
    return TP_OK;
}

static tp_status ntt_launch(uint32_t ring_dim, uint64_t count, uint64_t* out, const uint64_t* in, void* stream,
                            bool fwd, uint64_t in_stride, uint64_t out_stride);

tp_status tp_trace_eval_batch(tp_ks_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in, void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing (trace) context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t N = c->N, words = batch * 2 * N;
    // output = input * N^-1, then x += INTT(Auto_{2^j+1}(x)) for j = log2 N .. 1, then NTT of
    // both halves (trace_evaluation.cpp:135-158)
    tp::scale_kernel<<<(unsigned)std::min<uint64_t>((words + 255) / 256, 65535), 256, 0, st>>>(out, in, words,
                                                                                            c->tab->n_inv);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    tp_status s = ks_trace_steps(c, batch, out, 2 * N, c->logn, 1, st);
    if (s == TP_OK) s = ntt_launch((uint32_t)N, 2 * batch, out, out, stream, true, 0, 0);
    return s;
}

tp_status tp_trace_eval_auto_batch(tp_ks_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in,
                                   uint32_t auto_index, void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing (trace) context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    int j = 0;
    while (j <= c->logn && (1u << j) + 1 != auto_index) ++j;
    if (j < 1 || j > c->logn) return fail(TP_ERR_PARAM, "automorphism index must be 2^j + 1, 1 <= j <= log2 N");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    if (out == in) return fail(TP_ERR_PARAM, "automorphism output must not alias its input");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    tp::KsKernelParams kp = c->kp;
    kp.key = c->key + (uint64_t)(j - 1) * c->digits * 2 * c->N;
    kp.in = in;
    kp.out = out;
    kp.items = batch;
    kp.in_stride = kp.out_stride = 2ull * c->N;
    kp.auto_index = auto_index;
    kp.auto_index_inv = inv_mod_2n(auto_index, 2 * c->N);
    return ks_launch(c, tp::kKsAuto, kp, (cudaStream_t)stream);
}

// The compacted tree of LWEtoRLWEPacker::PackConsecutively (lwe_to_rlwe_packing.cpp:
// 260-393): a full tree over N leaves, leaf e holding input (N-1) ^ brv(e) when that is
// below len and an empty subtree otherwise; only nodes with an input below them are kept,
// a level's nodes in tree order. Level 0 lists the leaves' inputs, level l >= 1 one
// (left, right) pair of previous-level nodes per node (kNoNode: an empty subtree, zero).
static tp_status consec_plan(tp_ks_ctx* c, uint64_t len) {
    if (c->consec_len == len) return TP_OK;
    const uint64_t N = c->N;
    const int logn = c->logn;
    std::vector<uint32_t> plan;
    std::vector<uint64_t> off(logn + 1);
    std::vector<uint32_t> cnt(logn + 1);
    std::vector<int64_t> rank(N), next(N);
    off[0] = 0;
    for (uint64_t e = 0; e < N; ++e) {
        uint64_t r = 0;
        for (int b = 0; b < logn; ++b) r |= ((e >> b) & 1) << (logn - 1 - b);
        const uint64_t src = (N - 1) ^ r;
        rank[e] = src < len ? (int64_t)plan.size() : -1;
        if (src < len) plan.push_back((uint32_t)src);
    }
    cnt[0] = (uint32_t)plan.size();
    for (int l = 1; l <= logn; ++l) {
        off[l] = plan.size();
        uint32_t k = 0;
        for (uint64_t u = 0; u < (N >> l); ++u) {
            const int64_t a = rank[2 * u], b = rank[2 * u + 1];
            if (a < 0 && b < 0) {
                next[u] = -1;
                continue;
            }
            plan.push_back(a < 0 ? tp::kNoNode : (uint32_t)a);
            plan.push_back(b < 0 ? tp::kNoNode : (uint32_t)b);
            next[u] = k++;
        }
        cnt[l] = k;
        for (uint64_t u = 0; u < (N >> l); ++u) rank[u] = next[u];
    }
    cudaFree(c->consec_plan);
    c->consec_plan = nullptr;
    c->consec_len = 0;
    TP_CUDA(cudaMalloc(&c->consec_plan, plan.size() * 4));
    TP_CUDA(cudaMemcpy(c->consec_plan, plan.data(), plan.size() * 4, cudaMemcpyHostToDevice));
    if (!c->zero) {
        TP_CUDA(cudaMalloc(&c->zero, 2 * N * 8));
        TP_CUDA(cudaMemset(c->zero, 0, 2 * N * 8));
    }
    c->consec_off = off;
    c->consec_cnt = cnt;
    c->consec_len = len;
    return TP_OK;
}

tp_status tp_pack_consecutive_batch(tp_ks_ctx* c, uint64_t packs, uint64_t len, uint64_t* out, const uint64_t* in,
                                    void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (packs == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->N;
    if (len < 2 || len > N) return fail(TP_ERR_PARAM, "len must be in [2, N]");
    if (packs > (UINT64_MAX / 16) / (len * 2 * N))  // two halves of packs * len * 2N words must not wrap
        return fail(TP_ERR_PARAM, "packs * len * 2N words overflow (%llu packs of length %llu)",
                    (unsigned long long)packs, (unsigned long long)len);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    tp_status s = consec_plan(c, len);
    if (s != TP_OK) return s;
    const uint64_t half = packs * len * 2 * N;  // each level's nodes fit one half (at most len per pack)
    if (c->work_words < 2 * half) {
        cudaFree(c->work);
        c->work = nullptr;
        c->work_words = 0;
        TP_CUDA(cudaMalloc(&c->work, 2 * half * 8));
        c->work_words = 2 * half;
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t* buf[2] = {c->work, c->work + half};
    {
        const uint64_t total = packs * c->consec_cnt[0] * 2 * N;
        tp::pack_l0_idx_kernel<<<(unsigned)std::min<uint64_t>((total + 255) / 256, 65535), 256, 0, st>>>(
            buf[0], in, c->consec_plan, packs, c->consec_cnt[0], (uint32_t)len, (uint32_t)c->logn, c->tab->n_inv);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
    }
    const uint64_t kw = (uint64_t)c->digits * 2 * N;
    tp::KsKernelParams kp = c->kp;
    for (int l = 1; l <= c->logn; ++l) {
        kp.key = c->key + (uint64_t)(l - 1) * kw;
        kp.in = buf[(l - 1) & 1];
        kp.out = l == c->logn ? out : buf[l & 1];
        kp.items = packs * c->consec_cnt[l];
        kp.in_stride = kp.out_stride = 2 * N;
        kp.right_offset = 0;
        kp.pairs = c->consec_plan + c->consec_off[l];
        kp.zero = c->zero;
        kp.pair_count = c->consec_cnt[l];
        kp.prev_count = c->consec_cnt[l - 1];
        kp.auto_index = (1u << l) + 1;
        kp.auto_index_inv = inv_mod_2n(kp.auto_index, 2 * (uint32_t)N);
        kp.shift = (uint32_t)(N >> l);
        s = ks_launch(c, tp::kKsMerge, kp, st);
        if (s != TP_OK) return s;
    }
    return TP_OK;
}

// Merges of the packing tree (lwe_to_rlwe_packing.cpp:170-224) over `packs` regions
// of `count` nodes each (2N coefficient words per node, in tree position order, in
// place at `work`): relative level k = 1 .. log2(count) merges nodes 2^k q and
// 2^k q + 2^(k-1) of a region at absolute tree level L = level0 + k (automorphism
// key 2^L + 1, shift N >> L), leaving each region's root at its first node. The
// merge at a level depends on that level only, never on the node's place in the
// whole tree, so a subtree runs exactly like the bottom of a smaller tree.
static tp_status pack_merge_levels(tp_ks_ctx* c, uint64_t packs, uint64_t count, int level0, uint64_t* work,
                                   cudaStream_t st) {
    const uint64_t N = c->N;
    const uint64_t kw = (uint64_t)c->digits * 2 * N;
    tp::KsKernelParams kp = c->kp;
    const int levels = ilog2(count);
    for (int k = 1; k <= levels; ++k) {
        const int L = level0 + k;
        kp.key = c->key + (uint64_t)(L - 1) * kw;
        kp.in = work;
        kp.out = work;
        kp.items = packs * (count >> k);
        kp.in_stride = kp.out_stride = (1ull << k) * 2 * N;
        kp.right_offset = (1ull << (k - 1)) * 2 * N;
        kp.auto_index = (1u << L) + 1;
        kp.auto_index_inv = inv_mod_2n(kp.auto_index, 2 * (uint32_t)N);
        kp.shift = (uint32_t)(N >> L);
        tp_status s = ks_launch(c, tp::kKsMerge, kp, st);
        if (s != TP_OK) return s;
    }
    return TP_OK;
}

// The context's work area holds at least `words` words.
static tp_status pack_work(tp_ks_ctx* c, uint64_t words) {
    if (c->work_words < words) {
        cudaFree(c->work);
        c->work = nullptr;
        c->work_words = 0;
        TP_CUDA(cudaMalloc(&c->work, words * 8));
        c->work_words = words;
    }
    return TP_OK;
}

tp_status tp_pack_batch(tp_ks_ctx* c, uint64_t packs, uint64_t len, uint64_t* out, const uint64_t* in, void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (packs == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->N;
    if (len < 2 || len > N || (len & (len - 1))) return fail(TP_ERR_PARAM, "len must be a power of two in [2, N]");
    if (packs > (UINT64_MAX / 8) / (len * 2 * N))  // packs * len * 2N * 8 bytes must not wrap
        return fail(TP_ERR_PARAM, "packs * len * 2N words overflow (%llu packs of length %llu)",
                    (unsigned long long)packs, (unsigned long long)len);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    const uint64_t need = packs * len * 2 * N;
    {
        tp_status s = pack_work(c, need);
        if (s != TP_OK) return s;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int log_len = ilog2(len);
    {
        const uint64_t blocks = std::min<uint64_t>((need + 255) / 256, 65535 * 4ull);
        tp::pack_l0_kernel<<<(unsigned)std::min<uint64_t>(blocks, 65535), 256, 0, st>>>(
            c->work, in, packs, (uint32_t)len, (uint32_t)log_len, (uint32_t)c->logn, c->tab->n_inv);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
    }
    {
        tp_status s = pack_merge_levels(c, packs, len, 0, c->work, st);
        if (s != TP_OK) return s;
    }
    // trailing traces when len < N (lwe_to_rlwe_packing.cpp:228-234)
    {
        tp_status s = ks_trace_steps(c, packs, c->work, len * 2 * N, c->logn, log_len + 1, st);
        if (s != TP_OK) return s;
    }
    TP_CUDA(cudaMemcpy2DAsync(out, 2 * N * 8, c->work, len * 2 * N * 8, 2 * N * 8, packs, cudaMemcpyDeviceToDevice, st));
    return TP_OK;
}

// One shard of a packing split over several devices: the subtree of `len` inputs
// (L0 set-up and merges of levels 1 .. log2 len, no traces), its root left in the
// coefficient domain for tp_pack_merge_batch.
tp_status tp_pack_subtree_batch(tp_ks_ctx* c, uint64_t packs, uint64_t len, uint64_t* out, const uint64_t* in,
                                void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (packs == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->N;
    if (len < 1 || len > N || (len & (len - 1))) return fail(TP_ERR_PARAM, "len must be a power of two in [1, N]");
    if (packs > (UINT64_MAX / 8) / (len * 2 * N))
        return fail(TP_ERR_PARAM, "packs * len * 2N words overflow (%llu packs of length %llu)",
                    (unsigned long long)packs, (unsigned long long)len);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    const uint64_t need = packs * len * 2 * N;
    tp_status s = pack_work(c, need);
    if (s != TP_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    tp::pack_l0_kernel<<<(unsigned)std::min<uint64_t>((need + 255) / 256, 65535), 256, 0, st>>>(
        c->work, in, packs, (uint32_t)len, (uint32_t)ilog2(len), (uint32_t)c->logn, c->tab->n_inv);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    s = pack_merge_levels(c, packs, len, 0, c->work, st);
    if (s != TP_OK) return s;
    TP_CUDA(cudaMemcpy2DAsync(out, 2 * N * 8, c->work, len * 2 * N * 8, 2 * N * 8, packs, cudaMemcpyDeviceToDevice, st));
    return TP_OK;
}

// The tree above `count` subtree roots of level `level0` (position order), then, with
// `finish`, the trailing traces of levels level0 + log2(count) + 1 .. log2 N.
tp_status tp_pack_merge_batch(tp_ks_ctx* c, uint64_t packs, uint64_t count, uint32_t level0, int finish,
                              uint64_t* out, const uint64_t* nodes, void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (packs == 0) return TP_OK;
    if (!out || !nodes) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->N;
    if (count < 1 || count > N || (count & (count - 1)))
        return fail(TP_ERR_PARAM, "count must be a power of two in [1, N]");
    const int top = (int)level0 + ilog2(count);
    if (top > c->logn) return fail(TP_ERR_PARAM, "level0 + log2(count) must not exceed log2 N");
    if (packs > (UINT64_MAX / 8) / (count * 2 * N))
        return fail(TP_ERR_PARAM, "packs * count * 2N words overflow (%llu packs of %llu nodes)",
                    (unsigned long long)packs, (unsigned long long)count);
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    const uint64_t need = packs * count * 2 * N;
    tp_status s = pack_work(c, need);
    if (s != TP_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    TP_CUDA(cudaMemcpyAsync(c->work, nodes, need * 8, cudaMemcpyDeviceToDevice, st));
    s = pack_merge_levels(c, packs, count, (int)level0, c->work, st);
    if (s != TP_OK) return s;
    if (finish) {
        s = ks_trace_steps(c, packs, c->work, count * 2 * N, c->logn, top + 1, st);
        if (s != TP_OK) return s;
    }
    TP_CUDA(cudaMemcpy2DAsync(out, 2 * N * 8, c->work, count * 2 * N * 8, 2 * N * 8, packs, cudaMemcpyDeviceToDevice,
                              st));
    return TP_OK;
}

// ---------------------------------------------------------------------------
// LWE -> LWE key switching
// ---------------------------------------------------------------------------
struct tp_lwe_ks_ctx {
    int device = 0;
    uint32_t n_in = 0, n_out = 0, digits = 0;
    uint64_t basis = 0;
    uint64_t key_words = 0;
    uint64_t* key = nullptr;
    uint64_t* cterm = nullptr;    // n_out + 1 words, from the key (see lwe_ks_kernel)
    bool key_ready = false;
    tp::LweKsParams kp{};
};

tp_status tp_lwe_ks_create(uint64_t modulus, uint32_t n_in, uint32_t n_out, uint64_t basis, uint32_t digits,
                           int device, tp_lwe_ks_ctx** out) {
    if (!out) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (modulus != kP) return fail(TP_ERR_PARAM, "the GPU LWE key switch runs on the Goldilocks modulus only");
    if (n_in == 0 || n_out == 0) return fail(TP_ERR_PARAM, "dimensions must be positive");
    if (basis < 2 || (basis & (basis - 1))) return fail(TP_ERR_PARAM, "basis must be a power of two");
    const int beta = ilog2(basis);
    if (beta > 30) return fail(TP_ERR_PARAM, "basis above 2^30 is not supported");
    // LWEtoLWEConverter::Convert shifts by 64 - beta - j*beta for every digit j
    // (lwe_conversion.cpp:226-236); every shift must stay non-negative.
    if (digits < 1 || digits > 8 || (uint64_t)digits * beta > 64)
        return fail(TP_ERR_PARAM, "digits * log2(basis) must be at most 64 (and digits at most 8)");
    if ((uint64_t)n_in * digits > (1ull << 30))
        return fail(TP_ERR_PARAM, "n_in * digits above 2^30 is not supported");
    auto* c = new tp_lwe_ks_ctx();
    c->device = device;
    c->n_in = n_in;
    c->n_out = n_out;
    c->digits = digits;
    c->basis = basis;
    c->key_words = (uint64_t)n_in * digits * (n_out + 1);
    tp::LweKsParams& kp = c->kp;
    kp.n_in = n_in;
    kp.n_out = n_out;
    kp.digits = digits;
    const int max_digits = (64 + beta - 1) / beta;
    uint64_t corr = 0;
    int64_t shift = 64 - beta;
    while (shift > 0) {
        corr += 1ull << (shift + beta - 1);
        shift -= beta;
    }
    const uint64_t least = 1ull << (shift + beta - 1);
    corr += least;
    kp.corr = corr % kP;
    for (uint32_t j = 0; j < digits; ++j) {
        kp.dshift[j] = (uint32_t)(64 - beta - (int)j * beta);
        kp.dmask[j] = (1ull << beta) - 1;
        kp.ddelta[j] = (int)j != max_digits - 1 ? 1ull << (beta - 1) : least;
    }
    *out = c;
    return TP_OK;
}

tp_status tp_lwe_ks_destroy(tp_lwe_ks_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    cudaFree(c->key);
    cudaFree(c->cterm);
    delete c;
    return TP_OK;
}

uint64_t tp_lwe_ks_key_words(const tp_lwe_ks_ctx* c) { return c ? c->key_words : 0; }

tp_status tp_lwe_ks_upload_key(tp_lwe_ks_ctx* c, const uint64_t* ksk, uint64_t words) {
    if (!c || !ksk) return fail(TP_ERR_PARAM, "null argument");
    if (words != c->key_words)
        return fail(TP_ERR_LAYOUT, "key has %llu words, context expects %llu", (unsigned long long)words,
                    (unsigned long long)c->key_words);
    TP_CUDA(cudaSetDevice(c->device));
    c->key_ready = false;
    if (!c->key) TP_CUDA(cudaMalloc(&c->key, c->key_words * 8));
    if (!c->cterm) TP_CUDA(cudaMalloc(&c->cterm, ((uint64_t)c->n_out + 1) * 8));
    TP_CUDA(cudaMemcpy(c->key, ksk, c->key_words * 8, cudaMemcpyHostToDevice));
    tp::LweKsParams kp = c->kp;
    kp.ksk = c->key;
    const unsigned blocks = (c->n_out + 1 + 31) / 32;
    tp::lwe_ks_cterm_kernel<<<blocks, dim3(32, tp::kCtermSlices)>>>(c->cterm, kp);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    TP_CUDA(cudaDeviceSynchronize());
    c->kp.cterm = c->cterm;
    c->key_ready = true;
    return TP_OK;
}

tp_status tp_lwe_ks_batch(tp_lwe_ks_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    if (batch > 65535ull * tp::kLweKsRows) return fail(TP_ERR_PARAM, "batch too large for one launch");
    TP_CUDA(cudaSetDevice(c->device));
    tp::LweKsParams kp = c->kp;
    kp.ksk = c->key;
    kp.in = in;
    kp.out = out;
    kp.batch = batch;
    dim3 grid((c->n_out + 1 + tp::kLweKsCols - 1) / tp::kLweKsCols,
              (unsigned)((batch + tp::kLweKsRows - 1) / tp::kLweKsRows));
    tp::lwe_ks_kernel<<<grid, tp::kLweKsCols, 0, (cudaStream_t)stream>>>(kp);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Modulus switch and the bootstrap epilogue
// ---------------------------------------------------------------------------
static int pow2_log2(uint64_t t) {
    if (t < 2 || (t & (t - 1)) || t > (1ull << 32)) return 0;
    return ilog2(t);
}

tp_status tp_modulus_switch_batch(uint64_t count, uint64_t* vec, uint64_t source_modulus, uint64_t target_modulus,
                                  int type, void* stream) {
    if (source_modulus != kP) return fail(TP_ERR_PARAM, "the GPU modulus switch takes the Goldilocks modulus as source");
    const int k = pow2_log2(target_modulus);
    if (!k) return fail(TP_ERR_PARAM, "target modulus must be a power of two in [2, 2^32]");
    if (type != TP_MS_ROUND && type != TP_MS_FLOOR && type != TP_MS_CEIL)
        return fail(TP_ERR_PARAM, "type must be TP_MS_ROUND, TP_MS_FLOOR or TP_MS_CEIL");
    if (count == 0) return TP_OK;
    if (!vec) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t blocks = std::min<uint64_t>((count + 255) / 256, 65535);
    tp::ms_pow2_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(vec, count, (uint32_t)k, type);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

tp_status tp_pbs_epilogue_batch(tp_lwe_ks_ctx* c, uint64_t batch, uint64_t* out_lwe, const uint64_t* rlwe_coef,
                                uint64_t target_modulus, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (c->n_in < 2 || (c->n_in & (c->n_in - 1)))
        return fail(TP_ERR_PARAM, "the key switch's input dimension must be the ring dimension N (a power of two)");
    const int k = pow2_log2(target_modulus);
    if (!k) return fail(TP_ERR_PARAM, "target modulus must be a power of two in [2, 2^32]");
    if (batch == 0) return TP_OK;
    if (!out_lwe || !rlwe_coef) return fail(TP_ERR_PARAM, "null buffer");
    if (batch > 65535ull * tp::kLweKsRows) return fail(TP_ERR_PARAM, "batch too large for one launch");
    TP_CUDA(cudaSetDevice(c->device));
    tp::LweKsParams kp = c->kp;
    kp.ksk = c->key;
    kp.in = rlwe_coef;
    kp.out = out_lwe;
    kp.batch = batch;
    kp.rlwe_in = 1;
    kp.ms_log2 = (uint32_t)k;
    dim3 grid((c->n_out + 1 + tp::kLweKsCols - 1) / tp::kLweKsCols,
              (unsigned)((batch + tp::kLweKsRows - 1) / tp::kLweKsRows));
    tp::lwe_ks_kernel<<<grid, tp::kLweKsCols, 0, (cudaStream_t)stream>>>(kp);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

tp_status tp_pbs_graph_create(tp_br_ctx* br, tp_lwe_ks_ctx* ks, uint64_t batch, uint64_t* rlwe_scratch,
                              const uint64_t* lwes, const uint64_t* accs, uint64_t acc_stride, uint64_t* out_lwe,
                              tp_graph** out) {
    if (!br || !ks || !out) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    if (batch == 0) return fail(TP_ERR_PARAM, "empty batch");
    if (ks->n_in != br->prm.ring_dim)
        return fail(TP_ERR_PARAM, "the key switch's input dimension (%u) must be the rotation's ring dimension (%u)",
                    ks->n_in, br->prm.ring_dim);
    if (ks->device != br->device) return fail(TP_ERR_PARAM, "contexts live on different devices");
    TP_CUDA(cudaSetDevice(br->device));
    cudaStream_t s = nullptr;
    TP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(s);
        return fail(TP_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    ++tp::t_capturing;
    tp_status st = tp_br_blind_rotate_batch(br, batch, rlwe_scratch, lwes, (uint64_t)br->prm.lwe_dim + 1, accs,
                                            acc_stride, 1, s);
    if (st == TP_OK) st = tp_pbs_epilogue_batch(ks, batch, out_lwe, rlwe_scratch, 2ull * br->prm.ring_dim, s);
    --tp::t_capturing;
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    cudaStreamDestroy(s);
    if (st != TP_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    auto* gr = new tp_graph();
    gr->device = br->device;
    gr->kernels = graph_kernel_nodes(g);
    e = cudaGraphInstantiate(&gr->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        delete gr;
        return fail(TP_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
    }
    *out = gr;
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Key files (format in keyfile.cu): header checked against the context, then
// the payload read, hashed and uploaded like a key from memory
// ---------------------------------------------------------------------------
static tp_status key_file_payload(const char* path, const tp_key_info& want, std::vector<uint64_t>& words) {
    tp_key_info got{};
    tp_status s = tp_key_file_info(path, &got);
    if (s != TP_OK) return s;
    if (got.kind != want.kind || got.variant != want.variant || got.ring_dim != want.ring_dim ||
        got.lwe_dim != want.lwe_dim || got.digits != want.digits || got.modulus != want.modulus ||
        got.basis != want.basis || got.index != want.index || got.words != want.words)
        return fail(TP_ERR_LAYOUT,
                    "%s: key for kind %u variant %u N %u n %u digits %u basis %llu index %u (%llu words); the context "
                    "needs kind %u variant %u N %u n %u digits %u basis %llu index %u (%llu words)",
                    path, got.kind, got.variant, got.ring_dim, got.lwe_dim, got.digits,
                    (unsigned long long)got.basis, got.index, (unsigned long long)got.words, want.kind, want.variant,
                    want.ring_dim, want.lwe_dim, want.digits, (unsigned long long)want.basis, want.index,
                    (unsigned long long)want.words);
    words.resize(got.words);
    return tp_key_file_read(path, &got, words.data(), words.size());
}

tp_status tp_br_upload_key_file(tp_br_ctx* c, const char* path) {
    if (!c || !path) return fail(TP_ERR_PARAM, "null argument");
    tp_key_info want{};
    want.kind = TP_KEY_BLIND_ROTATION;
    want.variant = (uint32_t)c->prm.variant;
    want.ring_dim = c->prm.ring_dim;
    want.lwe_dim = c->prm.lwe_dim;
    want.digits = c->prm.digits;
    want.modulus = c->prm.modulus;
    want.basis = c->prm.basis;
    want.words = c->key_words;
    std::vector<uint64_t> w;
    tp_status s = key_file_payload(path, want, w);
    return s == TP_OK ? tp_br_upload_key(c, w.data(), w.size()) : s;
}

tp_status tp_ks_upload_key_file(tp_ks_ctx* c, const char* path) {
    if (!c || !path) return fail(TP_ERR_PARAM, "null argument");
    tp_key_info want{};
    want.kind = c->kind == 0 ? TP_KEY_RLWE_SWITCH : (c->kind == 1 ? TP_KEY_AUTOMORPHISM : TP_KEY_PACKING);
    want.ring_dim = c->N;
    want.digits = c->digits;
    want.modulus = kP;
    want.basis = c->basis;
    want.index = c->kind == 1 ? c->index : 0;
    want.words = c->key_words;
    std::vector<uint64_t> w;
    tp_status s = key_file_payload(path, want, w);
    return s == TP_OK ? tp_ks_upload_key(c, w.data(), w.size()) : s;
}

tp_status tp_lwe_ks_upload_key_file(tp_lwe_ks_ctx* c, const char* path) {
    if (!c || !path) return fail(TP_ERR_PARAM, "null argument");
    tp_key_info want{};
    want.kind = TP_KEY_LWE_SWITCH;
    want.ring_dim = c->n_in;
    want.lwe_dim = c->n_out;
    want.digits = c->digits;
    want.modulus = kP;
    want.basis = c->basis;
    want.words = c->key_words;
    std::vector<uint64_t> w;
    tp_status s = key_file_payload(path, want, w);
    return s == TP_OK ? tp_lwe_ks_upload_key(c, w.data(), w.size()) : s;
}

static tp_status ntt_launch(uint32_t ring_dim, uint64_t count, uint64_t* out, const uint64_t* in, void* stream,
                            bool fwd, uint64_t in_stride = 0, uint64_t out_stride = 0) {
    if (ring_dim < 128 || ring_dim > 65536 || (ring_dim & (ring_dim - 1)))
        return fail(TP_ERR_PARAM, "ring_dim must be a power of two in [128, 65536]");
    if (count == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    if (((uintptr_t)out & 15) || ((uintptr_t)in & 15)) return fail(TP_ERR_PARAM, "buffers must be 16-byte aligned");
    int device = 0;
    TP_CUDA(cudaGetDevice(&device));
    const int logn = ilog2(ring_dim);
    const Tables* tab = nullptr;
    tp_status s = get_tables(device, logn, &tab);
    if (s != TP_OK) return s;
    const void* k = tp::ntt_kernel_lookup(logn, fwd);
    if (!in_stride) in_stride = ring_dim;
    if (!out_stride) out_stride = ring_dim;
    const int logs = tp::br_cluster_logs(logn);
    if (logs > 0) {
        // one polynomial per cluster of 2^logs CTAs of N / 2^(logs+2) threads; shared
        // memory: 5 NL words (NL = N / 2^logs)
        const unsigned S = 1u << logs;
        const size_t smem = 5ull * (ring_dim >> logs) * 8;
        TP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (S > 8) TP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr = {};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = S;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(S * (unsigned)sm_count(device));
        cfg.blockDim = dim3(ring_dim >> (logs + 2));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = (cudaStream_t)stream;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        TP_CUDA(cudaOccupancyMaxActiveClusters(&clusters, k, &cfg));
        if (clusters < 1) return fail(TP_ERR_CUDA, "NTT cluster kernel (N=%u): no resident cluster", ring_dim);
        cfg.gridDim = dim3((unsigned)(std::min<uint64_t>(count, (uint64_t)clusters) << logs));
        const uint64_t* tw = fwd ? tab->tw_fwd : tab->tw_inv;
        uint64_t n_inv = tab->n_inv;
        void* args[] = {&out, &in, &count, &tw, &n_inv, &in_stride, &out_stride};
        TP_CUDA(cudaLaunchKernelExC(&cfg, k, args));
        tp::note_launch();
        return TP_OK;
    }
    const size_t smem = 3ull * ring_dim * 8;
    TP_CUDA(cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k, ring_dim / 8, smem));
    const uint64_t grid = std::min<uint64_t>(count, (uint64_t)std::max(1, per_sm) * sm_count(device));
    const uint64_t* tw = fwd ? tab->tw_fwd : tab->tw_inv;
    uint64_t n_inv = tab->n_inv;
    void* args[] = {&out, &in, &count, &tw, &n_inv, &in_stride, &out_stride};
    TP_CUDA(cudaLaunchKernel(k, dim3((unsigned)grid), dim3(ring_dim / 8), args, smem, (cudaStream_t)stream));
    tp::note_launch();
    return TP_OK;
}

tp_status tp_ntt_forward(uint32_t ring_dim, uint64_t count, uint64_t* out, const uint64_t* in, void* stream) {
    return ntt_launch(ring_dim, count, out, in, stream, true);
}

tp_status tp_ntt_backward(uint32_t ring_dim, uint64_t count, uint64_t* out, const uint64_t* in, void* stream) {
    return ntt_launch(ring_dim, count, out, in, stream, false);
}

// A rotation launch inside a composite operator: two blocks per rotation when the
// whole batch fits the two-block kernel's resident grid (small batches finish in
// about half the time), else one. The four-block form is not chosen here: its
// latency gain (15-30% more) costs 1.7x the two-block form's SM-time.
static tp_status br_rotate_auto(tp_br_ctx* br, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef,
                                void* stream) {
    const int split = batch <= tp::br_concurrency(br, 2) ? 2 : 1;
    return tp::br_batch_launch(br, batch, results, lwes, lwe_stride, accs, acc_stride, out_coef, stream, split);
}

// ---------------------------------------------------------------------------
// LWE -> RGSW scheme switching (lib/src/operators/lwe_to_rgsw_conversion.cpp)
// ---------------------------------------------------------------------------
struct tp_ss_ctx {
    int device = 0;
    uint32_t N = 0, n = 0, D = 0, logn = 0;
    tp_br_ctx* br = nullptr;      // CGGI binary rotation
    tp_ks_ctx* trace = nullptr;   // packing-kind context: automorphism keys 2^j + 1, j = 1..log2 N
    tp_ks_ctx* sq = nullptr;      // RLWE key switch s^2 -> s
    std::vector<uint64_t> acc_host;  // the converter's m_acc: [0 | -tp | tp], 3N words
    uint64_t* acc = nullptr;      // device copy
    uint64_t *rot = nullptr, *rows = nullptr, *sqin = nullptr, *sqout = nullptr;
    uint64_t cap = 0;             // ciphertexts the scratch holds
    bool ready = false;
    std::mutex mu;
};

// The test polynomial of LWEtoRGSWConverter's constructor (lines 120-160), in the
// reference's own integer arithmetic (the first scale is an int shift there).
static bool ss_test_polynomial(uint32_t N, uint32_t D, int basebits, std::vector<uint64_t>& acc) {
    const uint64_t bs = N / D;
    const uint64_t max_digits = (uint64_t)std::ceil(std::log2((long double)kP) / (long double)basebits);
    const uint64_t sh = (uint64_t)basebits * (max_digits - D);
    if (max_digits < D || sh >= 31) return false;
    uint64_t scale = (uint64_t)(1 << sh);
    acc.assign(3ull * N, 0);
    for (uint64_t i = 0; i < bs / 2; ++i) {
        acc[N + i] = scale;
        acc[2 * N - i - 1] = kP - scale;
    }
    for (uint64_t b = 1; b < D; ++b) {
        scale <<= basebits;
        for (uint64_t j = 0; j < bs; ++j) acc[N + b * bs + j - bs / 2] = scale;
    }
    const uint64_t two_inv = hinv(2);
    for (uint64_t i = 0; i < N; ++i) acc[N + i] = hmul(acc[N + i] % kP, two_inv);
    for (uint64_t i = 0; i < N; ++i) acc[2 * N + i] = acc[N + i];
    for (uint64_t i = 0; i < N; ++i) acc[N + i] = hmul(acc[2 * N + i], kP - 1);
    return true;
}

tp_status tp_ss_destroy(tp_ss_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    tp_br_destroy(c->br);
    tp_ks_destroy(c->trace);
    tp_ks_destroy(c->sq);
    cudaFree(c->acc);
    cudaFree(c->rot);
    cudaFree(c->rows);
    cudaFree(c->sqin);
    cudaFree(c->sqout);
    delete c;
    return TP_OK;
}

tp_status tp_ss_create(const tp_br_params* rotation, uint64_t trace_basis, uint32_t trace_digits,
                       uint64_t square_basis, uint32_t square_digits, uint32_t out_digits, uint64_t out_basis,
                       int device, tp_ss_ctx** out) {
    if (!out || !rotation) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    const uint32_t ring_dim = rotation->ring_dim, lwe_dim = rotation->lwe_dim;
    if (out_digits < 1 || (ring_dim % out_digits) || ((ring_dim / out_digits) & 1))
        return fail(TP_ERR_PARAM, "out_digits must divide N into blocks of even size");
    if (out_basis < 2 || (out_basis & (out_basis - 1))) return fail(TP_ERR_PARAM, "out_basis must be a power of two");
    auto* c = new tp_ss_ctx();
    c->device = device;
    c->N = ring_dim;
    c->n = lwe_dim;
    c->D = out_digits;
    c->logn = ilog2(ring_dim);
    if (!ss_test_polynomial(ring_dim, out_digits, ilog2(out_basis), c->acc_host)) {
        delete c;
        return fail(TP_ERR_PARAM, "output gadget (out_digits, out_basis) not supported: its first scale overflows");
    }
    tp_status s = tp_br_create(rotation, device, &c->br);
    if (s == TP_OK) s = tp_pack_create(ring_dim, trace_basis, trace_digits, device, &c->trace);
    if (s == TP_OK) s = tp_rlwe_ks_create(ring_dim, square_basis, square_digits, device, &c->sq);
    if (s != TP_OK) {
        tp_ss_destroy(c);
        return s;
    }
    cudaError_t e = cudaMalloc(&c->acc, c->acc_host.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(c->acc, c->acc_host.data(), c->acc_host.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        tp_ss_destroy(c);
        return fail(TP_ERR_CUDA, "test polynomial: %s", cudaGetErrorString(e));
    }
    *out = c;
    return TP_OK;
}

uint64_t tp_ss_key_words(const tp_ss_ctx* c, int which) {
    if (!c) return 0;
    return which == 0 ? tp_br_key_words(c->br) : tp_ks_key_words(which == 1 ? c->trace : c->sq);
}

tp_status tp_ss_upload_keys(tp_ss_ctx* c, const uint64_t* brk, uint64_t brk_words, const uint64_t* trace_keys,
                            uint64_t trace_words, const uint64_t* square_key, uint64_t square_words) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->ready = false;
    tp_status s = tp_br_upload_key(c->br, brk, brk_words);
    if (s == TP_OK) s = tp_ks_upload_key(c->trace, trace_keys, trace_words);
    if (s == TP_OK) s = tp_ks_upload_key(c->sq, square_key, square_words);
    if (s == TP_OK) c->ready = true;
    return s;
}

tp_status tp_ss_accumulator(const tp_ss_ctx* c, uint64_t* out_host) {
    if (!c || !out_host) return fail(TP_ERR_PARAM, "null argument");
    std::copy(c->acc_host.begin(), c->acc_host.end(), out_host);
    return TP_OK;
}

tp_status tp_lwe_to_rgsw_batch(tp_ss_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* lwes, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->ready) return fail(TP_ERR_STATE, "keys not uploaded");
    if (batch == 0) return TP_OK;
    if (!out || !lwes) return fail(TP_ERR_PARAM, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    const uint64_t N = c->N, D = c->D;
    if (c->cap < batch) {
        cudaFree(c->rot);
        cudaFree(c->rows);
        cudaFree(c->sqin);
        cudaFree(c->sqout);
        c->rot = c->rows = c->sqin = c->sqout = nullptr;
        c->cap = 0;
        TP_CUDA(cudaMalloc(&c->rot, batch * 2 * N * 8));
        TP_CUDA(cudaMalloc(&c->rows, batch * D * 2 * N * 8));
        TP_CUDA(cudaMalloc(&c->sqin, batch * D * 2 * N * 8));
        TP_CUDA(cudaMalloc(&c->sqout, batch * D * 2 * N * 8));
        c->cap = batch;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t rowsn = batch * D;
    const uint64_t total = rowsn * 2 * N;
    const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 65535);
    // 1. rotation of [0 | -tp] with coefficient output (line 178)
    tp_status s = br_rotate_auto(c->br, batch, c->rot, lwes, (uint64_t)c->n + 1, c->acc, 0, 1, stream);
    if (s != TP_OK) return s;
    // 2. + (0, tp), Lev rows, times N^-1 (lines 180-200; trace_evaluation.cpp:143)
    tp::ss_rows_kernel<<<blocks, 256, 0, st>>>(c->rows, c->rot, c->acc + 2 * N, batch, (uint32_t)ilog2(D),
                                                 c->logn, (uint32_t)(N / D), c->br->tab->n_inv);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    // 3. trace: automorphisms N+1 down to 3 (trace_evaluation.cpp:145-153), then NTT of both halves
    s = ks_trace_steps(c->trace, rowsn, c->rows, 2 * N, (int)c->logn, 1, st);
    if (s != TP_OK) return s;
    s = ntt_launch((uint32_t)N, 2 * rowsn, c->rows, c->rows, stream, true);
    if (s != TP_OK) return s;
    // 4. squaring input [INTT(row.A) | 0], key switch s^2 -> s into zero rows (lines 212-216)
    s = ntt_launch((uint32_t)N, rowsn, c->sqin, c->rows, stream, false, 2 * N, 2 * N);
    if (s != TP_OK) return s;
    TP_CUDA(cudaMemset2DAsync(c->sqin + N, 2 * N * 8, 0, N * 8, rowsn, st));
    TP_CUDA(cudaMemsetAsync(c->sqout, 0, total * 8, st));
    s = tp_rlwe_ks_batch(c->sq, rowsn, c->sqout, c->sqin, stream);
    if (s != TP_OK) return s;
    // 5. RGSW = [lev_left | lev_right] (lines 218-224)
    tp::ss_assemble_kernel<<<blocks, 256, 0, st>>>(out, c->rows, c->sqout, batch, (uint32_t)ilog2(D), c->logn);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

// ---------------------------------------------------------------------------
// SAP digit decomposition (lib/src/operators/sap_decomposer.cpp)
// ---------------------------------------------------------------------------
struct tp_sap_ctx {
    int device = 0;
    uint32_t N = 0, n = 0, logn = 0;
    tp_br_ctx* br = nullptr;          // rotation of any variant
    tp_ks_ctx* trace = nullptr;       // automorphism keys 2^j + 1, j = 1..log2 N
    tp_lwe_ks_ctx* lks = nullptr;     // LWE key switch N -> n (the reset)
    bool ready = false;
    // constants: [extract poly | pad poly | overflow poly] in the NTT domain, fresh acc (0, Q/2N)
    uint64_t* consts = nullptr;
    uint64_t* fresh = nullptr;
    uint64_t radix = 0;               // radix the constants were made for
    // scratch, sized for `cap` LWEs and `leaves` tree leaves per LWE
    uint64_t *copy = nullptr, *sub = nullptr, *modulus = nullptr, *acc = nullptr, *ext = nullptr, *lw = nullptr,
             *tree = nullptr;
    uint8_t* flags = nullptr;
    uint64_t cap = 0, leaves = 0;
    std::mutex mu;
};

tp_status tp_sap_destroy(tp_sap_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    tp_br_destroy(c->br);
    tp_ks_destroy(c->trace);
    tp_lwe_ks_destroy(c->lks);
    for (void* p : {(void*)c->consts, (void*)c->fresh, (void*)c->copy, (void*)c->sub, (void*)c->modulus,
                    (void*)c->acc, (void*)c->ext, (void*)c->lw, (void*)c->tree, (void*)c->flags})
        cudaFree(p);
    delete c;
    return TP_OK;
}

tp_status tp_sap_create(const tp_br_params* rotation, uint64_t trace_basis, uint32_t trace_digits, uint64_t ks_basis,
                        uint32_t ks_digits, int device, tp_sap_ctx** out) {
    if (!out || !rotation) return fail(TP_ERR_PARAM, "null argument");
    *out = nullptr;
    auto* c = new tp_sap_ctx();
    c->device = device;
    c->N = rotation->ring_dim;
    c->n = rotation->lwe_dim;
    tp_status s = tp_br_create(rotation, device, &c->br);
    if (s == TP_OK) {
        c->logn = ilog2(c->N);
        s = tp_pack_create(c->N, trace_basis, trace_digits, device, &c->trace);
    }
    if (s == TP_OK) s = tp_lwe_ks_create(kP, c->N, c->n, ks_basis, ks_digits, device, &c->lks);
    if (s != TP_OK) {
        tp_sap_destroy(c);
        return s;
    }
    std::vector<uint64_t> fresh(2ull * c->N, 0);
    fresh[c->N] = kP / (2ull * c->N);
    cudaError_t e = cudaMalloc(&c->fresh, fresh.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(c->fresh, fresh.data(), fresh.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&c->consts, 4ull * c->N * 8);
    if (e != cudaSuccess) {
        tp_sap_destroy(c);
        return fail(TP_ERR_CUDA, "SAP constants: %s", cudaGetErrorString(e));
    }
    *out = c;
    return TP_OK;
}

uint64_t tp_sap_key_words(const tp_sap_ctx* c, int which) {
    if (!c) return 0;
    if (which == 0) return tp_br_key_words(c->br);
    if (which == 1) return tp_ks_key_words(c->trace);
    return tp_lwe_ks_key_words(c->lks);
}

tp_status tp_sap_upload_keys(tp_sap_ctx* c, const uint64_t* brk, uint64_t brk_words, const uint64_t* trace_keys,
                             uint64_t trace_words, const uint64_t* lwe_ksk, uint64_t lwe_ksk_words) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->ready = false;
    tp_status s = tp_br_upload_key(c->br, brk, brk_words);
    if (s == TP_OK) s = tp_ks_upload_key(c->trace, trace_keys, trace_words);
    if (s == TP_OK) s = tp_lwe_ks_upload_key(c->lks, lwe_ksk, lwe_ksk_words);
    if (s == TP_OK) c->ready = true;
    return s;
}

// Constants for `radix` (NTT domain): the extraction polynomial x -> x mod radix,
// reversed (lines 394-399), the truncation pad sum_{i<radix} X^(i-(radix-1))
// (lines 212-217), and the reset's overflow polynomial -((N-i) >> r << r) at X^i
// (lines 320-324) for r = IntLog2(0) = 0, as Decompose passes radix 0, and for
// r = IntLog2(radix).
static tp_status sap_constants(tp_sap_ctx* c, uint64_t radix, cudaStream_t st) {
    if (c->radix == radix) return TP_OK;
    const uint64_t N = c->N;
    const int r = ilog2(radix);
    std::vector<uint64_t> h(4 * N, 0);
    for (uint64_t i = 1; i < N; ++i) h[N - i] = (kP - (i & (radix - 1))) % kP;
    for (uint64_t i = N - (radix - 1); i < N; ++i) h[N + i] = kP - 1;
    h[N] = 1;
    for (uint64_t i = 1; i < N; ++i) h[2 * N + i] = kP - (N - i);
    for (uint64_t i = 1; i < N; ++i) h[3 * N + i] = (kP - (((N - i) >> r) << r)) % kP;
    TP_CUDA(cudaMemcpyAsync(c->consts, h.data(), h.size() * 8, cudaMemcpyHostToDevice, st));
    tp_status s = ntt_launch((uint32_t)N, 4, c->consts, c->consts, st, true);
    if (s != TP_OK) return s;
    TP_CUDA(cudaStreamSynchronize(st));
    c->radix = radix;
    return TP_OK;
}

static unsigned sap_blocks(uint64_t work) { return (unsigned)std::min<uint64_t>((work + 255) / 256, 65535); }

// Scratch for `batch` LWEs and trees of `leaves` leaves.
static tp_status sap_reserve(tp_sap_ctx* c, uint64_t batch, uint64_t leaves) {
    if (c->cap >= batch && c->leaves >= leaves) return TP_OK;
    const uint64_t N = c->N, n = c->n;
    const uint64_t B = std::max(batch, c->cap), Lv = std::max(leaves, c->leaves);
    for (void* p : {(void*)c->copy, (void*)c->sub, (void*)c->modulus, (void*)c->acc, (void*)c->ext, (void*)c->lw,
                    (void*)c->tree, (void*)c->flags})
        cudaFree(p);
    c->copy = c->sub = c->modulus = c->acc = c->ext = c->lw = c->tree = nullptr;
    c->flags = nullptr;
    c->cap = c->leaves = 0;
    TP_CUDA(cudaMalloc(&c->copy, B * (n + 1) * 8));
    TP_CUDA(cudaMalloc(&c->sub, B * (n + 1) * 8));
    TP_CUDA(cudaMalloc(&c->lw, B * (n + 1) * 8));
    TP_CUDA(cudaMalloc(&c->modulus, B * 8));
    TP_CUDA(cudaMalloc(&c->flags, B));
    TP_CUDA(cudaMalloc(&c->acc, B * 2 * N * 8));
    TP_CUDA(cudaMalloc(&c->ext, B * 2 * N * 8));
    TP_CUDA(cudaMalloc(&c->tree, B * Lv * 2 * N * 8));
    c->cap = B;
    c->leaves = Lv;
    return TP_OK;
}

// HomTrunc (lines 189-291) of `batch` NTT-domain RLWEs into coefficient-domain
// results: N^-1 and the pad, INTT, the partial trace over N+1 .. 2^(L+1)+1, the
// truncation tree level by level (kKsSplit), the leaf sum. Uses c->tree.
static tp_status sap_trunc(tp_sap_ctx* c, uint64_t batch, const uint64_t* in_ntt, uint64_t* out_coef, uint64_t radix,
                           cudaStream_t st) {
    const uint64_t N = c->N;
    const uint32_t L = c->logn - (uint32_t)ilog2(radix);
    const uint64_t S = (2 * N) << L;  // words of one LWE's tree
    tp::sap_mul_poly_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(c->tree, S, in_ntt, c->consts + N,
                                                                     c->br->tab->n_inv, batch, c->logn);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    tp_status s = ntt_launch((uint32_t)N, batch, c->tree, c->tree, st, false, S, S);
    if (s == TP_OK) s = ntt_launch((uint32_t)N, batch, c->tree + N, c->tree + N, st, false, S, S);
    if (s == TP_OK) s = ks_trace_steps(c->trace, batch, c->tree, S, (int)c->logn, (int)(L + 1), st);
    if (s != TP_OK) return s;
    for (uint32_t l = L; l >= 1; --l) {
        tp::KsKernelParams kp = c->trace->kp;
        kp.key = c->trace->key + (uint64_t)(l - 1) * c->trace->digits * 2 * N;
        kp.in = c->tree;
        kp.out = c->tree;
        kp.items = batch << (L - l);
        kp.in_stride = kp.out_stride = (2 * N) << l;
        kp.right_offset = (2 * N) << (l - 1);
        kp.auto_index = (1u << l) + 1;
        kp.auto_index_inv = inv_mod_2n(kp.auto_index, 2 * (uint32_t)N);
        kp.shift = (uint32_t)(N >> l);
        s = ks_launch(c->trace, tp::kKsSplit, kp, st);
        if (s != TP_OK) return s;
    }
    tp::sap_leaf_sum_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(out_coef, c->tree, batch, c->logn, L);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    return TP_OK;
}

// ResetAccumulator (lines 293-351) of `batch` NTT-domain accumulators into fresh
// NTT-domain ones: overflow extraction (polynomial `ovf`), INTT, the fused
// SampleExtract -> LWE key switch -> FLOOR switch to 2N, a rotation of (0, Q/2N).
// Uses c->ext and c->lw; `fresh` may be c->ext.
static tp_status sap_reset_into(tp_sap_ctx* c, uint64_t batch, const uint64_t* acc_ntt, const uint64_t* ovf,
                                uint64_t* fresh, cudaStream_t st) {
    const uint64_t N = c->N, n = c->n;
    tp::sap_mul_poly_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(c->ext, 2 * N, acc_ntt, ovf, 1, batch,
                                                                     c->logn);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    tp_status s = ntt_launch((uint32_t)N, 2 * batch, c->ext, c->ext, st, false);
    if (s == TP_OK) s = tp_pbs_epilogue_batch(c->lks, batch, c->lw, c->ext, 2 * N, st);
    if (s == TP_OK) s = br_rotate_auto(c->br, batch, fresh, c->lw, n + 1, c->fresh, 0, 0, st);
    return s;
}

tp_status tp_sap_decompose_batch(tp_sap_ctx* c, uint64_t batch, uint64_t* out, uint64_t out_digits,
                                 const uint64_t* lwes, uint64_t radix, uint64_t hamming_weight,
                                 uint64_t restart_period, uint32_t* digits_host, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->ready) return fail(TP_ERR_STATE, "keys not uploaded");
    const uint64_t N = c->N, n = c->n;
    if (radix < 2 || radix > N || (radix & (radix - 1)))
        return fail(TP_ERR_PARAM, "radix must be a power of two in [2, N]");
    if (restart_period == 0) return fail(TP_ERR_PARAM, "restart period must be positive (UINT64_MAX: never)");
    if (batch == 0) return TP_OK;
    if (!out || !lwes) return fail(TP_ERR_PARAM, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t logr = (uint32_t)ilog2(radix);
    tp_status s = sap_reserve(c, batch, 1ull << (c->logn - logr));
    if (s == TP_OK) s = sap_constants(c, radix, st);
    if (s != TP_OK) return s;

    // input moduli and digit counts (lines 409-416); one read-back to plan the steps
    tp::sap_init_kernel<<<(unsigned)((batch + 127) / 128), 128, 0, st>>>(c->copy, c->modulus, lwes, batch,
                                                                       (uint32_t)n);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    tp::sap_acc_init_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(c->acc, batch, c->logn);
    tp::note_launch();
    TP_CUDA(cudaGetLastError());
    std::vector<uint64_t> M(batch);
    TP_CUDA(cudaMemcpyAsync(M.data(), c->modulus, batch * 8, cudaMemcpyDeviceToHost, st));
    TP_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> digits(batch, 0);
    uint32_t steps = 0;
    for (uint64_t b = 0; b < batch; ++b) {
        for (uint64_t m = M[b]; m > 1; m >>= logr) ++digits[b];
        steps = std::max(steps, digits[b]);
    }
    if (digits_host) std::copy(digits.begin(), digits.end(), digits_host);
    for (uint64_t b = 0; b < batch; ++b)
        if (digits[b] > out_digits)
            return fail(TP_ERR_PARAM, "LWE %llu needs %u digits, the output holds %llu", (unsigned long long)b,
                        digits[b], (unsigned long long)out_digits);

    const uint64_t out_stride = out_digits * (N + 1);
    for (uint32_t d = 0; d < steps; ++d) {
        bool any_reset = false, more = false;
        for (uint64_t b = 0; b < batch; ++b) {
            if (d < digits[b] && (d + 1) % restart_period == 0 && (M[b] >> (logr * (d + 1ull))) != 0)
                any_reset = true;
            if (d + 1 < digits[b]) more = true;
        }
        tp::sap_digit_kernel<<<sap_blocks(batch * (n + 1)), 256, 0, st>>>(
            c->copy, c->sub, c->modulus, c->flags, batch, (uint32_t)n, (uint32_t)N, logr, hamming_weight, d,
            restart_period);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
        // rotation of the coefficient-domain accumulator in place, NTT output (lines 432-434)
        s = br_rotate_auto(c->br, batch, c->acc, c->sub, n + 1, c->acc, 2 * N, 0, stream);
        if (s != TP_OK) return s;
        // digit d = SampleExtract(INTT(acc (.) extract poly)) (lines 438-445)
        tp::sap_mul_poly_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(c->ext, 2 * N, c->acc, c->consts, 1,
                                                                         batch, c->logn);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
        s = ntt_launch((uint32_t)N, 2 * batch, c->ext, c->ext, stream, false);
        if (s != TP_OK) return s;
        tp::sap_extract_kernel<<<sap_blocks(batch * (N + 1)), 256, 0, st>>>(out, out_stride, d, c->ext, c->flags,
                                                                          batch, (uint32_t)N);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
        if (any_reset) {
            // ResetAccumulator(acc, 0) (line 452), taken where flagged
            s = sap_reset_into(c, batch, c->acc, c->consts + 2 * N, c->ext, st);
            if (s != TP_OK) return s;
            tp::sap_select_kernel<<<sap_blocks(batch * 2 * N), 256, 0, st>>>(c->acc, c->ext, c->flags, batch,
                                                                           c->logn);
            tp::note_launch();
            TP_CUDA(cudaGetLastError());
        }
        if (!more) break;
        // HomTrunc (line 457); its coefficient-domain result is the next rotation's accumulator
        s = sap_trunc(c, batch, c->acc, c->acc, radix, st);
        if (s != TP_OK) return s;
    }
    return TP_OK;
}

tp_status tp_sap_homtrunc_batch(tp_sap_ctx* c, uint64_t batch, uint64_t* out, const uint64_t* in, uint64_t radix,
                                void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->ready) return fail(TP_ERR_STATE, "keys not uploaded");
    if (radix < 2 || radix > c->N || (radix & (radix - 1)))
        return fail(TP_ERR_PARAM, "radix must be a power of two in [2, N]");
    if (batch == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = (cudaStream_t)stream;
    tp_status s = sap_reserve(c, batch, 1ull << (c->logn - ilog2(radix)));
    if (s == TP_OK) s = sap_constants(c, radix, st);
    if (s == TP_OK) s = sap_trunc(c, batch, in, out, radix, st);
    // the reference's HomTrunc output is in the NTT domain
    if (s == TP_OK) s = ntt_launch(c->N, 2 * batch, out, out, stream, true);
    return s;
}

tp_status tp_sap_reset_batch(tp_sap_ctx* c, uint64_t batch, uint64_t* acc, uint64_t radix, void* stream) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->ready) return fail(TP_ERR_STATE, "keys not uploaded");
    if (radix > c->N || (radix & (radix - 1))) return fail(TP_ERR_PARAM, "radix must be 0 or a power of two <= N");
    if (batch == 0) return TP_OK;
    if (!acc) return fail(TP_ERR_PARAM, "null buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = (cudaStream_t)stream;
    // radix 0 and 1 give the same polynomial (IntLog2 of both is 0); keep the
    // extraction and pad constants of a real radix if they are loaded
    const uint64_t key = radix >= 2 ? radix : (c->radix ? c->radix : 2);
    tp_status s = sap_reserve(c, batch, 1);
    if (s == TP_OK) s = sap_constants(c, key, st);
    if (s != TP_OK) return s;
    const uint64_t* ovf = radix >= 2 ? c->consts + 3 * c->N : c->consts + 2 * c->N;
    s = sap_reset_into(c, batch, acc, ovf, c->ext, st);
    if (s == TP_OK)
        TP_CUDA(cudaMemcpyAsync(acc, c->ext, batch * 2 * c->N * 8, cudaMemcpyDeviceToDevice, st));
    return s;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Packing without any device allocation
// ---------------------------------------------------------------------------
// Callers that cannot allocate device memory at call time use this: a serving
// process whose device memory is owned by another allocator (for example a
// framework pool that has reserved nearly all of HBM up front), or a latency
// loop that must not pay for cudaMalloc/cudaFree, which can block and
// synchronise the device. tp_pack_batch grows a work area with cudaMalloc;
// this variant keeps its packing-tree nodes in the fixed array below instead.
//
// The array is a file-scope device variable: every GPU that loads this
// library reserves its kPackScratchWords * 8 bytes (16 MiB) until the process
// exits. In host code the name `g_pack_scratch` only stands in for the
// variable, it is not a device address; the device address is fetched once
// per device with cudaGetSymbolAddress and cached. The cache assumes the
// device's primary context lives until the process exits: after a
// cudaDeviceReset the module may load at another address, so a process that
// resets a device must not call this entry point on it again.

namespace {
constexpr uint64_t kPackScratchWords = 2ull << 20;  // 16 MiB of packing-tree nodes
constexpr int kMaxDevices = 64;
std::mutex g_pack_scratch_mu;
uint64_t* g_pack_scratch_addr[kMaxDevices] = {};
}  // namespace

static __device__ __align__(256) uint64_t g_pack_scratch[kPackScratchWords];

extern "C" tp_status tp_pack_batch_noalloc(tp_ks_ctx* c, uint64_t packs, uint64_t len, uint64_t* out,
                                           const uint64_t* in, void* stream) {
    if (!c || c->kind != 2) return fail(TP_ERR_PARAM, "not a packing context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no keys uploaded");
    if (packs == 0) return TP_OK;
    if (!out || !in) return fail(TP_ERR_PARAM, "null buffer");
    const uint64_t N = c->N;
    if (len < 2 || len > N || (len & (len - 1))) return fail(TP_ERR_PARAM, "len must be a power of two in [2, N]");
    // compared by division: packs * len * 2N itself can wrap around 64 bits
    const uint64_t per_pack = len * 2 * N;
    if (packs > kPackScratchWords / per_pack)
        return fail(TP_ERR_PARAM,
                    "packs * len * 2N (%llu packs of %llu words) exceeds the fixed scratch of %llu words (16 MiB); "
                    "use fewer packs per call or tp_pack_batch",
                    (unsigned long long)packs, (unsigned long long)per_pack, (unsigned long long)kPackScratchWords);
    const uint64_t need = packs * per_pack;
    if (c->device < 0 || c->device >= kMaxDevices) return fail(TP_ERR_PARAM, "device index out of range");
    // The context's key, tile and tables are read under its lock, as in tp_pack_batch:
    // tp_ks_set_tile or tp_ks_upload_key on another thread cannot swap them mid-call.
    std::lock_guard<std::mutex> ctx_lock(c->mu);
    TP_CUDA(cudaSetDevice(c->device));
    uint64_t* work = nullptr;
    {
        // First call on this device (now current): look up the array's device address.
        std::lock_guard<std::mutex> lk(g_pack_scratch_mu);
        if (!g_pack_scratch_addr[c->device]) {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_pack_scratch);
            if (e != cudaSuccess || !addr)
                return fail(TP_ERR_CUDA, "cudaGetSymbolAddress(g_pack_scratch): %s", cudaGetErrorString(e));
            g_pack_scratch_addr[c->device] = static_cast<uint64_t*>(addr);
        }
        work = g_pack_scratch_addr[c->device];
    }
    // Every word of the nodes in use is written by the set-up kernel below
    // before any merge reads it, so nothing left by an earlier call is read.
    cudaStream_t st = (cudaStream_t)stream;
    const int log_len = ilog2(len);
    {
        const uint64_t blocks = std::min<uint64_t>((need + 255) / 256, 65535);
        tp::pack_l0_kernel<<<(unsigned)blocks, 256, 0, st>>>(work, in, packs, (uint32_t)len, (uint32_t)log_len,
                                                            (uint32_t)c->logn, c->tab->n_inv);
        tp::note_launch();
        TP_CUDA(cudaGetLastError());
    }
    {
        tp_status s = pack_merge_levels(c, packs, len, 0, work, st);  // the merges of tp_pack_batch
        if (s != TP_OK) return s;
    }
    {
        tp_status s = ks_trace_steps(c, packs, work, len * 2 * N, c->logn, log_len + 1, st);
        if (s != TP_OK) return s;
    }
    TP_CUDA(cudaMemcpy2DAsync(out, 2 * N * 8, work, len * 2 * N * 8, 2 * N * 8, packs, cudaMemcpyDeviceToDevice, st));
    return TP_OK;
}

namespace tp {

tp_status set_error(tp_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

// The one-block kernel a launch uses: the digit-staged form when selected and
// the tile is 4 coefficients per thread, else the row-by-row form of the tile.
static bool br_uses_ds(const tp_br_ctx* c) {
    return c->loge == 2 && c->mac == TP_MAC_DIGIT_STAGED && c->ds_kernel;
}

// The one-block kernel of the context's settings: tile, multiply-accumulate form
// and radix (each form falls back to what is built).
static tp_br_ctx::Form br_one_block(const tp_br_ctx* c) {
    const bool ds = br_uses_ds(c);
    if (c->loge == 2 && c->radix == 4) {
        if (ds && c->r4_ds.k) return c->r4_ds;
        if (!ds && c->r4_row.k) return c->r4_row;
    }
    tp_br_ctx::Form f;
    f.k = ds ? c->ds_kernel : c->kernels[c->loge];
    f.smem = ds ? c->ds_smem : c->smem[c->loge];
    f.cap = ds ? c->ds_cap : c->grid_caps[c->loge];
    return f;
}

int br_cluster_ctas(const tp_br_ctx* c) { return c ? 1 << c->logs : 1; }

uint64_t br_concurrency(const tp_br_ctx* c, int split) {
    if (!c) return 0;
    if (split == 2) return c->loge == 2 ? (uint64_t)c->pair_cap : 0;
    if (split == 4) return c->loge == 2 ? (uint64_t)c->quad_cap : 0;
    return (uint64_t)br_one_block(c).cap;
}

tp_status br_batch_launch(tp_br_ctx* c, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                          uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef, void* stream,
                          int split) {
    if (!c) return fail(TP_ERR_PARAM, "null context");
    if (!c->key_ready) return fail(TP_ERR_STATE, "no key uploaded");
    if (batch == 0) return TP_OK;
    if (!results || !lwes || !accs) return fail(TP_ERR_PARAM, "null buffer");
    if (lwe_stride < (uint64_t)c->prm.lwe_dim + 1) return fail(TP_ERR_PARAM, "lwe_stride below n+1");
    if (acc_stride != 0 && acc_stride < 2ull * c->prm.ring_dim) return fail(TP_ERR_PARAM, "acc_stride below 2N");
    if (((uintptr_t)results & 15) || ((uintptr_t)accs & 7) || ((uintptr_t)lwes & 7))
        return fail(TP_ERR_PARAM, "results must be 16-byte aligned, lwes/accs 8-byte aligned");
    if (split == 0) split = c->split;
    if (split == 4 && br_concurrency(c, 4) == 0) split = 2;
    if (split == 2 && br_concurrency(c, 2) == 0) split = 1;
    TP_CUDA(cudaSetDevice(c->device));
    BrKernelParams kp = c->kp;
    kp.key = c->key;
    kp.lwes = lwes;
    kp.lwe_stride = lwe_stride;
    kp.accs = accs;
    kp.acc_stride = acc_stride;
    kp.out = results;
    kp.batch = batch;
    kp.out_coef = out_coef ? 1u : 0u;
    void* args[] = {&kp};
    if (split == 2 || split == 4) {
        const unsigned clusters = (unsigned)std::min<uint64_t>(batch, br_concurrency(c, split));
        TP_CUDA(cudaLaunchKernel(split == 2 ? c->pair_kernel : c->quad_kernel, dim3((unsigned)split * clusters),
                                 dim3(c->prm.ring_dim >> 2), args, split == 2 ? c->pair_smem : c->quad_smem,
                                 (cudaStream_t)stream));
        tp::note_launch();
        return TP_OK;
    }
    const bool ds = br_uses_ds(c);
    const unsigned grid = (unsigned)std::min<uint64_t>(batch, br_concurrency(c, 1));
    if (c->logs > 0) {
        // one rotation per cluster of 2^logs CTAs
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr = {};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = 1u << c->logs;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(grid << c->logs);
        cfg.blockDim = dim3(c->prm.ring_dim >> (c->logs + 2));
        cfg.dynamicSmemBytes = ds ? c->ds_smem : c->smem[2];
        cfg.stream = (cudaStream_t)stream;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        TP_CUDA(cudaLaunchKernelExC(&cfg, ds ? c->ds_kernel : c->kernels[2], args));
        tp::note_launch();
        return TP_OK;
    }
    const tp_br_ctx::Form f = br_one_block(c);
    TP_CUDA(cudaLaunchKernel(f.k, dim3(grid), dim3(c->prm.ring_dim >> c->loge), args, f.smem, (cudaStream_t)stream));
    tp::note_launch();
    return TP_OK;
}

}  // namespace tp

// ---------------------------------------------------------------------------
// Short names (the same calls)
// ---------------------------------------------------------------------------
extern "C" {

tp_status tp_ctx_create(const tp_params* params, tp_ctx** out) { return tp_br_create(params, 0, out); }

tp_status tp_ctx_destroy(tp_ctx* ctx) { return tp_br_destroy(ctx); }

tp_status tp_brk_upload(tp_ctx* ctx, const uint64_t* brk, uint64_t words, int layout_tag) {
    if (layout_tag != TP_LAYOUT_REFERENCE)
        return fail(TP_ERR_LAYOUT, "key layout tag %d: only the reference's m_brk layout (0) is accepted",
                    layout_tag);
    return tp_br_upload_key(ctx, brk, words);
}

tp_status tp_blind_rotate(tp_ctx* ctx, uint64_t* result, const uint64_t* lwe, const uint64_t* acc, int out_coef) {
    return tp_br_blind_rotate(ctx, result, lwe, acc, out_coef);
}

tp_status tp_blind_rotate_batch(tp_ctx* ctx, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                const uint64_t* accs, uint64_t acc_stride, int out_coef, void* stream) {
    if (!ctx) return fail(TP_ERR_PARAM, "null context");
    return tp_br_blind_rotate_batch(ctx, batch, results, lwes, (uint64_t)ctx->prm.lwe_dim + 1, accs, acc_stride,
                                    out_coef, stream);
}

tp_status tp_auto_ks_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out, const uint64_t* in, void* stream) {
    return tp_auto_eval_batch(ctx, batch, out, in, stream);
}

const char* tp_last_error_string(void) { return tp_last_error(); }

}  // extern "C"
