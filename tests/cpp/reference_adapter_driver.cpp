// Test driver of the reference-side adapter (fhetoothpaste_b200/host/reference_adapter.hpp).
//
// TEST INFRASTRUCTURE: built by oracle/Makefile against the reference library compiled
// from its own sources (oracle/_ref/libtpref.so) and libtoothpaste_gpu.so. Each entry
// point runs an unchanged reference caller of BlindRotator twice on the same inputs,
// with keys drawn from the same sampler seed: once over the reference's CPU rotator
// (the reference tests' own wiring, a CGGI / BMMP context passed as
// OperatorContext<BlindRotator>) and once over toothpaste_b200::GpuRotationContext.
// The Python test compares the two outputs word for word.
//
// NegacyclicFunctionEvaluator is not driven: its constructor
// (negacyclic_function_evaluator.cpp:64-66) casts the rotation context's input container,
// a tuple (LWE, RLWE) for CGGI and BMMP contexts, to an RLWE container and dereferences
// the null result, so the reference cannot construct it over any rotation context (its
// own negacyclic_func_test included). Its EvalFunc body is BlindRotate with coefficient
// output followed by SampleExtract, which adp_rotate_in_place covers.
//
// The adapter needs read access to the generated key (m_brk); a reference tree adds
// an accessor for it, here the access specifiers are opened instead.

#include <bits/stdc++.h>

#define private public
#define protected public
#include "base_crypto.h"
#include "operators/bmmp_blind_rotation.h"
#include "operators/cggi_blind_rotation.h"
#include "operators/endo_glwe_conversion.h"
#include "operators/lwe_to_rgsw_conversion.h"
#include "operators/sap_decomposition.h"
#include "operators/trace_evaluation.h"
#undef private
#undef protected

#include "reference_adapter.hpp"

extern "C" void ref_seed(uint64_t s);  // the seeded sampler of the reference build (ref_driver.cpp)

namespace toothpaste_b200 {
const AlignedBuffer& ReferenceRotationKey(const CGGIBlindRotator& op) { return op.m_brk; }
const AlignedBuffer& ReferenceRotationKey(const BMMPBlindRotator& op) { return op.m_brk; }
}  // namespace toothpaste_b200

namespace {
const uint64_t kQ = 0xFFFFFFFF00000001ULL;
std::string g_err;

// The reference CPU rotation context for a variant (0 CGGI binary, 1 CGGI ternary,
// 2 BMMP binary step 2) and the GPU context over the same parameters.
struct Contexts {
    std::shared_ptr<OperatorContext<BlindRotator>> cpu, gpu;
    std::shared_ptr<MathWorker> ntt;
};

Contexts make_contexts(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits, double std_dev) {
    Contexts c;
    if (variant == 2) {
        auto br = std::make_shared<BMMPBlindRotationContext>(KeyDistribution::BINARY, kQ, N, n, 1ULL << basis_log2,
                                                             digits, std_dev, 2);
        c.ntt = br->GetNTT();
        c.cpu = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
        c.gpu = std::make_shared<toothpaste_b200::GpuRotationContext>(br);
    } else {
        auto br = std::make_shared<CGGIBlindRotationContext>(
            variant == 0 ? KeyDistribution::BINARY : KeyDistribution::TERNARY, kQ, N, n, 1ULL << basis_log2, digits,
            std_dev);
        c.ntt = br->GetNTT();
        c.cpu = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
        c.gpu = std::make_shared<toothpaste_b200::GpuRotationContext>(br);
    }
    return c;
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
    } catch (...) {
        g_err = "unknown exception";
    }
    return -1;
}
}  // namespace

extern "C" {

const char* adp_last_error(void) { return g_err.c_str(); }

// LWEtoRGSWConverter::Convert(output, input) (lwe_to_rgsw_conversion.cpp:168-225) with its
// rotation, trace and squaring gadgets: outputs 4 N out_digits words each, zeroed first.
int adp_lwe_to_rgsw(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                    uint64_t tr_basis_log2, uint64_t tr_digits, uint64_t sq_basis_log2, uint64_t sq_digits,
                    double std_dev, uint64_t out_digits, uint64_t out_basis_log2, const uint64_t* lwe_key,
                    const uint64_t* rlwe_key, uint64_t seed, uint64_t count, const uint64_t* lwes, uint64_t* out_cpu,
                    uint64_t* out_gpu) {
    return guarded([&]() {
        Contexts c = make_contexts(variant, N, n, br_basis_log2, br_digits, std_dev);
        auto tr = std::make_shared<TraceEvaluationContext>(BINARY, c.ntt, 1ULL << tr_basis_log2, tr_digits, std_dev);
        auto sq = std::make_shared<RLWEConversionContext>(BINARY, c.ntt, 1ULL << sq_basis_log2, sq_digits, std_dev);
        std::vector<GenericKey> keys = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
        const uint64_t words = 4 * N * out_digits;
        for (int side = 0; side < 2; ++side) {
            auto ctx = std::make_shared<SchemeSwitchingContext>(side ? c.gpu : c.cpu, tr, sq, out_digits,
                                                                1ULL << out_basis_log2);
            ref_seed(seed);
            auto op = ctx->ConstructOperator(keys);
            uint64_t* out = side ? out_gpu : out_cpu;
            for (uint64_t b = 0; b < count; ++b) {
                std::fill(out + b * words, out + (b + 1) * words, 0);
                op->Convert(out + b * words, lwes + b * (n + 1));
            }
        }
    });
}

// SAPDecomposer::Decompose(output, input, radix) (sap_decomposer.cpp:353-464): repeated
// rotations with result == accumulator. Outputs out_words words each, zeroed first; the
// LWE converter's accumulator is cleared before each call (its own clear is partial,
// lwe_conversion.cpp:217), so every call behaves as on a fresh converter.
int adp_sap(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits, uint64_t tr_basis_log2,
            uint64_t tr_digits, uint64_t ks_basis_log2, uint64_t ks_digits, double std_dev, uint64_t radix,
            const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t seed, uint64_t count, const uint64_t* lwes,
            uint64_t out_words, uint64_t* out_cpu, uint64_t* out_gpu) {
    return guarded([&]() {
        Contexts c = make_contexts(variant, N, n, br_basis_log2, br_digits, std_dev);
        auto tr = std::make_shared<TraceEvaluationContext>(BINARY, c.ntt, 1ULL << tr_basis_log2, tr_digits, std_dev);
        auto cv = std::make_shared<LWEConversionContext>(BINARY, kQ, N, n, 1ULL << ks_basis_log2, ks_digits, std_dev);
        std::vector<GenericKey> keys = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
        for (int side = 0; side < 2; ++side) {
            auto ctx = std::make_shared<SAPDecompositionContext>(side ? c.gpu : c.cpu, tr, cv, radix);
            ref_seed(seed);
            auto op = ctx->ConstructOperator(keys);
            uint64_t* out = side ? out_gpu : out_cpu;
            for (uint64_t b = 0; b < count; ++b) {
                auto& acc = op->m_lwe_converter->m_acc;
                std::fill(acc.begin(), acc.end(), 0);
                std::fill(out + b * out_words, out + (b + 1) * out_words, 0);
                op->Decompose(out + b * out_words, lwes + b * (n + 1), radix);
            }
        }
    });
}

// The GPU rotator alone, for a direct BlindRotator::BlindRotate comparison: rotates
// `count` (lwe, acc) pairs with result == accumulator, as SAPDecomposer calls it.
int adp_rotate_in_place(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits, double std_dev,
                        const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t seed, uint64_t count,
                        const uint64_t* lwes, uint64_t* accs_cpu, uint64_t* accs_gpu, int out_coef) {
    return guarded([&]() {
        Contexts c = make_contexts(variant, N, n, basis_log2, digits, std_dev);
        std::vector<GenericKey> keys = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
        for (int side = 0; side < 2; ++side) {
            ref_seed(seed);
            auto rot = (side ? c.gpu : c.cpu)->ConstructOperator(keys);
            uint64_t* accs = side ? accs_gpu : accs_cpu;
            for (uint64_t b = 0; b < count; ++b)
                rot->BlindRotate(accs + b * 2 * N, lwes + b * (n + 1), accs + b * 2 * N, out_coef != 0);
        }
    });
}

}  // extern "C"
