// Thin C entry points over the reference library itself (TEST INFRASTRUCTURE).
//
// oracle/Makefile compiles the reference's own sources, unmodified, from the
// reference tree together with this file and the shims in oracle/shim/, into
// oracle/_ref/libtpref.so. Tests use it to pin the C oracle (tests/golden/
// fixtures are generated through it) and bench.py's reference arm times its
// blind rotation as the CPU baseline. Nothing here is part of the product.
//
// Private members (the generated key m_brk / m_ksk) are read by compiling this
// translation unit with access specifiers opened after the standard headers.

#include <bits/stdc++.h>
#include <immintrin.h>
#include <pthread.h>

#define private public
#define protected public
#include "backend/backend.h"
#include "backend/solinas_worker.h"
#include "base_crypto.h"
#include "operators/automorphism_evaluation.h"
#include "operators/bmmp_blind_rotation.h"
#include "operators/cggi_blind_rotation.h"
#include "operators/endo_glwe_conversion.h"
#include "operators/lwe_to_rgsw_conversion.h"
#include "operators/lwe_to_rlwe_packing.h"
#include "operators/sap_decomposition.h"
#include "operators/trace_evaluation.h"
#include "static/keys.h"
#include "static/modulus_switching.h"
#include "static/sample_extraction.h"
#undef private
#undef protected

#include "openfhe.h"

namespace {
const uint64_t kQ = 0xFFFFFFFF00000001ULL;

struct BRHandle {
    int variant = 0;
    uint64_t N = 0, n = 0;
    std::shared_ptr<CGGIBlindRotationContext> cggi_ctx;
    std::shared_ptr<BMMPBlindRotationContext> bmmp_ctx;
    std::unique_ptr<CGGIBlindRotator> cggi;
    std::unique_ptr<BMMPBlindRotator> bmmp;
    BlindRotator* rot() { return cggi ? (BlindRotator*)cggi.get() : (BlindRotator*)bmmp.get(); }
    const AlignedBuffer& brk() const { return cggi ? cggi->m_brk : bmmp->m_brk; }
};
}  // namespace

extern "C" {

void ref_seed(uint64_t s) { tp_shim::seed(s); }

int ref_ntt_forward(uint64_t N, uint64_t* out, const uint64_t* in) {
    try {
        SelectWorker(kQ, N)->ForwardNTT(out, in);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_ntt_backward(uint64_t N, uint64_t* out, const uint64_t* in) {
    try {
        SelectWorker(kQ, N)->BackwardNTT(out, in);
        return 0;
    } catch (...) {
        return -1;
    }
}

// variant: 0 CGGI binary, 1 CGGI ternary, 2 BMMP binary (step 2).
void* ref_br_create(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits, double std_dev,
                    const uint64_t* lwe_key, const uint64_t* rlwe_key) {
    auto* h = new BRHandle();
    h->variant = variant;
    h->N = N;
    h->n = n;
    std::vector<GenericKey> bundle = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
    const uint64_t basis = 1ULL << basis_log2;
    if (variant == 2) {
        h->bmmp_ctx = std::make_shared<BMMPBlindRotationContext>(KeyDistribution::BINARY, kQ, N, n, basis, digits,
                                                                 std_dev, 2);
        h->bmmp = h->bmmp_ctx->ConstructOperator(bundle);
    } else {
        h->cggi_ctx = std::make_shared<CGGIBlindRotationContext>(
            variant == 0 ? KeyDistribution::BINARY : KeyDistribution::TERNARY, kQ, N, n, basis, digits, std_dev);
        h->cggi = h->cggi_ctx->ConstructOperator(bundle);
    }
    return h;
}

uint64_t ref_br_key_words(void* hp) { return ((BRHandle*)hp)->brk().size(); }

void ref_br_key_copy(void* hp, uint64_t* out) {
    const auto& k = ((BRHandle*)hp)->brk();
    std::copy(k.begin(), k.end(), out);
}

void ref_br_rotate(void* hp, uint64_t* result, const uint64_t* lwe, const uint64_t* acc, int out_coef) {
    auto* h = (BRHandle*)hp;
    std::vector<uint64_t> a(acc, acc + 2 * h->N);
    h->rot()->BlindRotate(result, lwe, a.data(), out_coef != 0);
}

void ref_br_destroy(void* hp) { delete (BRHandle*)hp; }

// Times `count` rotations spread over `threads` threads, one rotator per thread
// (operators are not reentrant); every rotator shares the first one's key bytes.
// Returns the wall-clock seconds of the rotation phase only.
double ref_br_rotate_many(void* hp, uint64_t* results, const uint64_t* lwes, const uint64_t* accs, uint64_t count,
                          int out_coef, int threads) {
    auto* h = (BRHandle*)hp;
    if (threads < 1) threads = 1;
    const uint64_t N = h->N, n = h->n;
    std::vector<std::unique_ptr<CGGIBlindRotator>> cg;
    std::vector<std::unique_ptr<BMMPBlindRotator>> bm;
    std::vector<BlindRotator*> rots;
    for (int t = 0; t < threads; ++t) {
        if (h->cggi) {
            cg.push_back(std::make_unique<CGGIBlindRotator>(h->cggi_ctx));
            cg.back()->m_brk = h->cggi->m_brk;
            cg.back()->m_keys_generated = true;
            rots.push_back(cg.back().get());
        } else {
            bm.push_back(std::make_unique<BMMPBlindRotator>(h->bmmp_ctx));
            bm.back()->m_brk = h->bmmp->m_brk;
            bm.back()->m_keys_generated = true;
            rots.push_back(bm.back().get());
        }
    }
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) {
        th.emplace_back([&, t]() {
            std::vector<uint64_t> a(2 * N);
            for (uint64_t b = (uint64_t)t; b < count; b += (uint64_t)threads) {
                std::copy(accs + b * 2 * N, accs + (b + 1) * 2 * N, a.begin());
                rots[t]->BlindRotate(results + b * 2 * N, lwes + b * (n + 1), a.data(), out_coef != 0);
            }
        });
    }
    for (auto& x : th) x.join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// RLWE -> RLWE key switching.
void* ref_rlwe_ks_create(uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev, const uint64_t* src_key,
                         const uint64_t* tgt_key) {
    auto ctx = std::make_shared<RLWEConversionContext>(KeyDistribution::TERNARY, kQ, N, 1ULL << basis_log2, digits,
                                                       std_dev);
    std::vector<GenericKey> keys = {{"SRC", src_key, N}, {"TGT", tgt_key, N}};
    auto op = ctx->ConstructOperator(keys);
    return op.release();
}

void ref_rlwe_ks_key_copy(void* hp, uint64_t* out) {
    auto* op = (RLWEtoRLWEConverter*)hp;
    std::copy(op->m_ksk.begin(), op->m_ksk.end(), out);
}

void ref_rlwe_ks_convert(void* hp, uint64_t* out, const uint64_t* in) { ((RLWEtoRLWEConverter*)hp)->Convert(out, in); }

void ref_rlwe_ks_destroy(void* hp) { delete (RLWEtoRLWEConverter*)hp; }

// LWE -> LWE key switching (modulus q).
void* ref_lwe_ks_create(uint64_t q, uint64_t n_in, uint64_t n_out, uint64_t basis_log2, uint64_t digits,
                        double std_dev, const uint64_t* src_key, const uint64_t* tgt_key) {
    auto ctx = std::make_shared<LWEConversionContext>(KeyDistribution::TERNARY, q, n_in, n_out, 1ULL << basis_log2,
                                                      digits, std_dev);
    std::vector<GenericKey> keys = {{"SRC", src_key, n_in}, {"TGT", tgt_key, n_out}};
    auto op = ctx->ConstructOperator(keys);
    return op.release();
}

void ref_lwe_ks_key_copy(void* hp, uint64_t* out) {
    auto* op = (LWEtoLWEConverter*)hp;
    std::copy(op->m_ksk.begin(), op->m_ksk.end(), out);
}

void ref_lwe_ks_convert(void* hp, uint64_t* out, const uint64_t* in) { ((LWEtoLWEConverter*)hp)->Convert(out, in); }

void ref_lwe_ks_destroy(void* hp) { delete (LWEtoLWEConverter*)hp; }

// Automorphism evaluation X -> X^index followed by the key switch back to s.
void* ref_auto_create(uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev, uint32_t index,
                      const uint64_t* key) {
    auto ctx = std::make_shared<AutomorphismContext>(KeyDistribution::TERNARY, kQ, N, 1ULL << basis_log2, digits,
                                                     std_dev, index);
    std::vector<GenericKey> keys = {{"KEY", key, N}};
    auto op = ctx->ConstructOperator(keys);
    return op.release();
}

void ref_auto_eval(void* hp, uint64_t* out, const uint64_t* in) { ((AutomorphismEvaluator*)hp)->Eval(out, in); }

void ref_auto_key_copy(void* hp, uint64_t* out) {
    const auto& k = ((AutomorphismEvaluator*)hp)->m_converter->m_ksk;
    std::copy(k.begin(), k.end(), out);
}

void ref_auto_destroy(void* hp) { delete (AutomorphismEvaluator*)hp; }

// n-LWE -> RLWE packing.
void* ref_pack_create(uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev, const uint64_t* key) {
    auto ctx = std::make_shared<LWEtoRLWEPackingContext>(KeyDistribution::TERNARY, kQ, N, 1ULL << basis_log2, digits,
                                                         std_dev);
    std::vector<GenericKey> keys = {{"KEY", key, N}};
    auto op = ctx->ConstructOperator(keys);
    return op.release();
}

void ref_pack(void* hp, uint64_t* out, const uint64_t* in, uint64_t len) { ((LWEtoRLWEPacker*)hp)->Pack(out, in, len); }

void ref_pack_consecutive(void* hp, uint64_t* out, const uint64_t* in, uint64_t len) {
    ((LWEtoRLWEPacker*)hp)->PackConsecutively(out, in, len);
}

// The packer's automorphism keys (index 2^j + 1, j = 1..logN), concatenated.
void ref_pack_key_copy(void* hp, uint64_t* out) {
    for (auto& ev : ((LWEtoRLWEPacker*)hp)->m_auto_evaluators) {
        const auto& k = ev->m_converter->m_ksk;
        out = std::copy(k.begin(), k.end(), out);
    }
}

void ref_pack_destroy(void* hp) { delete (LWEtoRLWEPacker*)hp; }

// TraceEvaluationContext(BINARY, modulus, N, basis, digits, std) and its operator.
void* ref_trace_create(uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev, const uint64_t* key) {
    auto ctx = std::make_shared<TraceEvaluationContext>(BINARY, kQ, N, 1ULL << basis_log2, digits, std_dev);
    std::vector<GenericKey> keys = {{"KEY", key, N}};
    return ctx->ConstructOperator(keys).release();
}

void ref_trace_key_copy(void* hp, uint64_t* out) {
    for (auto& ev : ((TraceEvaluator*)hp)->m_trace_evaluators) {
        const auto& k = ev->m_converter->m_ksk;
        out = std::copy(k.begin(), k.end(), out);
    }
}

void ref_trace_eval(void* hp, uint64_t* out, const uint64_t* in) { ((TraceEvaluator*)hp)->Eval(out, in); }

void ref_trace_eval_auto(void* hp, uint64_t* out, const uint64_t* in, uint64_t index) {
    ((TraceEvaluator*)hp)->EvalAuto(out, in, index);
}

void ref_trace_destroy(void* hp) { delete (TraceEvaluator*)hp; }

void ref_sample_extract(uint64_t* out_lwe, uint64_t* rlwe, uint64_t index, uint64_t N) {
    SampleExtract<uint64_t>(out_lwe, rlwe, index, N, kQ);
}

// LWE -> RGSW scheme switching (lib/src/operators/lwe_to_rgsw_conversion.cpp): CGGI binary
// rotation, trace and squaring contexts all with (base 2^basis_log2, digits), output RGSW
// with (out_digits, 2^out_basis_log2), as tests/scheme_switch_tests.cpp builds them.
struct SSHandle {
    std::shared_ptr<SchemeSwitchingContext> ctx;
    std::unique_ptr<LWEtoRGSWConverter> op;
    uint64_t N = 0, out_digits = 0;
};

// variant as in ref_br_create; each component has its own gadget (basis 2^b, digits)
void* ref_ss_create(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                    uint64_t tr_basis_log2, uint64_t tr_digits, uint64_t sq_basis_log2, uint64_t sq_digits,
                    double std_dev, uint64_t out_digits, uint64_t out_basis_log2, const uint64_t* lwe_key,
                    const uint64_t* rlwe_key) {
    auto* h = new SSHandle();
    h->N = N;
    h->out_digits = out_digits;
    std::shared_ptr<OperatorContext<BlindRotator>> rot;
    std::shared_ptr<MathWorker> ntt;
    if (variant == 2) {
        auto br = std::make_shared<BMMPBlindRotationContext>(KeyDistribution::BINARY, kQ, N, n, 1ULL << br_basis_log2,
                                                             br_digits, std_dev, 2);
        ntt = br->GetNTT();
        rot = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
    } else {
        auto br = std::make_shared<CGGIBlindRotationContext>(
            variant == 0 ? KeyDistribution::BINARY : KeyDistribution::TERNARY, kQ, N, n, 1ULL << br_basis_log2,
            br_digits, std_dev);
        ntt = br->GetNTT();
        rot = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
    }
    auto tr = std::make_shared<TraceEvaluationContext>(BINARY, ntt, 1ULL << tr_basis_log2, tr_digits, std_dev);
    auto sq = std::make_shared<RLWEConversionContext>(BINARY, ntt, 1ULL << sq_basis_log2, sq_digits, std_dev);
    h->ctx = std::make_shared<SchemeSwitchingContext>(rot, tr, sq, out_digits, 1ULL << out_basis_log2);
    std::vector<GenericKey> keys = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
    h->op = h->ctx->ConstructOperator(keys);
    return h;
}

static const AlignedBuffer& ss_brk(SSHandle* h) {
    if (auto* c = dynamic_cast<CGGIBlindRotator*>(h->op->m_rotator.get())) return c->m_brk;
    return dynamic_cast<BMMPBlindRotator*>(h->op->m_rotator.get())->m_brk;
}

// what: 0 blind-rotation key, 1 trace keys (indices 3, 5, 9, .., N+1 concatenated), 2 squaring key
uint64_t ref_ss_key_words(void* hp, int what) {
    auto* h = (SSHandle*)hp;
    if (what == 0) return ss_brk(h).size();
    if (what == 1) {
        uint64_t w = 0;
        for (auto& e : h->op->m_trace_eval->m_trace_evaluators) w += e->m_converter->m_ksk.size();
        return w;
    }
    return h->op->m_square_eval->m_ksk.size();
}

void ref_ss_key_copy(void* hp, int what, uint64_t* out) {
    auto* h = (SSHandle*)hp;
    if (what == 0) {
        const auto& k = ss_brk(h);
        std::copy(k.begin(), k.end(), out);
    } else if (what == 1) {
        for (auto& e : h->op->m_trace_eval->m_trace_evaluators)
            out = std::copy(e->m_converter->m_ksk.begin(), e->m_converter->m_ksk.end(), out);
    } else {
        const auto& k = h->op->m_square_eval->m_ksk;
        std::copy(k.begin(), k.end(), out);
    }
}

// out: 4 N out_digits words (pre-zeroed here), [lev_left | lev_right], NTT domain
void ref_ss_convert(void* hp, uint64_t* out, const uint64_t* lwe) {
    auto* h = (SSHandle*)hp;
    std::fill(out, out + 4 * h->N * h->out_digits, 0);
    h->op->Convert(out, lwe);
}

void ref_ss_test_poly(void* hp, uint64_t* out) {  // the converter's m_acc (3N words)
    auto* h = (SSHandle*)hp;
    std::copy(h->op->m_acc.begin(), h->op->m_acc.end(), out);
}

void ref_ss_destroy(void* hp) { delete (SSHandle*)hp; }

struct SAPHandle {
    std::shared_ptr<SAPDecompositionContext> ctx;
    std::unique_ptr<SAPDecomposer> op;
    uint64_t N = 0, n = 0;
};

// SAPDecompositionContext(rotation, trace, LWE conversion N -> n, radix) and its operator.
void* ref_sap_create(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                     uint64_t tr_basis_log2, uint64_t tr_digits, uint64_t ks_basis_log2, uint64_t ks_digits,
                     double std_dev, uint64_t radix, const uint64_t* lwe_key, const uint64_t* rlwe_key) {
    auto* h = new SAPHandle();
    h->N = N;
    h->n = n;
    std::shared_ptr<OperatorContext<BlindRotator>> rot;
    std::shared_ptr<MathWorker> ntt;
    if (variant == 2) {
        auto br = std::make_shared<BMMPBlindRotationContext>(KeyDistribution::BINARY, kQ, N, n, 1ULL << br_basis_log2,
                                                             br_digits, std_dev, 2);
        ntt = br->GetNTT();
        rot = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
    } else {
        auto br = std::make_shared<CGGIBlindRotationContext>(
            variant == 0 ? KeyDistribution::BINARY : KeyDistribution::TERNARY, kQ, N, n, 1ULL << br_basis_log2,
            br_digits, std_dev);
        ntt = br->GetNTT();
        rot = std::reinterpret_pointer_cast<OperatorContext<BlindRotator>>(br);
    }
    auto tr = std::make_shared<TraceEvaluationContext>(BINARY, ntt, 1ULL << tr_basis_log2, tr_digits, std_dev);
    auto cv = std::make_shared<LWEConversionContext>(BINARY, kQ, N, n, 1ULL << ks_basis_log2, ks_digits, std_dev);
    h->ctx = std::make_shared<SAPDecompositionContext>(rot, tr, cv, radix);
    std::vector<GenericKey> keys = {{"LWE", lwe_key, n}, {"RLWE", rlwe_key, N}};
    h->op = h->ctx->ConstructOperator(keys);
    return h;
}

uint64_t ref_sap_restart(void* hp) { return ((SAPHandle*)hp)->op->m_restart_iteration; }
void ref_sap_set_restart(void* hp, uint64_t r) { ((SAPHandle*)hp)->op->m_restart_iteration = r; }
uint64_t ref_sap_beta(void* hp) { return ((SAPHandle*)hp)->op->m_beta; }

static const AlignedBuffer& sap_brk(SAPHandle* h) {
    if (auto* c = dynamic_cast<CGGIBlindRotator*>(h->op->m_rotator.get())) return c->m_brk;
    return dynamic_cast<BMMPBlindRotator*>(h->op->m_rotator.get())->m_brk;
}

// what: 0 blind-rotation key, 1 trace keys (indices 3, 5, 9, .., N+1 concatenated), 2 LWE key switch
uint64_t ref_sap_key_words(void* hp, int what) {
    auto* h = (SAPHandle*)hp;
    if (what == 0) return sap_brk(h).size();
    if (what == 1) {
        uint64_t w = 0;
        for (auto& e : h->op->m_packer->m_trace_evaluators) w += e->m_converter->m_ksk.size();
        return w;
    }
    return h->op->m_lwe_converter->m_ksk.size();
}

void ref_sap_key_copy(void* hp, int what, uint64_t* out) {
    auto* h = (SAPHandle*)hp;
    if (what == 0) {
        const auto& k = sap_brk(h);
        std::copy(k.begin(), k.end(), out);
    } else if (what == 1) {
        for (auto& e : h->op->m_packer->m_trace_evaluators)
            out = std::copy(e->m_converter->m_ksk.begin(), e->m_converter->m_ksk.end(), out);
    } else {
        const auto& k = h->op->m_lwe_converter->m_ksk;
        std::copy(k.begin(), k.end(), out);
    }
}

// Decompose with the LWE converter's accumulator fully cleared first (its own clear is
// partial, lwe_conversion.cpp:217), so a reset inside behaves as on a fresh converter.
// out: out_words words, zeroed here (SampleExtract writes only nonzero words).
void ref_sap_decompose(void* hp, uint64_t* out, uint64_t out_words, const uint64_t* in, uint64_t radix) {
    auto* h = (SAPHandle*)hp;
    auto& acc = h->op->m_lwe_converter->m_acc;
    std::fill(acc.begin(), acc.end(), 0);
    std::fill(out, out + out_words, 0);
    h->op->Decompose(out, in, radix);
}

void ref_sap_homtrunc(void* hp, uint64_t* out, uint64_t* in, uint64_t radix) {
    ((SAPHandle*)hp)->op->HomTrunc(out, in, radix);
}

void ref_sap_reset(void* hp, uint64_t* acc, uint64_t radix) {
    auto* h = (SAPHandle*)hp;
    auto& a = h->op->m_lwe_converter->m_acc;
    std::fill(a.begin(), a.end(), 0);
    h->op->ResetAccumulator(acc, radix);
}

void ref_sap_destroy(void* hp) { delete (SAPHandle*)hp; }

// type: 0 ROUND, 1 FLOOR, 2 CEIL (ModulusSwitchType order)
void ref_modulus_switch(uint64_t* vec, uint64_t n, uint64_t source, uint64_t target, int type) {
    const ModulusSwitchType t[] = {ModulusSwitchType::ROUND, ModulusSwitchType::FLOOR, ModulusSwitchType::CEIL};
    ModulusSwitch(vec, n, source, target, t[type]);
}

}  // extern "C"
