// C++ drop-in operators over the B200 C ABI (include/toothpaste_gpu.h).
//
// These classes carry the reference's operator names, constructor parameters
// and call signatures (lib/include/interfaces/blindrotation_operator.h:20-49,
// lib/include/operators/cggi_blind_rotation.h:19-161,
// lib/include/operators/bmmp_blind_rotation.h:18-176,
// lib/include/operators/endo_glwe_conversion.h, automorphism_evaluation.h,
// lwe_to_rlwe_packing.h), so host code written against the reference compiles
// against them with a namespace change. ConstructOperator runs key generation
// on the host (toothpaste_b200.cpp: the reference's MakeRLWE/MakeRGSW
// steps with a seeded sampler) and uploads the key once; every BlindRotate /
// Convert / Eval / Pack then runs on the GPU. A key produced elsewhere (for
// instance by the reference's own operator) can be given to the Gpu* classes
// directly in the reference's layout.
//
// Errors: a failing call throws std::runtime_error with tp_last_error().
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "toothpaste_gpu.h"

namespace toothpaste_b200 {

constexpr uint64_t kGoldilocks = 0xFFFFFFFF00000001ull;

// lib/include/static/enum_ids.h
enum KeyDistribution { BINARY, TERNARY, GAUSSIAN };

inline void check(tp_status s) {
    if (s != TP_OK) throw std::runtime_error(std::string("toothpaste_b200: ") + tp_last_error());
}

// Seeded stand-in for the reference's OpenFHE samplers (splitmix64 stream;
// uniform by masked rejection, Gaussian by Box-Muller rounded to nearest).
class Sampler {
public:
    explicit Sampler(uint64_t seed) : m_s(seed) {}
    uint64_t Next();
    uint64_t Uniform(uint64_t q);
    uint64_t Gaussian(double std_dev, uint64_t q);

private:
    uint64_t m_s;
};

// Host key generation following the reference's RLWEEncryptor (lib/src/base_crypto.cpp:27-97)
// and the operators' KeyGen loops. Outputs are in the reference's layouts.
namespace keygen {
std::vector<uint64_t> BlindRotationKey(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t basis_log2,
                                       uint32_t digits, double std_dev, const std::vector<uint64_t>& lwe_key,
                                       const std::vector<uint64_t>& rlwe_key);
std::vector<uint64_t> RLWESwitchingKey(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double std_dev,
                                       const std::vector<uint64_t>& source_key, const std::vector<uint64_t>& target_key);
std::vector<uint64_t> AutomorphismKey(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double std_dev,
                                      uint32_t index, const std::vector<uint64_t>& key);
std::vector<uint64_t> PackingKeys(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double std_dev,
                                  const std::vector<uint64_t>& key);
// LWEtoLWEConverter::KeyGen (lib/src/operators/lwe_conversion.cpp:174-203) on the Goldilocks
// modulus: row (i, j) encrypts source_i * 2^(64 - beta (j + 1)) under the target key.
std::vector<uint64_t> LWESwitchingKey(Sampler& rng, uint32_t n_in, uint32_t n_out, uint32_t basis_log2,
                                      uint32_t digits, double std_dev, const std::vector<uint64_t>& source_key,
                                      const std::vector<uint64_t>& target_key);
// SAPDecompositionContext::ConstructOperator (lib/src/operators/sap_decomposer.cpp:166-186)
// from one sampler stream: the rotation key, the trace keys, then the LWE key switch from the
// RLWE key's coefficients (N) to the LWE key (n).
struct SAPKeySet {
    std::vector<uint64_t> rotation, trace, lwe_switch;
};
SAPKeySet SAPKeys(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t br_basis_log2, uint32_t br_digits,
                  uint32_t tr_basis_log2, uint32_t tr_digits, uint32_t ks_basis_log2, uint32_t ks_digits,
                  double std_dev, const std::vector<uint64_t>& lwe_key, const std::vector<uint64_t>& rlwe_key);
// SchemeSwitchingContext::ConstructOperator (lib/src/operators/lwe_to_rgsw_conversion.cpp:72-108)
// from one sampler stream: the rotation key, the trace's automorphism keys (indices 3, 5, .., N+1),
// then the key switch from s^2 to s.
struct SchemeSwitchingKeySet {
    std::vector<uint64_t> rotation, trace, square;
};
SchemeSwitchingKeySet SchemeSwitchingKeys(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t br_basis_log2,
                                          uint32_t br_digits, uint32_t tr_basis_log2, uint32_t tr_digits,
                                          uint32_t sq_basis_log2, uint32_t sq_digits, double std_dev,
                                          const std::vector<uint64_t>& lwe_key, const std::vector<uint64_t>& rlwe_key);
}  // namespace keygen

// BlindRotator (lib/include/interfaces/blindrotation_operator.h:20-49).
struct BlindRotator {
    virtual void BlindRotate(std::vector<uint64_t>& result, const std::vector<uint64_t>& lwe_ciphertext,
                             std::vector<uint64_t>& accumulator, bool output_as_coefficients = false) = 0;
    virtual void BlindRotate(uint64_t* result, const uint64_t* lwe_vec, uint64_t* accumulator,
                             bool output_as_coefficients = false) = 0;
    virtual ~BlindRotator() = default;
};

// A blind-rotation key resident on one GPU (CGGI binary/ternary or BMMP).
class GpuBlindRotator : public BlindRotator {
public:
    GpuBlindRotator(tp_br_variant variant, uint32_t N, uint32_t n, uint64_t basis, uint32_t digits,
                    const std::vector<uint64_t>& brk, int device = 0);
    ~GpuBlindRotator() override;
    GpuBlindRotator(const GpuBlindRotator&) = delete;
    GpuBlindRotator& operator=(const GpuBlindRotator&) = delete;

    void BlindRotate(std::vector<uint64_t>& result, const std::vector<uint64_t>& lwe_ciphertext,
                     std::vector<uint64_t>& accumulator, bool output_as_coefficients = false) override;
    void BlindRotate(uint64_t* result, const uint64_t* lwe_vec, uint64_t* accumulator,
                     bool output_as_coefficients = false) override;
    // Many rotations at once on host buffers (lwe rows of n+1 words, acc rows of 2N words
    // or one shared row when acc_stride == 0).
    void BlindRotateBatch(uint64_t batch, uint64_t* results, const uint64_t* lwes, const uint64_t* accs,
                          uint64_t acc_stride, bool output_as_coefficients = false);
    // GPU launch form (no reference counterpart; same output words in every form):
    // coefficients per thread (4 or 8), thread blocks per rotation (1, 2 or 4; 2 and 4
    // need 4 per thread), or both chosen by timing `batch` synthetic rotations.
    void SetTile(uint32_t coef_per_thread);
    void SetSplit(uint32_t blocks_per_rotation);
    // multiply-accumulate form (TP_MAC_ROWWISE / TP_MAC_DIGIT_STAGED) and NTT radix (2 or 4)
    void SetMacForm(uint32_t form);
    void SetRadix(uint32_t radix);
    uint32_t MacForm() const;
    uint32_t Radix() const;
    uint32_t Tile() const;
    uint32_t Split() const;
    // returns the chosen coefficients per thread (the split is read back with Split())
    uint32_t Autotune(uint64_t batch, double* rotations_per_s = nullptr);
    tp_br_ctx* Handle() const { return m_ctx; }
    uint32_t RingDimension() const { return m_N; }
    uint32_t LWEDimension() const { return m_n; }

private:
    tp_br_ctx* m_ctx = nullptr;
    uint32_t m_N, m_n;
};

// CGGIBlindRotationContext(distr, modulus, ring_dim, lwe_dim, basis, digits, std)
// (lib/src/operators/cggi_blind_rotation.cpp:14-25).
class CGGIBlindRotationContext : public std::enable_shared_from_this<CGGIBlindRotationContext> {
public:
    CGGIBlindRotationContext(KeyDistribution distr, uint64_t modulus, uint64_t ring_dim, uint64_t lwe_dim,
                             uint64_t basis, uint64_t digits, double std_dev, int device = 0, uint64_t seed = 1);
    // keys = {LWE key (n words; ternary -1 as any value other than 0/1), RLWE key (N words, coefficients)}
    std::unique_ptr<GpuBlindRotator> ConstructOperator(const std::vector<std::vector<uint64_t>>& keys) const;
    KeyDistribution GetKeyDistribution() const { return m_distr; }
    uint64_t GetModulus() const { return m_q; }
    uint64_t GetRingDimension() const { return m_N; }
    uint64_t GetLWEDimension() const { return m_n; }
    uint64_t GetBlindRotationBasis() const { return m_basis; }
    uint64_t GetBlindRotationRGSWDigits() const { return m_digits; }
    double GetStd() const { return m_std; }

private:
    KeyDistribution m_distr;
    uint64_t m_q, m_N, m_n, m_basis, m_digits;
    double m_std;
    int m_device;
    uint64_t m_seed;
};

// BMMPBlindRotationContext(distr, modulus, ring_dim, lwe_dim, basis, digits, std, step_size)
// (lib/src/operators/bmmp_blind_rotation.cpp:13-37); binary keys, step size 2.
class BMMPBlindRotationContext : public std::enable_shared_from_this<BMMPBlindRotationContext> {
public:
    BMMPBlindRotationContext(KeyDistribution distr, uint64_t modulus, uint64_t ring_dim, uint64_t lwe_dim,
                             uint64_t basis, uint64_t digits, double std_dev, uint64_t step_size, int device = 0,
                             uint64_t seed = 1);
    std::unique_ptr<GpuBlindRotator> ConstructOperator(const std::vector<std::vector<uint64_t>>& keys) const;

private:
    uint64_t m_N, m_n, m_basis, m_digits;
    double m_std;
    int m_device;
    uint64_t m_seed;
};

// NegacyclicFunctionEvaluator (lib/src/operators/negacyclic_function_evaluator.cpp:72-101):
// a programmable bootstrap = BlindRotate with coefficient output, then SampleExtract at 0.
// The result is an LWE of dimension N mod Q (N + 1 words). As in the reference,
// SampleExtract leaves a result word untouched where the rotated A coefficient is 0,
// and EvalFunc(function) builds the test RLWE with f(0) at A[0] and -f(N - i) at B[i]
// (lines 82-84), reproduced word for word.
class GpuNegacyclicFunctionEvaluator {
public:
    explicit GpuNegacyclicFunctionEvaluator(std::unique_ptr<GpuBlindRotator> rotator);
    void EvalFunc(uint64_t* result, const uint64_t* input_lwe, uint64_t* lut_rlwe);
    void EvalFunc(uint64_t* result, const uint64_t* input_lwe, std::function<uint64_t(uint64_t)>& function);
    void EvalFunc(std::vector<uint64_t>& result, const std::vector<uint64_t>& input, std::vector<uint64_t>& lut_rlwe);
    void EvalFunc(std::vector<uint64_t>& result, const std::vector<uint64_t>& input,
                  std::function<uint64_t(uint64_t)>& function);
    // Many at once on host buffers: lwes rows of n+1 words, luts rows of 2N words (lut_stride 0:
    // one shared test RLWE), results rows of N+1 words (extracted in place of what they hold).
    void EvalFuncBatch(uint64_t batch, uint64_t* results, const uint64_t* lwes, const uint64_t* luts,
                       uint64_t lut_stride);
    GpuBlindRotator& Rotator() { return *m_rot; }

private:
    std::unique_ptr<GpuBlindRotator> m_rot;
    std::vector<uint64_t> m_acc;
};

// RLWEtoRLWEConverter::Convert (lib/src/operators/rlwe_conversion.cpp:224-249).
class GpuRLWEtoRLWEConverter {
public:
    GpuRLWEtoRLWEConverter(uint32_t N, uint64_t basis, uint32_t digits, const std::vector<uint64_t>& ksk,
                           int device = 0);
    ~GpuRLWEtoRLWEConverter();
    // output -= KS(input.A); output.B += input.B  (output pre-zeroed by the caller, as in the reference)
    void Convert(uint64_t* output, const uint64_t* input);
    void Convert(std::vector<uint64_t>& output, const std::vector<uint64_t>& input);

private:
    tp_ks_ctx* m_ctx = nullptr;
    uint32_t m_N;
};

// AutomorphismEvaluator::Eval (lib/src/operators/automorphism_evaluation.cpp:150-159).
class GpuAutomorphismEvaluator {
public:
    GpuAutomorphismEvaluator(uint32_t N, uint64_t basis, uint32_t digits, uint32_t index,
                             const std::vector<uint64_t>& ksk, int device = 0);
    ~GpuAutomorphismEvaluator();
    void Eval(uint64_t* output, const uint64_t* input);

private:
    tp_ks_ctx* m_ctx = nullptr;
    uint32_t m_N;
};

// LWEtoRLWEPacker::Pack (lib/src/operators/lwe_to_rlwe_packing.cpp:129-236).
class GpuLWEtoRLWEPacker {
public:
    GpuLWEtoRLWEPacker(uint32_t N, uint64_t basis, uint32_t digits, const std::vector<uint64_t>& keys,
                       int device = 0);
    ~GpuLWEtoRLWEPacker();
    void Pack(uint64_t* output, const uint64_t* input, uint64_t len);
    // lwe_to_rlwe_packing.cpp:260-393: the inputs on the first len coefficients, any 2 <= len <= N
    void PackConsecutively(uint64_t* output, const uint64_t* input, uint64_t len);
    // One shard of a Pack split over devices (no reference counterpart): the subtree of len inputs
    // (L0 set-up and merges, no traces), its root (2N coefficient words) to `root`
    // (tp_pack_subtree_batch).
    void PackSubtree(uint64_t* root, const uint64_t* input, uint64_t len);
    // The tree above `count` roots of tree level `level0` (position order); with `finish` the
    // trailing traces as well, so `output` is what Pack gives for the whole tree
    // (tp_pack_merge_batch).
    void PackMerge(uint64_t* output, const uint64_t* roots, uint64_t count, uint32_t level0, bool finish);

private:
    tp_ks_ctx* m_ctx = nullptr;
    uint32_t m_N;
};

// LWEtoLWEConverter::Convert (lib/src/operators/lwe_conversion.cpp:205-239), Goldilocks modulus.
class GpuLWEtoLWEConverter {
public:
    GpuLWEtoLWEConverter(uint32_t n_in, uint32_t n_out, uint64_t basis, uint32_t digits,
                         const std::vector<uint64_t>& ksk, int device = 0);
    ~GpuLWEtoLWEConverter();
    void Convert(uint64_t* output, const uint64_t* input);

private:
    tp_lwe_ks_ctx* m_ctx = nullptr;
    uint32_t m_n_in, m_n_out;
};

// LWEtoRGSWConverter (lib/src/operators/lwe_to_rgsw_conversion.cpp:115-225): Convert writes
// 4 N out_digits words [lev_left rows | lev_right rows] in the NTT domain. The reference
// accumulates the squaring step into the caller's lev_left rows, so its callers pass a zeroed
// output; here those rows are written fresh, which is the same result.
class GpuLWEtoRGSWConverter {
public:
    GpuLWEtoRGSWConverter(const tp_br_params& rotation, uint64_t trace_basis, uint32_t trace_digits,
                          uint64_t square_basis, uint32_t square_digits, uint32_t out_digits, uint64_t out_basis,
                          const std::vector<uint64_t>& brk, const std::vector<uint64_t>& trace_keys,
                          const std::vector<uint64_t>& square_key, int device = 0);
    ~GpuLWEtoRGSWConverter();
    GpuLWEtoRGSWConverter(const GpuLWEtoRGSWConverter&) = delete;
    GpuLWEtoRGSWConverter& operator=(const GpuLWEtoRGSWConverter&) = delete;
    void Convert(uint64_t* output, const uint64_t* input);
    void Convert(std::vector<uint64_t>& output, const std::vector<uint64_t>& input);
    // Many at once on host buffers: lwes rows of n+1 words, outputs rows of 4 N out_digits words.
    void ConvertBatch(uint64_t batch, uint64_t* outputs, const uint64_t* lwes);
    uint64_t OutputWords() const { return 4ull * m_N * m_D; }

private:
    tp_ss_ctx* m_ctx = nullptr;
    uint32_t m_N, m_n, m_D;
};

// SchemeSwitchingContext(rotation, trace, squaring, output_digits, output_basis)
// (lib/src/operators/lwe_to_rgsw_conversion.cpp:10-108): the rotation context's parameters, the
// trace's and the squaring converter's gadgets, and the output gadget of the RGSW.
class SchemeSwitchingContext {
public:
    SchemeSwitchingContext(const tp_br_params& rotation, uint64_t trace_basis, uint64_t trace_digits,
                           uint64_t square_basis, uint64_t square_digits, uint64_t output_digits,
                           uint64_t output_basis, double std_dev, int device = 0, uint64_t seed = 1);
    // keys = {LWE key (n words), RLWE key (N words, coefficients)}
    std::unique_ptr<GpuLWEtoRGSWConverter> ConstructOperator(const std::vector<std::vector<uint64_t>>& keys) const;
    uint64_t GetOutputDigits() const { return m_out_digits; }
    uint64_t GetOutputBasis() const { return m_out_basis; }
    void SetOutputDigits(uint64_t d) { m_out_digits = d; }
    void SetOutputBasis(uint64_t b) { m_out_basis = b; }

private:
    tp_br_params m_rot;
    uint64_t m_tr_basis, m_tr_digits, m_sq_basis, m_sq_digits, m_out_digits, m_out_basis;
    double m_std;
    int m_device;
    uint64_t m_seed;
};

// SAPDecomposer (lib/src/operators/sap_decomposer.cpp:353-512). Decompose writes one LWE of
// dimension N per radix digit at output + d (N + 1); like the reference it stops at the digit
// count the input's words imply. The reference writes only the nonzero words of each digit
// into a caller-zeroed output; here every word of a digit is written.
class GpuSAPDecomposer {
public:
    GpuSAPDecomposer(const tp_br_params& rotation, uint64_t trace_basis, uint32_t trace_digits, uint64_t ks_basis,
                     uint32_t ks_digits, const std::vector<uint64_t>& brk, const std::vector<uint64_t>& trace_keys,
                     const std::vector<uint64_t>& lwe_ksk, uint64_t hamming_weight, uint64_t restart_period,
                     uint64_t max_digits = 64, int device = 0);
    ~GpuSAPDecomposer();
    GpuSAPDecomposer(const GpuSAPDecomposer&) = delete;
    GpuSAPDecomposer& operator=(const GpuSAPDecomposer&) = delete;
    void Decompose(uint64_t* output, const uint64_t* input, uint64_t radix);
    void Decompose(std::vector<uint64_t>& output, const std::vector<uint64_t>& input, uint64_t radix);
    // Many at once on host buffers: lwes rows of n+1 words; outputs rows of out_digits x (N+1)
    // words. Returns each LWE's digit count.
    std::vector<uint32_t> DecomposeBatch(uint64_t batch, uint64_t* outputs, uint64_t out_digits, const uint64_t* lwes,
                                         uint64_t radix);
    // HomTrunc (lines 189-291) and ResetAccumulator (lines 293-351), reference signatures;
    // 2N-word RLWEs in the NTT domain.
    void HomTrunc(uint64_t* output, uint64_t* input, uint64_t radix);
    void ResetAccumulator(uint64_t* acc, uint64_t radix);

private:
    tp_sap_ctx* m_ctx = nullptr;
    uint32_t m_N, m_n;
    uint64_t m_beta, m_restart, m_max_digits;
};

// SAPDecompositionContext(rotation, trace, LWE conversion N -> n, default_radix)
// (lib/src/operators/sap_decomposer.cpp:15-186). The reference derives the restart period from
// its floating-point variance models (ComputeRestartIterationForRadix, lines 78-145); those are
// not part of this path, so the period is given here (SAPDecompositionContext's
// GetRestartIteration(); UINT64_MAX: never).
class SAPDecompositionContext {
public:
    SAPDecompositionContext(const tp_br_params& rotation, uint64_t trace_basis, uint64_t trace_digits,
                            uint64_t ks_basis, uint64_t ks_digits, uint64_t default_radix, double std_dev,
                            uint64_t restart_period = ~0ull, int device = 0, uint64_t seed = 1);
    // keys = {LWE key (n words), RLWE key (N words, coefficients)}; the Hamming weight is the
    // LWE key's nonzero count, as in the reference (lines 170-174).
    std::unique_ptr<GpuSAPDecomposer> ConstructOperator(const std::vector<std::vector<uint64_t>>& keys) const;
    uint64_t GetDefaultRadix() const { return m_radix; }
    uint64_t GetRestartIteration() const { return m_restart; }

private:
    tp_br_params m_rot;
    uint64_t m_tr_basis, m_tr_digits, m_ks_basis, m_ks_digits, m_radix;
    double m_std;
    uint64_t m_restart;
    int m_device;
    uint64_t m_seed;
};

}  // namespace toothpaste_b200
