// Reference-side adapter: the reference's own BlindRotator interface over the GPU.
//
// Compiled INSIDE a Toothpaste build (it includes the reference's headers:
// interfaces/blindrotation_operator.h, operators/cggi_blind_rotation.h,
// operators/bmmp_blind_rotation.h) and linked against libtoothpaste_gpu.so.
//
//   auto cpu = std::make_shared<CGGIBlindRotationContext>(TERNARY, Q, N, n, 1 << 12, 3, 3.2);
//   auto gpu = std::make_shared<toothpaste_b200::GpuRotationContext>(cpu);
//   // any caller that takes an OperatorContext<BlindRotator> now rotates on the GPU:
//   auto eval = std::make_shared<NegacyclicFunctionEvaluationContext>(gpu);
//   auto op = eval->ConstructOperator({lwe_key, rlwe_key});
//
// GpuRotationContext is an OperatorContext<BlindRotator>
// (lib/include/interfaces/operator_context.h:22-63). Its ConstructOperator runs the
// reference operator's own key generation (CGGIBlindRotationContext::ConstructOperator,
// cggi_blind_rotation.cpp:184-199, or the BMMP one), so the keys are the ones the CPU
// operator would use, uploads the generated m_brk once in the reference's layout and
// returns a GpuReferenceRotator, a BlindRotator (blindrotation_operator.h:20-49) whose
// two BlindRotate overloads run on the GPU (tp_br_blind_rotate, host pointers; result
// may equal the accumulator, as SAPDecomposer passes it). Every other context query
// (variance model, containers, operator id) is answered by the wrapped CPU context,
// so callers that inspect it (NegacyclicFunctionEvaluator::EvalFunc,
// negacyclic_function_evaluator.cpp:70-101; LWEtoRGSWConverter,
// lwe_to_rgsw_conversion.cpp:85; SAPDecomposer, sap_decomposer.cpp:181,369,460) see
// the reference's values.
//
// The one addition the reference needs is read access to the generated key: the
// integrating build defines the two ReferenceRotationKey functions below, normally as
// `return op.BlindRotationKey();` over a const accessor returning m_brk added to
// CGGIBlindRotator and BMMPBlindRotator.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "interfaces/blindrotation_operator.h"
#include "operators/bmmp_blind_rotation.h"
#include "operators/cggi_blind_rotation.h"
#include "toothpaste_gpu.h"

namespace toothpaste_b200 {

// The generated blind-rotation key (m_brk) of a constructed reference operator.
const AlignedBuffer& ReferenceRotationKey(const CGGIBlindRotator& op);
const AlignedBuffer& ReferenceRotationKey(const BMMPBlindRotator& op);

inline void adapter_check(tp_status s) {
    if (s != TP_OK) throw std::runtime_error(std::string("toothpaste_gpu: ") + tp_last_error());
}

class GpuRotationContext;

// BlindRotator whose rotations run on the GPU with an uploaded key.
class GpuReferenceRotator : public BlindRotator {
public:
    GpuReferenceRotator(std::shared_ptr<const GpuRotationContext> ctx, const tp_br_params& p, const uint64_t* brk,
                        uint64_t words, int device)
        : m_ctx(std::move(ctx)), m_N(p.ring_dim) {
        adapter_check(tp_br_create(&p, device, &m_gpu));
        const tp_status s = tp_br_upload_key(m_gpu, brk, words);
        if (s != TP_OK) {
            tp_br_destroy(m_gpu);
            adapter_check(s);
        }
    }
    GpuReferenceRotator(const GpuReferenceRotator&) = delete;
    GpuReferenceRotator& operator=(const GpuReferenceRotator&) = delete;
    ~GpuReferenceRotator() override { tp_br_destroy(m_gpu); }

    void BlindRotate(uint64_t* result, const uint64_t* lwe_vec, uint64_t* accumulator,
                     bool output_as_coefficients = false) override {
        adapter_check(tp_br_blind_rotate(m_gpu, result, lwe_vec, accumulator, output_as_coefficients ? 1 : 0));
    }

    void BlindRotate(std::vector<uint64_t>& result, const std::vector<uint64_t>& lwe_ciphertext,
                     std::vector<uint64_t>& accumulator, bool output_as_coefficients = false) override {
        result.resize(2 * m_N);
        BlindRotate(result.data(), lwe_ciphertext.data(), accumulator.data(), output_as_coefficients);
    }

    [[nodiscard]] const std::shared_ptr<const OperatorContext<BlindRotator>> GetContext() const override;

    tp_br_ctx* Handle() const { return m_gpu; }

private:
    std::shared_ptr<const GpuRotationContext> m_ctx;
    uint64_t m_N;
    tp_br_ctx* m_gpu = nullptr;
};

// OperatorContext<BlindRotator> over a reference CGGI or BMMP context.
class GpuRotationContext : public OperatorContext<BlindRotator>,
                           public std::enable_shared_from_this<GpuRotationContext> {
public:
    explicit GpuRotationContext(std::shared_ptr<CGGIBlindRotationContext> cggi, int device = 0)
        : m_cggi(std::move(cggi)), m_device(device) {
        m_params = {m_cggi->GetKeyDistribution() == KeyDistribution::BINARY ? TP_BR_CGGI_BINARY : TP_BR_CGGI_TERNARY,
                    m_cggi->GetModulus(), (uint32_t)m_cggi->GetRingDimension(), (uint32_t)m_cggi->GetLWEDimension(),
                    m_cggi->GetBlindRotationBasis(), (uint32_t)m_cggi->GetBlindRotationRGSWDigits()};
    }
    explicit GpuRotationContext(std::shared_ptr<BMMPBlindRotationContext> bmmp, int device = 0)
        : m_bmmp(std::move(bmmp)), m_device(device) {
        m_params = {TP_BR_BMMP_BINARY, m_bmmp->GetModulus(), (uint32_t)m_bmmp->GetRingDimension(),
                    (uint32_t)m_bmmp->GetLWEDimension(), m_bmmp->GetBlindRotationBasis(),
                    (uint32_t)m_bmmp->GetBlindRotationRGSWDigits()};
    }

    [[nodiscard]] long double ComputeOutputVariance(long double input_variance = 0.0) const override {
        return m_cggi ? m_cggi->ComputeOutputVariance(input_variance) : m_bmmp->ComputeOutputVariance(input_variance);
    }
    [[nodiscard]] Container GetInputContainer() const override {
        return m_cggi ? m_cggi->GetInputContainer() : m_bmmp->GetInputContainer();
    }
    [[nodiscard]] Container GetOutputContainer(Container input) const override {
        return m_cggi ? m_cggi->GetOutputContainer(std::move(input)) : m_bmmp->GetOutputContainer(std::move(input));
    }
    [[nodiscard]] OperatorID GetOperatorID() const override {
        return m_cggi ? m_cggi->GetOperatorID() : m_bmmp->GetOperatorID();
    }

    // Runs the reference operator's key generation, then uploads its key to the GPU.
    [[nodiscard]] std::unique_ptr<BlindRotator> ConstructOperator(const std::vector<GenericKey>& keys) const override {
        auto self = shared_from_this();
        if (m_cggi) {
            auto cpu = m_cggi->ConstructOperator(keys);
            const AlignedBuffer& brk = ReferenceRotationKey(*cpu);
            return std::make_unique<GpuReferenceRotator>(self, m_params, brk.data(), brk.size(), m_device);
        }
        auto cpu = m_bmmp->ConstructOperator(keys);
        const AlignedBuffer& brk = ReferenceRotationKey(*cpu);
        return std::make_unique<GpuReferenceRotator>(self, m_params, brk.data(), brk.size(), m_device);
    }

    const tp_br_params& Params() const { return m_params; }

private:
    std::shared_ptr<CGGIBlindRotationContext> m_cggi;
    std::shared_ptr<BMMPBlindRotationContext> m_bmmp;
    int m_device = 0;
    tp_br_params m_params{};
};

inline const std::shared_ptr<const OperatorContext<BlindRotator>> GpuReferenceRotator::GetContext() const {
    return m_ctx;
}

}  // namespace toothpaste_b200
