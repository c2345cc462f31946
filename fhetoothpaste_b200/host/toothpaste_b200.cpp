// Host side of the C++ drop-in operators: key generation and the Gpu* wrappers.
#include "toothpaste_b200.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

namespace toothpaste_b200 {

namespace {

using u128 = unsigned __int128;
constexpr uint64_t P = kGoldilocks;

uint64_t addp(uint64_t a, uint64_t b) {
    const u128 s = (u128)a + b;
    return (uint64_t)(s >= P ? s - P : s);
}
uint64_t subp(uint64_t a, uint64_t b) { return a >= b ? a - b : a + (P - b); }
uint64_t mulp(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % P); }
uint64_t powp(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= P;
    for (; e; e >>= 1, b = mulp(b, b))
        if (e & 1) r = mulp(r, b);
    return r;
}

// Host negacyclic NTT with the reference's slot order (natural coefficients in,
// slot k = a(psi^(2 brv(k) + 1)) out), used only for key generation.
class HostNtt {
public:
    explicit HostNtt(uint32_t N) : m_N(N) {
        int logn = 0;
        while ((1u << logn) < N) ++logn;
        const uint64_t psi = powp(7, (P - 1) >> (logn + 1));
        m_tw.resize(N);
        for (uint32_t k = 0; k < N; ++k) {
            uint32_t r = 0;
            for (int b = 0; b < logn; ++b) r |= ((k >> b) & 1u) << (logn - 1 - b);
            m_tw[k] = powp(psi, r);
        }
    }
    void Forward(uint64_t* a) const {
        for (uint32_t m = 1, t = m_N / 2; m < m_N; m <<= 1, t >>= 1)
            for (uint32_t i = 0; i < m; ++i) {
                const uint64_t w = m_tw[m + i];
                for (uint32_t j = 2 * i * t; j < 2 * i * t + t; ++j) {
                    const uint64_t u = a[j], v = mulp(a[j + t], w);
                    a[j] = addp(u, v);
                    a[j + t] = subp(u, v);
                }
            }
    }

private:
    uint32_t m_N;
    std::vector<uint64_t> m_tw;
};

const HostNtt& ntt_for(uint32_t N) {
    static std::mutex mu;
    static std::vector<std::unique_ptr<HostNtt>> cache(17);
    int logn = 0;
    while ((1u << logn) < N) ++logn;
    std::lock_guard<std::mutex> lk(mu);
    if (!cache[logn]) cache[logn] = std::make_unique<HostNtt>(N);
    return *cache[logn];
}

// RLWE(msg): A uniform (taken as NTT domain), B = A*s + NTT(e + msg) or NTT(e) + msg.
void make_rlwe(Sampler& rng, uint32_t N, double sd, uint64_t* out, const uint64_t* msg, const uint64_t* s_ntt,
               bool msg_is_ntt) {
    std::vector<uint64_t> e(N);
    for (uint32_t i = 0; i < N; ++i) out[i] = rng.Uniform(P);
    for (uint32_t i = 0; i < N; ++i) e[i] = rng.Gaussian(sd, P);
    for (uint32_t i = 0; i < N; ++i) out[N + i] = mulp(out[i], s_ntt[i]);
    const HostNtt& ntt = ntt_for(N);
    if (msg_is_ntt) {
        ntt.Forward(e.data());
        for (uint32_t i = 0; i < N; ++i) e[i] = addp(e[i], msg[i]);
    } else {
        for (uint32_t i = 0; i < N; ++i) e[i] = addp(e[i], msg[i]);
        ntt.Forward(e.data());
    }
    for (uint32_t i = 0; i < N; ++i) out[N + i] = addp(out[N + i], e[i]);
}

// RGSW(msg) with msg in coefficients: rows 0..l-1 encrypt -s*m*g_j, rows l..2l-1 m*g_j,
// g_j = B^(max_digits-1-j) (the row order of lib/src/base_crypto.cpp:60-97).
void make_rgsw(Sampler& rng, uint32_t N, double sd, uint64_t* out, const uint64_t* msg, const uint64_t* s_ntt,
               uint64_t basis, uint32_t digits) {
    std::vector<uint64_t> tmp(3 * N, 0);
    const uint64_t max_digits = (uint64_t)std::ceil(std::log2((long double)P) / std::log2((long double)basis));
    std::memcpy(tmp.data(), msg, N * 8);
    ntt_for(N).Forward(tmp.data());
    for (uint32_t i = 0; i < N; ++i) tmp[2 * N + i] = mulp(tmp[i], s_ntt[i]);
    for (uint32_t i = 0; i < N; ++i) tmp[N + i] = subp(0, tmp[2 * N + i]);
    for (uint64_t d = 0; d + digits < max_digits; ++d)
        for (uint32_t i = 0; i < 2 * N; ++i) tmp[i] = mulp(tmp[i], basis);
    for (uint32_t d = 0; d < digits; ++d) {
        const uint64_t off = digits - d - 1;
        make_rlwe(rng, N, sd, out + off * 2 * N, tmp.data() + N, s_ntt, true);
        make_rlwe(rng, N, sd, out + off * 2 * N + 2ull * N * digits, tmp.data(), s_ntt, true);
        for (uint32_t i = 0; i < 2 * N; ++i) tmp[i] = mulp(tmp[i], basis);
    }
}

std::vector<uint64_t> ntt_of(const std::vector<uint64_t>& a) {
    std::vector<uint64_t> r(a);
    for (auto& x : r) x %= P;
    ntt_for((uint32_t)r.size()).Forward(r.data());
    return r;
}

}  // namespace

uint64_t Sampler::Next() {
    uint64_t z = (m_s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t Sampler::Uniform(uint64_t q) {
    if (q == 0) return Next();
    uint64_t mask = q - 1;
    for (int s = 1; s < 64; s <<= 1) mask |= mask >> s;
    for (;;) {
        const uint64_t x = Next() & mask;
        if (x < q) return x;
    }
}

uint64_t Sampler::Gaussian(double sd, uint64_t q) {
    if (sd == 0.0) return 0;
    const double u1 = (double)((Next() >> 11) + 1) * 0x1.0p-53;
    const double u2 = (double)(Next() >> 11) * 0x1.0p-53;
    const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    const long long k = std::llround(z * sd);
    if (k >= 0) return (uint64_t)k % q;
    const uint64_t m = (uint64_t)(-k) % q;
    return m == 0 ? 0 : q - m;
}

namespace keygen {

std::vector<uint64_t> BlindRotationKey(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t basis_log2,
                                       uint32_t digits, double sd, const std::vector<uint64_t>& lwe_key,
                                       const std::vector<uint64_t>& rlwe_key) {
    const uint64_t L = 1ull << basis_log2;
    const uint64_t rg = 4ull * N * digits;
    const std::vector<uint64_t> s = ntt_of(rlwe_key);
    std::vector<uint64_t> data(2 * N, 0);
    std::vector<uint64_t> brk;
    if (variant == TP_BR_CGGI_BINARY) {  // cggi_blind_rotation.cpp:264-280
        brk.resize(n * rg);
        for (uint32_t i = 0; i < n; ++i) {
            data[0] = lwe_key[i];
            make_rgsw(rng, N, sd, brk.data() + i * rg, data.data(), s.data(), L, digits);
        }
    } else if (variant == TP_BR_CGGI_TERNARY) {  // cggi_blind_rotation.cpp:282-311
        brk.resize(2ull * n * rg);
        for (uint32_t i = 0; i < n; ++i) {
            data[0] = lwe_key[i] == 1;
            data[N] = lwe_key[i] != 0 && lwe_key[i] != 1;
            make_rgsw(rng, N, sd, brk.data() + 2 * i * rg, data.data(), s.data(), L, digits);
            make_rgsw(rng, N, sd, brk.data() + 2 * i * rg + rg, data.data() + N, s.data(), L, digits);
        }
    } else {  // BMMP, bmmp_blind_rotation.cpp:229-262
        brk.resize(3ull * (n / 2) * rg);
        for (uint32_t i = 0; i < n; i += 2) {
            uint64_t* chunk = brk.data() + 3ull * (i / 2) * rg;
            data[0] = lwe_key[i];
            make_rgsw(rng, N, sd, chunk, data.data(), s.data(), L, digits);
            data[0] = lwe_key[i + 1];
            make_rgsw(rng, N, sd, chunk + rg, data.data(), s.data(), L, digits);
            data[0] = lwe_key[i + 1] * lwe_key[i];
            make_rgsw(rng, N, sd, chunk + 2 * rg, data.data(), s.data(), L, digits);
        }
    }
    return brk;
}

std::vector<uint64_t> RLWESwitchingKey(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double sd,
                                       const std::vector<uint64_t>& source_key, const std::vector<uint64_t>& target_key) {
    // rlwe_conversion.cpp:187-218: chunk i encrypts source * 2^(64 - beta - i*beta) under target
    const std::vector<uint64_t> t = ntt_of(target_key);
    std::vector<uint64_t> ksk(2ull * N * digits), g(N);
    uint64_t gij = 1ull << (64 - basis_log2);
    for (uint32_t i = 0; i < digits; ++i) {
        for (uint32_t k = 0; k < N; ++k) g[k] = mulp(source_key[k] % P, gij % P);
        make_rlwe(rng, N, sd, ksk.data() + 2ull * i * N, g.data(), t.data(), false);
        gij >>= basis_log2;
        if (gij == 0) gij = 1;
    }
    return ksk;
}

std::vector<uint64_t> AutomorphismKey(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double sd,
                                      uint32_t index, const std::vector<uint64_t>& key) {
    // automorphism_evaluation.cpp:43-63: switch from s(X^index) back to s(X)
    std::vector<uint64_t> ka(N);
    for (uint32_t i = 0; i < N; ++i) {
        const uint64_t tpos = ((uint64_t)i * index) & (2ull * N - 1);
        const uint64_t v = key[i] % P;
        ka[tpos & (N - 1)] = tpos >= N ? (v == 0 ? 0 : P - v) : v;
    }
    return RLWESwitchingKey(rng, N, basis_log2, digits, sd, ka, key);
}

std::vector<uint64_t> PackingKeys(Sampler& rng, uint32_t N, uint32_t basis_log2, uint32_t digits, double sd,
                                  const std::vector<uint64_t>& key) {
    // lwe_to_rlwe_packing.cpp:46-58: one key per index 2^j + 1, j = 1..log2 N
    std::vector<uint64_t> all;
    for (uint32_t j = 1; (1u << j) <= N; ++j) {
        const auto k = AutomorphismKey(rng, N, basis_log2, digits, sd, (1u << j) + 1, key);
        all.insert(all.end(), k.begin(), k.end());
    }
    return all;
}

std::vector<uint64_t> LWESwitchingKey(Sampler& rng, uint32_t n_in, uint32_t n_out, uint32_t basis_log2,
                                      uint32_t digits, double sd, const std::vector<uint64_t>& source_key,
                                      const std::vector<uint64_t>& target_key) {
    std::vector<uint64_t> ksk((uint64_t)n_in * digits * (n_out + 1ull));
    for (uint32_t i = 0; i < n_in; ++i) {
        uint64_t g = 1ull << (64 - basis_log2);  // IntLog2(p) = 64
        for (uint32_t j = 0; j < digits; ++j, g >>= basis_log2) {
            uint64_t* row = ksk.data() + ((uint64_t)i * digits + j) * (n_out + 1ull);
            // LWEEncryptor::MakeLWE (base_crypto.cpp:137-155): a uniform, b = e + <a, t> + msg
            for (uint32_t k = 0; k < n_out; ++k) row[k] = rng.Uniform(P);
            uint64_t b = rng.Gaussian(sd, P);
            for (uint32_t k = 0; k < n_out; ++k) b = addp(b, mulp(row[k], target_key[k] % P));
            row[n_out] = addp(b, mulp(g % P, source_key[i] % P));
        }
    }
    return ksk;
}

SAPKeySet SAPKeys(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t br_bl, uint32_t br_dg, uint32_t tr_bl,
                  uint32_t tr_dg, uint32_t ks_bl, uint32_t ks_dg, double sd, const std::vector<uint64_t>& lwe_key,
                  const std::vector<uint64_t>& rlwe_key) {
    SAPKeySet k;
    k.rotation = BlindRotationKey(rng, variant, N, n, br_bl, br_dg, sd, lwe_key, rlwe_key);
    k.trace = PackingKeys(rng, N, tr_bl, tr_dg, sd, rlwe_key);
    k.lwe_switch = LWESwitchingKey(rng, N, n, ks_bl, ks_dg, sd, rlwe_key, lwe_key);
    return k;
}

SchemeSwitchingKeySet SchemeSwitchingKeys(Sampler& rng, int variant, uint32_t N, uint32_t n, uint32_t br_bl,
                                          uint32_t br_dg, uint32_t tr_bl, uint32_t tr_dg, uint32_t sq_bl,
                                          uint32_t sq_dg, double sd, const std::vector<uint64_t>& lwe_key,
                                          const std::vector<uint64_t>& rlwe_key) {
    SchemeSwitchingKeySet k;
    k.rotation = BlindRotationKey(rng, variant, N, n, br_bl, br_dg, sd, lwe_key, rlwe_key);
    k.trace = PackingKeys(rng, N, tr_bl, tr_dg, sd, rlwe_key);
    // s^2 in Z_p[X]/(X^N + 1) (the reference's INTT(NTT(s)^2), lines 91-94), schoolbook
    std::vector<uint64_t> sq(N, 0);
    for (uint32_t i = 0; i < N; ++i) {
        const uint64_t a = rlwe_key[i] % P;
        if (!a) continue;
        for (uint32_t j = 0; j < N; ++j) {
            const uint64_t t = mulp(a, rlwe_key[j] % P);
            const uint32_t d = i + j;
            if (d < N) sq[d] = addp(sq[d], t);
            else sq[d - N] = subp(sq[d - N], t);
        }
    }
    k.square = RLWESwitchingKey(rng, N, sq_bl, sq_dg, sd, sq, rlwe_key);
    return k;
}

}  // namespace keygen

// ---- GpuBlindRotator ----

GpuBlindRotator::GpuBlindRotator(tp_br_variant variant, uint32_t N, uint32_t n, uint64_t basis, uint32_t digits,
                                 const std::vector<uint64_t>& brk, int device)
    : m_N(N), m_n(n) {
    tp_br_params p{variant, kGoldilocks, N, n, basis, digits};
    check(tp_br_create(&p, device, &m_ctx));
    tp_status s = tp_br_upload_key(m_ctx, brk.data(), brk.size());
    if (s != TP_OK) {
        tp_br_destroy(m_ctx);
        check(s);
    }
}

GpuBlindRotator::~GpuBlindRotator() { tp_br_destroy(m_ctx); }

void GpuBlindRotator::BlindRotate(uint64_t* result, const uint64_t* lwe_vec, uint64_t* accumulator,
                                  bool output_as_coefficients) {
    check(tp_br_blind_rotate(m_ctx, result, lwe_vec, accumulator, output_as_coefficients ? 1 : 0));
}

void GpuBlindRotator::BlindRotate(std::vector<uint64_t>& result, const std::vector<uint64_t>& lwe_ciphertext,
                                  std::vector<uint64_t>& accumulator, bool output_as_coefficients) {
    if (lwe_ciphertext.size() < m_n + 1u || accumulator.size() < 2ull * m_N)
        throw std::invalid_argument("toothpaste_b200: LWE or accumulator shorter than the operator's dimensions");
    result.resize(2ull * m_N);
    BlindRotate(result.data(), lwe_ciphertext.data(), accumulator.data(), output_as_coefficients);
}

void GpuBlindRotator::BlindRotateBatch(uint64_t batch, uint64_t* results, const uint64_t* lwes, const uint64_t* accs,
                                       uint64_t acc_stride, bool output_as_coefficients) {
    check(tp_br_blind_rotate_batch_host(m_ctx, batch, results, lwes, m_n + 1, accs, acc_stride,
                                        output_as_coefficients ? 1 : 0, nullptr));
    check(tp_br_check(m_ctx, nullptr));
}

void GpuBlindRotator::SetTile(uint32_t coef_per_thread) { check(tp_br_set_tile(m_ctx, coef_per_thread)); }

void GpuBlindRotator::SetSplit(uint32_t blocks_per_rotation) { check(tp_br_set_split(m_ctx, blocks_per_rotation)); }

uint32_t GpuBlindRotator::Tile() const { return tp_br_get_tile(m_ctx); }

uint32_t GpuBlindRotator::Split() const { return tp_br_get_split(m_ctx); }

void GpuBlindRotator::SetMacForm(uint32_t form) { check(tp_br_set_mac_form(m_ctx, form)); }

void GpuBlindRotator::SetRadix(uint32_t radix) { check(tp_br_set_radix(m_ctx, radix)); }

uint32_t GpuBlindRotator::MacForm() const { return tp_br_get_mac_form(m_ctx); }

uint32_t GpuBlindRotator::Radix() const { return tp_br_get_radix(m_ctx); }

uint32_t GpuBlindRotator::Autotune(uint64_t batch, double* rotations_per_s) {
    uint32_t coef = 0;
    check(tp_br_autotune(m_ctx, batch, &coef, rotations_per_s));
    return coef;
}

// ---- contexts ----

CGGIBlindRotationContext::CGGIBlindRotationContext(KeyDistribution distr, uint64_t modulus, uint64_t ring_dim,
                                                   uint64_t lwe_dim, uint64_t basis, uint64_t digits, double std_dev,
                                                   int device, uint64_t seed)
    : m_distr(distr), m_q(modulus), m_N(ring_dim), m_n(lwe_dim), m_basis(basis), m_digits(digits), m_std(std_dev),
      m_device(device), m_seed(seed) {
    if (modulus != kGoldilocks) throw std::invalid_argument("toothpaste_b200: only the Goldilocks modulus is served");
    if (distr == GAUSSIAN) throw std::invalid_argument("toothpaste_b200: Gaussian LWE keys are not supported");
}

std::unique_ptr<GpuBlindRotator> CGGIBlindRotationContext::ConstructOperator(
    const std::vector<std::vector<uint64_t>>& keys) const {
    if (keys.size() < 2 || keys[0].size() < m_n || keys[1].size() < m_N)
        throw std::invalid_argument("toothpaste_b200: keys = {LWE key (n), RLWE key (N)}");
    int beta = 0;
    while ((1ull << beta) < m_basis) ++beta;
    const int variant = m_distr == BINARY ? TP_BR_CGGI_BINARY : TP_BR_CGGI_TERNARY;
    Sampler rng(m_seed);
    const auto brk = keygen::BlindRotationKey(rng, variant, (uint32_t)m_N, (uint32_t)m_n, (uint32_t)beta,
                                              (uint32_t)m_digits, m_std, keys[0], keys[1]);
    return std::make_unique<GpuBlindRotator>((tp_br_variant)variant, (uint32_t)m_N, (uint32_t)m_n, m_basis,
                                             (uint32_t)m_digits, brk, m_device);
}

BMMPBlindRotationContext::BMMPBlindRotationContext(KeyDistribution distr, uint64_t modulus, uint64_t ring_dim,
                                                   uint64_t lwe_dim, uint64_t basis, uint64_t digits, double std_dev,
                                                   uint64_t step_size, int device, uint64_t seed)
    : m_N(ring_dim), m_n(lwe_dim), m_basis(basis), m_digits(digits), m_std(std_dev), m_device(device), m_seed(seed) {
    // the reference asserts these (bmmp_blind_rotation.cpp:16-24)
    if (step_size != 2) throw std::invalid_argument("toothpaste_b200: BMMP supports step size 2 only");
    if (lwe_dim % step_size) throw std::invalid_argument("toothpaste_b200: LWE dimension not divisible by 2");
    if (distr != BINARY) throw std::invalid_argument("toothpaste_b200: BMMP needs binary keys");
    if (modulus != kGoldilocks) throw std::invalid_argument("toothpaste_b200: only the Goldilocks modulus is served");
}

std::unique_ptr<GpuBlindRotator> BMMPBlindRotationContext::ConstructOperator(
    const std::vector<std::vector<uint64_t>>& keys) const {
    if (keys.size() < 2 || keys[0].size() < m_n || keys[1].size() < m_N)
        throw std::invalid_argument("toothpaste_b200: keys = {LWE key (n), RLWE key (N)}");
    int beta = 0;
    while ((1ull << beta) < m_basis) ++beta;
    Sampler rng(m_seed);
    const auto brk = keygen::BlindRotationKey(rng, TP_BR_BMMP_BINARY, (uint32_t)m_N, (uint32_t)m_n, (uint32_t)beta,
                                              (uint32_t)m_digits, m_std, keys[0], keys[1]);
    return std::make_unique<GpuBlindRotator>(TP_BR_BMMP_BINARY, (uint32_t)m_N, (uint32_t)m_n, m_basis,
                                             (uint32_t)m_digits, brk, m_device);
}

// ---- programmable bootstrap ----

namespace {
// SampleExtract at index 0 (lib/include/static/sample_extraction.h:20-36): a word of the
// result is written only where the source coefficient is non-zero.
void sample_extract0(uint64_t* out, const uint64_t* rlwe, uint64_t N) {
    out[0] = rlwe[0];
    for (uint64_t i = 1; i < N; ++i)
        if (rlwe[N - i] != 0) out[i] = P - rlwe[N - i];
    out[N] = rlwe[N];
}
}  // namespace

GpuNegacyclicFunctionEvaluator::GpuNegacyclicFunctionEvaluator(std::unique_ptr<GpuBlindRotator> rotator)
    : m_rot(std::move(rotator)) {
    if (!m_rot) throw std::invalid_argument("toothpaste_b200: null rotator");
    m_acc.assign(2ull * m_rot->RingDimension(), 0);
}

void GpuNegacyclicFunctionEvaluator::EvalFunc(uint64_t* result, const uint64_t* input_lwe, uint64_t* lut_rlwe) {
    const uint64_t N = m_rot->RingDimension();
    m_rot->BlindRotate(m_acc.data(), input_lwe, lut_rlwe, true);
    sample_extract0(result, m_acc.data(), N);
}

void GpuNegacyclicFunctionEvaluator::EvalFunc(uint64_t* result, const uint64_t* input_lwe,
                                              std::function<uint64_t(uint64_t)>& function) {
    const uint64_t N = m_rot->RingDimension();
    std::vector<uint64_t> tmp(2 * N, 0);
    tmp[0] = function(0);  // negacyclic_function_evaluator.cpp:82-84, as the reference places it
    for (uint64_t i = 1; i < N; ++i) tmp[i + N] = subp(0, function(N - i) % P);
    EvalFunc(result, input_lwe, tmp.data());
}

void GpuNegacyclicFunctionEvaluator::EvalFunc(std::vector<uint64_t>& result, const std::vector<uint64_t>& input,
                                              std::vector<uint64_t>& lut_rlwe) {
    result.resize(m_rot->RingDimension() + 1ull);
    EvalFunc(result.data(), input.data(), lut_rlwe.data());
}

void GpuNegacyclicFunctionEvaluator::EvalFunc(std::vector<uint64_t>& result, const std::vector<uint64_t>& input,
                                              std::function<uint64_t(uint64_t)>& function) {
    result.resize(m_rot->RingDimension() + 1ull);
    EvalFunc(result.data(), input.data(), function);
}

void GpuNegacyclicFunctionEvaluator::EvalFuncBatch(uint64_t batch, uint64_t* results, const uint64_t* lwes,
                                                   const uint64_t* luts, uint64_t lut_stride) {
    const uint64_t N = m_rot->RingDimension();
    std::vector<uint64_t> rl(batch * 2 * N);
    m_rot->BlindRotateBatch(batch, rl.data(), lwes, luts, lut_stride, true);
    for (uint64_t b = 0; b < batch; ++b) sample_extract0(results + b * (N + 1), rl.data() + b * 2 * N, N);
}

// ---- key switching wrappers (synchronous, host buffers) ----

namespace {
struct DevBuf {
    uint64_t* p = nullptr;
    explicit DevBuf(size_t words) {
        if (words && cudaMalloc(reinterpret_cast<void**>(&p), words * 8) != cudaSuccess)
            throw std::runtime_error("toothpaste_b200: device allocation failed");
    }
    ~DevBuf() { cudaFree(p); }
};
}  // namespace

GpuRLWEtoRLWEConverter::GpuRLWEtoRLWEConverter(uint32_t N, uint64_t basis, uint32_t digits,
                                               const std::vector<uint64_t>& ksk, int device)
    : m_N(N) {
    check(tp_rlwe_ks_create(N, basis, digits, device, &m_ctx));
    check(tp_ks_upload_key(m_ctx, ksk.data(), ksk.size()));
}
GpuRLWEtoRLWEConverter::~GpuRLWEtoRLWEConverter() { tp_ks_destroy(m_ctx); }

void GpuRLWEtoRLWEConverter::Convert(uint64_t* output, const uint64_t* input) {
    DevBuf din(2ull * m_N), dout(2ull * m_N);
    cudaMemcpy(din.p, input, 16ull * m_N, cudaMemcpyHostToDevice);
    cudaMemcpy(dout.p, output, 16ull * m_N, cudaMemcpyHostToDevice);
    check(tp_rlwe_ks_batch(m_ctx, 1, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuRLWEtoRLWEConverter::Convert(std::vector<uint64_t>& output, const std::vector<uint64_t>& input) {
    output.resize(2ull * m_N);
    Convert(output.data(), input.data());
}

GpuAutomorphismEvaluator::GpuAutomorphismEvaluator(uint32_t N, uint64_t basis, uint32_t digits, uint32_t index,
                                                   const std::vector<uint64_t>& ksk, int device)
    : m_N(N) {
    check(tp_auto_create(N, basis, digits, index, device, &m_ctx));
    check(tp_ks_upload_key(m_ctx, ksk.data(), ksk.size()));
}
GpuAutomorphismEvaluator::~GpuAutomorphismEvaluator() { tp_ks_destroy(m_ctx); }

void GpuAutomorphismEvaluator::Eval(uint64_t* output, const uint64_t* input) {
    DevBuf din(2ull * m_N), dout(2ull * m_N);
    cudaMemcpy(din.p, input, 16ull * m_N, cudaMemcpyHostToDevice);
    cudaMemcpy(dout.p, output, 16ull * m_N, cudaMemcpyHostToDevice);
    check(tp_auto_eval_batch(m_ctx, 1, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

GpuLWEtoRLWEPacker::GpuLWEtoRLWEPacker(uint32_t N, uint64_t basis, uint32_t digits, const std::vector<uint64_t>& keys,
                                       int device)
    : m_N(N) {
    check(tp_pack_create(N, basis, digits, device, &m_ctx));
    check(tp_ks_upload_key(m_ctx, keys.data(), keys.size()));
}
GpuLWEtoRLWEPacker::~GpuLWEtoRLWEPacker() { tp_ks_destroy(m_ctx); }

void GpuLWEtoRLWEPacker::Pack(uint64_t* output, const uint64_t* input, uint64_t len) {
    DevBuf din(len * (m_N + 1ull)), dout(2ull * m_N);
    cudaMemcpy(din.p, input, len * (m_N + 1ull) * 8, cudaMemcpyHostToDevice);
    check(tp_pack_batch(m_ctx, 1, len, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuLWEtoRLWEPacker::PackConsecutively(uint64_t* output, const uint64_t* input, uint64_t len) {
    DevBuf din(len * (m_N + 1ull)), dout(2ull * m_N);
    if (cudaMemcpy(din.p, input, len * (m_N + 1ull) * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_pack_consecutive_batch(m_ctx, 1, len, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuLWEtoRLWEPacker::PackSubtree(uint64_t* root, const uint64_t* input, uint64_t len) {
    DevBuf din(len * (m_N + 1ull)), dout(2ull * m_N);
    if (cudaMemcpy(din.p, input, len * (m_N + 1ull) * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_pack_subtree_batch(m_ctx, 1, len, dout.p, din.p, nullptr));
    if (cudaMemcpy(root, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuLWEtoRLWEPacker::PackMerge(uint64_t* output, const uint64_t* roots, uint64_t count, uint32_t level0,
                                   bool finish) {
    DevBuf din(count * 2ull * m_N), dout(2ull * m_N);
    if (cudaMemcpy(din.p, roots, count * 16ull * m_N, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_pack_merge_batch(m_ctx, 1, count, level0, finish ? 1 : 0, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, 16ull * m_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

GpuLWEtoLWEConverter::GpuLWEtoLWEConverter(uint32_t n_in, uint32_t n_out, uint64_t basis, uint32_t digits,
                                           const std::vector<uint64_t>& ksk, int device)
    : m_n_in(n_in), m_n_out(n_out) {
    check(tp_lwe_ks_create(kGoldilocks, n_in, n_out, basis, digits, device, &m_ctx));
    check(tp_lwe_ks_upload_key(m_ctx, ksk.data(), ksk.size()));
}
GpuLWEtoLWEConverter::~GpuLWEtoLWEConverter() { tp_lwe_ks_destroy(m_ctx); }

void GpuLWEtoLWEConverter::Convert(uint64_t* output, const uint64_t* input) {
    DevBuf din(m_n_in + 1ull), dout(m_n_out + 1ull);
    cudaMemcpy(din.p, input, (m_n_in + 1ull) * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dout.p, output, (m_n_out + 1ull) * 8, cudaMemcpyHostToDevice);
    check(tp_lwe_ks_batch(m_ctx, 1, dout.p, din.p, nullptr));
    if (cudaMemcpy(output, dout.p, (m_n_out + 1ull) * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

// ---- scheme switching ----

static uint32_t log2_of(uint64_t b) {
    uint32_t k = 0;
    while ((1ull << k) < b) ++k;
    return k;
}

GpuLWEtoRGSWConverter::GpuLWEtoRGSWConverter(const tp_br_params& rotation, uint64_t trace_basis,
                                             uint32_t trace_digits, uint64_t square_basis, uint32_t square_digits,
                                             uint32_t out_digits, uint64_t out_basis, const std::vector<uint64_t>& brk,
                                             const std::vector<uint64_t>& trace_keys,
                                             const std::vector<uint64_t>& square_key, int device)
    : m_N(rotation.ring_dim), m_n(rotation.lwe_dim), m_D(out_digits) {
    check(tp_ss_create(&rotation, trace_basis, trace_digits, square_basis, square_digits, out_digits, out_basis,
                       device, &m_ctx));
    tp_status s = tp_ss_upload_keys(m_ctx, brk.data(), brk.size(), trace_keys.data(), trace_keys.size(),
                                    square_key.data(), square_key.size());
    if (s != TP_OK) {
        tp_ss_destroy(m_ctx);
        check(s);
    }
}
GpuLWEtoRGSWConverter::~GpuLWEtoRGSWConverter() { tp_ss_destroy(m_ctx); }

void GpuLWEtoRGSWConverter::ConvertBatch(uint64_t batch, uint64_t* outputs, const uint64_t* lwes) {
    if (batch == 0) return;
    DevBuf din(batch * (m_n + 1ull)), dout(batch * OutputWords());
    if (cudaMemcpy(din.p, lwes, batch * (m_n + 1ull) * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_lwe_to_rgsw_batch(m_ctx, batch, dout.p, din.p, nullptr));
    if (cudaMemcpy(outputs, dout.p, batch * OutputWords() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuLWEtoRGSWConverter::Convert(uint64_t* output, const uint64_t* input) { ConvertBatch(1, output, input); }

void GpuLWEtoRGSWConverter::Convert(std::vector<uint64_t>& output, const std::vector<uint64_t>& input) {
    output.resize(OutputWords());
    ConvertBatch(1, output.data(), input.data());
}

SchemeSwitchingContext::SchemeSwitchingContext(const tp_br_params& rotation, uint64_t trace_basis,
                                               uint64_t trace_digits, uint64_t square_basis, uint64_t square_digits,
                                               uint64_t output_digits, uint64_t output_basis, double std_dev,
                                               int device, uint64_t seed)
    : m_rot(rotation), m_tr_basis(trace_basis), m_tr_digits(trace_digits), m_sq_basis(square_basis),
      m_sq_digits(square_digits), m_out_digits(output_digits), m_out_basis(output_basis), m_std(std_dev),
      m_device(device), m_seed(seed) {
    if (rotation.modulus != kGoldilocks)
        throw std::invalid_argument("toothpaste_b200: modulus must be 2^64 - 2^32 + 1");
    for (uint64_t b : {rotation.basis, trace_basis, square_basis, output_basis})
        if (b < 2 || (b & (b - 1))) throw std::invalid_argument("toothpaste_b200: gadget bases must be powers of two");
}

std::unique_ptr<GpuLWEtoRGSWConverter> SchemeSwitchingContext::ConstructOperator(
    const std::vector<std::vector<uint64_t>>& keys) const {
    if (keys.size() < 2 || keys[0].size() < m_rot.lwe_dim || keys[1].size() < m_rot.ring_dim)
        throw std::invalid_argument("toothpaste_b200: keys = {LWE key (n), RLWE key (N)}");
    Sampler rng(m_seed);
    auto k = keygen::SchemeSwitchingKeys(rng, m_rot.variant, m_rot.ring_dim, m_rot.lwe_dim, log2_of(m_rot.basis),
                                         m_rot.digits, log2_of(m_tr_basis), (uint32_t)m_tr_digits,
                                         log2_of(m_sq_basis), (uint32_t)m_sq_digits, m_std, keys[0], keys[1]);
    return std::make_unique<GpuLWEtoRGSWConverter>(m_rot, m_tr_basis, (uint32_t)m_tr_digits, m_sq_basis,
                                                   (uint32_t)m_sq_digits, (uint32_t)m_out_digits, m_out_basis,
                                                   k.rotation, k.trace, k.square, m_device);
}

// ---- SAP decomposition ----

GpuSAPDecomposer::GpuSAPDecomposer(const tp_br_params& rotation, uint64_t trace_basis, uint32_t trace_digits,
                                   uint64_t ks_basis, uint32_t ks_digits, const std::vector<uint64_t>& brk,
                                   const std::vector<uint64_t>& trace_keys, const std::vector<uint64_t>& lwe_ksk,
                                   uint64_t hamming_weight, uint64_t restart_period, uint64_t max_digits, int device)
    : m_N(rotation.ring_dim), m_n(rotation.lwe_dim), m_beta(hamming_weight), m_restart(restart_period),
      m_max_digits(max_digits) {
    check(tp_sap_create(&rotation, trace_basis, trace_digits, ks_basis, ks_digits, device, &m_ctx));
    tp_status s = tp_sap_upload_keys(m_ctx, brk.data(), brk.size(), trace_keys.data(), trace_keys.size(),
                                     lwe_ksk.data(), lwe_ksk.size());
    if (s != TP_OK) {
        tp_sap_destroy(m_ctx);
        check(s);
    }
}
GpuSAPDecomposer::~GpuSAPDecomposer() { tp_sap_destroy(m_ctx); }

std::vector<uint32_t> GpuSAPDecomposer::DecomposeBatch(uint64_t batch, uint64_t* outputs, uint64_t out_digits,
                                                       const uint64_t* lwes, uint64_t radix) {
    std::vector<uint32_t> digits(batch, 0);
    if (batch == 0) return digits;
    const uint64_t in_words = batch * (m_n + 1ull), out_words = batch * out_digits * (m_N + 1ull);
    DevBuf din(in_words), dout(out_words);
    if (cudaMemcpy(din.p, lwes, in_words * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dout.p, outputs, out_words * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_sap_decompose_batch(m_ctx, batch, dout.p, out_digits, din.p, radix, m_beta, m_restart, digits.data(),
                                 nullptr));
    if (cudaMemcpy(outputs, dout.p, out_words * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
    return digits;
}

void GpuSAPDecomposer::HomTrunc(uint64_t* output, uint64_t* input, uint64_t radix) {
    DevBuf din(2ull * m_N), dout(2ull * m_N);
    if (cudaMemcpy(din.p, input, 2ull * m_N * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_sap_homtrunc_batch(m_ctx, 1, dout.p, din.p, radix, nullptr));
    if (cudaMemcpy(output, dout.p, 2ull * m_N * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuSAPDecomposer::ResetAccumulator(uint64_t* acc, uint64_t radix) {
    DevBuf d(2ull * m_N);
    if (cudaMemcpy(d.p, acc, 2ull * m_N * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy in failed");
    check(tp_sap_reset_batch(m_ctx, 1, d.p, radix, nullptr));
    if (cudaMemcpy(acc, d.p, 2ull * m_N * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("toothpaste_b200: copy back failed");
}

void GpuSAPDecomposer::Decompose(uint64_t* output, const uint64_t* input, uint64_t radix) {
    // the output holds as many digits as the input implies; stage through a buffer of the
    // context's maximum and copy those back
    std::vector<uint64_t> buf(m_max_digits * (m_N + 1ull), 0);
    const auto d = DecomposeBatch(1, buf.data(), m_max_digits, input, radix);
    std::copy(buf.begin(), buf.begin() + d[0] * (m_N + 1ull), output);
}

void GpuSAPDecomposer::Decompose(std::vector<uint64_t>& output, const std::vector<uint64_t>& input, uint64_t radix) {
    std::vector<uint64_t> buf(m_max_digits * (m_N + 1ull), 0);
    const auto d = DecomposeBatch(1, buf.data(), m_max_digits, input.data(), radix);
    if (output.size() < d[0] * (m_N + 1ull)) output.resize(d[0] * (m_N + 1ull));
    std::copy(buf.begin(), buf.begin() + d[0] * (m_N + 1ull), output.begin());
}

SAPDecompositionContext::SAPDecompositionContext(const tp_br_params& rotation, uint64_t trace_basis,
                                                 uint64_t trace_digits, uint64_t ks_basis, uint64_t ks_digits,
                                                 uint64_t default_radix, double std_dev, uint64_t restart_period,
                                                 int device, uint64_t seed)
    : m_rot(rotation), m_tr_basis(trace_basis), m_tr_digits(trace_digits), m_ks_basis(ks_basis),
      m_ks_digits(ks_digits), m_radix(default_radix), m_std(std_dev), m_restart(restart_period), m_device(device),
      m_seed(seed) {
    if (rotation.modulus != kGoldilocks)
        throw std::invalid_argument("toothpaste_b200: modulus must be 2^64 - 2^32 + 1");
    for (uint64_t b : {rotation.basis, trace_basis, ks_basis, default_radix})
        if (b < 2 || (b & (b - 1))) throw std::invalid_argument("toothpaste_b200: bases and radix must be powers of two");
    if (restart_period == 0) throw std::invalid_argument("toothpaste_b200: restart period must be positive");
}

std::unique_ptr<GpuSAPDecomposer> SAPDecompositionContext::ConstructOperator(
    const std::vector<std::vector<uint64_t>>& keys) const {
    if (keys.size() < 2 || keys[0].size() < m_rot.lwe_dim || keys[1].size() < m_rot.ring_dim)
        throw std::invalid_argument("toothpaste_b200: keys = {LWE key (n), RLWE key (N)}");
    uint64_t weight = 0;
    for (uint32_t i = 0; i < m_rot.lwe_dim; ++i) weight += keys[0][i] != 0;
    Sampler rng(m_seed);
    auto k = keygen::SAPKeys(rng, m_rot.variant, m_rot.ring_dim, m_rot.lwe_dim, log2_of(m_rot.basis), m_rot.digits,
                             log2_of(m_tr_basis), (uint32_t)m_tr_digits, log2_of(m_ks_basis), (uint32_t)m_ks_digits,
                             m_std, keys[0], keys[1]);
    return std::make_unique<GpuSAPDecomposer>(m_rot, m_tr_basis, (uint32_t)m_tr_digits, m_ks_basis,
                                              (uint32_t)m_ks_digits, k.rotation, k.trace, k.lwe_switch, weight,
                                              m_restart, 64, m_device);
}

}  // namespace toothpaste_b200
