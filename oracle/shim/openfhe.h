// Build shim for compiling the reference library as a test oracle (TEST INFRASTRUCTURE).
//
// OpenFHE (unvendored, cloned at HEAD by install_dependencies.sh) provides only
// the two samplers used for key and noise generation (lib/src/base_crypto.cpp:34-39,
// 139-142); the reference never seeds them. This shim substitutes one seeded,
// process-global stream with the draw rules of oracle/tp_oracle.c (splitmix64;
// uniform by masked rejection; Gaussian by Box-Muller rounded to nearest), so a
// seeded reference build and the C oracle produce the same keys.
#ifndef TP_SHIM_OPENFHE_H
#define TP_SHIM_OPENFHE_H

#include <cmath>
#include <cstdint>
#include <vector>

namespace tp_shim {
inline uint64_t& state() {
    static uint64_t s = 0;
    return s;
}
inline void seed(uint64_t v) { state() = v; }
inline uint64_t next64() {
    uint64_t z = (state() += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
inline uint64_t uniform(uint64_t q) {
    if (q == 0) return next64();
    uint64_t mask = q - 1;
    mask |= mask >> 1; mask |= mask >> 2; mask |= mask >> 4;
    mask |= mask >> 8; mask |= mask >> 16; mask |= mask >> 32;
    for (;;) {
        const uint64_t x = next64() & mask;
        if (x < q) return x;
    }
}
inline uint64_t gaussian(double std_dev, uint64_t q) {
    if (std_dev == 0.0) return 0;
    const double u1 = (double)((next64() >> 11) + 1) * 0x1.0p-53;
    const double u2 = (double)(next64() >> 11) * 0x1.0p-53;
    const double rad = std::sqrt(-2.0 * std::log(u1));
    const double ang = 6.283185307179586 * u2;
    const double z = rad * std::cos(ang);
    const long long k = std::llround(z * std_dev);
    if (k >= 0) return (uint64_t)k % q;
    const uint64_t m = (uint64_t)(-k) % q;
    return m == 0 ? 0 : q - m;
}
}  // namespace tp_shim

struct NativeInteger {
    uint64_t v = 0;
    template <typename T>
    T ConvertToInt() const { return (T)v; }
};
using NativeVector = std::vector<NativeInteger>;

namespace lbcrypto {
template <typename VecType>
class DiscreteUniformGeneratorImpl {
public:
    explicit DiscreteUniformGeneratorImpl(uint64_t q) : m_q(q) {}
    VecType GenerateVector(uint64_t n) const {
        VecType v(n);
        for (auto& x : v) x.v = tp_shim::uniform(m_q);
        return v;
    }
private:
    uint64_t m_q;
};

template <typename VecType>
class DiscreteGaussianGeneratorImpl {
public:
    explicit DiscreteGaussianGeneratorImpl(double std_dev) : m_std(std_dev) {}
    VecType GenerateVector(uint64_t n, uint64_t q) const {
        VecType v(n);
        for (auto& x : v) x.v = tp_shim::gaussian(m_std, q);
        return v;
    }
    NativeInteger GenerateInteger(uint64_t q) const { return NativeInteger{tp_shim::gaussian(m_std, q)}; }
private:
    double m_std;
};
}  // namespace lbcrypto

#endif
