// Build shim for compiling the reference library as a test oracle (TEST INFRASTRUCTURE).
//
// Intel HEXL is an unvendored, unpinned dependency of the reference
// (install_dependencies.sh clones github.com/intel/hexl at HEAD). Only the
// scalar and element-wise helpers below are reached on the Goldilocks path.
// This header restates their documented contract — canonical results mod q for
// canonical inputs — with 128-bit integer arithmetic. HEXL's own vectorised
// kernels are specified for moduli below 2^62..2^63; on Goldilocks this shim
// gives the mathematically defined value. hexl::NTT exists only so that the
// generic-modulus backend compiles; it is never reached for Goldilocks.
#ifndef TP_SHIM_HEXL_HPP
#define TP_SHIM_HEXL_HPP

#include <cstddef>
#include <cstdint>
#include <stdexcept>

namespace intel {
namespace hexl {

using u128 = unsigned __int128;

inline uint64_t AddUIntMod(uint64_t x, uint64_t y, uint64_t q) { return (uint64_t)(((u128)x + y) % q); }
inline uint64_t SubUIntMod(uint64_t x, uint64_t y, uint64_t q) {
    return x >= y ? x - y : (uint64_t)((u128)x + q - y);
}
inline uint64_t MultiplyMod(uint64_t x, uint64_t y, uint64_t q) { return (uint64_t)(((u128)x * y) % q); }
inline uint64_t MultiplyMod(uint64_t x, uint64_t y, uint64_t /*barrett*/, uint64_t q) { return MultiplyMod(x, y, q); }
inline uint64_t PowMod(uint64_t b, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    b %= q;
    while (e) {
        if (e & 1) r = MultiplyMod(r, b, q);
        b = MultiplyMod(b, b, q);
        e >>= 1;
    }
    return r;
}
// q prime in every use; inverse by Fermat.
inline uint64_t InverseMod(uint64_t x, uint64_t q) { return x % q == 0 ? 0 : PowMod(x, q - 2, q); }

class MultiplyFactor {
public:
    MultiplyFactor(uint64_t operand, uint64_t bit_shift, uint64_t q)
        : m_factor(bit_shift >= 64 ? 0 : (uint64_t)(((u128)operand << bit_shift) / q)) {}
    uint64_t BarrettFactor() const { return m_factor; }
private:
    uint64_t m_factor;
};

inline void EltwiseAddMod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q) {
    for (uint64_t i = 0; i < n; ++i) r[i] = AddUIntMod(a[i], b[i], q);
}
inline void EltwiseAddMod(uint64_t* r, const uint64_t* a, uint64_t s, uint64_t n, uint64_t q) {
    for (uint64_t i = 0; i < n; ++i) r[i] = AddUIntMod(a[i], s, q);
}
inline void EltwiseSubMod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q) {
    for (uint64_t i = 0; i < n; ++i) r[i] = SubUIntMod(a[i], b[i], q);
}
inline void EltwiseSubMod(uint64_t* r, const uint64_t* a, uint64_t s, uint64_t n, uint64_t q) {
    for (uint64_t i = 0; i < n; ++i) r[i] = SubUIntMod(a[i], s, q);
}
inline void EltwiseMultMod(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t n, uint64_t q,
                           uint64_t /*input_mod_factor*/) {
    for (uint64_t i = 0; i < n; ++i) r[i] = MultiplyMod(a[i], b[i], q);
}
// r = a * s (+ c), c may be nullptr.
inline void EltwiseFMAMod(uint64_t* r, const uint64_t* a, uint64_t s, const uint64_t* c, uint64_t n,
                          uint64_t q, uint64_t /*input_mod_factor*/) {
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t p = MultiplyMod(a[i], s % q, q);
        r[i] = c ? AddUIntMod(p, c[i], q) : p;
    }
}
inline void EltwiseReduceMod(uint64_t* r, const uint64_t* a, uint64_t n, uint64_t q, uint64_t /*in*/,
                             uint64_t /*out*/) {
    for (uint64_t i = 0; i < n; ++i) r[i] = a[i] % q;
}

class NTT {
public:
    NTT() = default;
    NTT(uint64_t degree, uint64_t q) : m_degree(degree), m_q(q) {}
    void ComputeForward(uint64_t*, const uint64_t*, uint64_t, uint64_t) {
        throw std::logic_error("hexl shim: generic-modulus NTT is outside the oracle's scope");
    }
    void ComputeInverse(uint64_t*, const uint64_t*, uint64_t, uint64_t) {
        throw std::logic_error("hexl shim: generic-modulus NTT is outside the oracle's scope");
    }
private:
    uint64_t m_degree = 0, m_q = 0;
};

}  // namespace hexl
}  // namespace intel

#endif
