/*
 * CPU oracle for the Toothpaste blind-rotation hot path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of the reference library's algorithms over the
 * Goldilocks prime p = 2^64 - 2^32 + 1. It exists only to check the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and never as the thing that is measured or shipped.
 *
 * Parity pins: every routine is checked against the reference itself, compiled
 * from its own sources by oracle/Makefile into oracle/_ref/, through the golden
 * fixtures under tests/golden/ (generated by tests/golden/make_golden.py).
 *
 * Each function cites the reference file:line it restates (paths relative to
 * the reference project root).
 */
#ifndef TP_ORACLE_H
#define TP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TPO_P 0xFFFFFFFF00000001ULL

/* ---- seeded sampler (project-defined stand-in for the OpenFHE samplers) ----
 * Stream: splitmix64. uniform(q): rejection sampling on the smallest all-ones
 * mask >= q-1. gaussian(std, q): Box-Muller (first output only), rounded to the
 * nearest integer (ties away from zero), returned mod q; std == 0 gives 0 and
 * draws nothing. The oracle/shim/openfhe.h shim draws in exactly the same way,
 * so a reference build seeded identically produces identical keys. */
typedef struct { uint64_t s; } tpo_rng;
void tpo_rng_seed(tpo_rng* r, uint64_t seed);
uint64_t tpo_next64(tpo_rng* r);
uint64_t tpo_uniform(tpo_rng* r, uint64_t q);
uint64_t tpo_gaussian(tpo_rng* r, double std_dev, uint64_t q);

/* ---- Goldilocks scalar arithmetic (lib/include/backend/solinas_internal.h:39-113) */
uint64_t tpo_add(uint64_t a, uint64_t b);
uint64_t tpo_sub(uint64_t a, uint64_t b);
uint64_t tpo_mul(uint64_t a, uint64_t b);
uint64_t tpo_pow(uint64_t b, uint64_t e);
uint64_t tpo_inv(uint64_t a);

/* ---- negacyclic NTT (lib/src/backend/solinas.cpp:168-313) ----
 * Forward: natural-order coefficients -> evaluations in bit-reversed order,
 * out[k] = a(psi^(2*brv(k)+1)), psi = 7^((p-1)/2N). Backward includes 1/N.
 * In-place allowed. Returns 0, or -1 for an unsupported N. */
int tpo_ntt_forward(uint64_t N, uint64_t* out, const uint64_t* in);
int tpo_ntt_backward(uint64_t N, uint64_t* out, const uint64_t* in);
uint64_t tpo_psi(uint64_t N);

/* ---- gadget decomposition, coefficient domain (lib/include/static/gadget_decomp.h) ----
 * out is digits x N, digit-major. Signed: :16-28 + :156-205. Unsigned (the
 * binary-CGGI rule of lib/src/operators/mux_operator.cpp:24-26,46-69). */
void tpo_signed_digits(uint64_t* out, const uint64_t* in, uint64_t N, uint64_t digits, uint64_t basis_log2);
void tpo_unsigned_digits(uint64_t* out, const uint64_t* in, uint64_t N, uint64_t digits, uint64_t basis_log2);

/* ---- encryption / key generation (lib/src/base_crypto.cpp:27-97,137-155) ---- */
void tpo_make_rlwe(tpo_rng* r, uint64_t N, double std_dev, uint64_t* out, const uint64_t* msg,
                   const uint64_t* sk_ntt, int msg_is_ntt);
void tpo_make_rgsw(tpo_rng* r, uint64_t N, double std_dev, uint64_t* out, const uint64_t* msg,
                   const uint64_t* sk_ntt, uint64_t basis, uint64_t digits, int msg_is_ntt);
void tpo_phase_rlwe(uint64_t N, uint64_t* out, const uint64_t* rlwe, const uint64_t* sk_ntt);

enum { TPO_CGGI_BINARY = 0, TPO_CGGI_TERNARY = 1, TPO_BMMP_BINARY = 2 };

/* Words of the blind-rotation key in the reference layout (m_brk). */
uint64_t tpo_brk_words(int variant, uint64_t N, uint64_t n, uint64_t digits);

/* CGGI KeyGenBinary / KeyGenTernary (lib/src/operators/cggi_blind_rotation.cpp:264-311)
 * and BMMP KeyGenBinary (lib/src/operators/bmmp_blind_rotation.cpp:229-262). */
void tpo_br_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                   double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk);
void tpo_br_keygen_aligned(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                           double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk);

/* BlindRotate: CGGI (cggi_blind_rotation.cpp:236-262, 313-472) and BMMP
 * (bmmp_blind_rotation.cpp:325-335, 280-323, 354-419; MultiMux mux_operator.cpp:204-294).
 * result may equal acc. Returns 0, or -1 on bad parameters. */
int tpo_blind_rotate(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                     const uint64_t* brk, uint64_t* result, const uint64_t* lwe, const uint64_t* acc,
                     int out_coef);

/* Same, for `count` independent rotations on `threads` POSIX threads
 * (lwe stride n+1, acc/result stride 2N). Used as the CPU baseline. */
int tpo_blind_rotate_many(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                          const uint64_t* brk, uint64_t* results, const uint64_t* lwes,
                          const uint64_t* accs, uint64_t count, int out_coef, int threads);

/* ---- key switching (lib/src/operators/rlwe_conversion.cpp:187-249,
 *      lib/src/operators/lwe_conversion.cpp:174-239) ---- */
void tpo_rlwe_ks_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                        const uint64_t* source_key, const uint64_t* target_key, uint64_t* ksk);
/* out -= sum_j NTT(d_j(in.A)) * ksk_j ; out.B += in.B. in = [A coef | B ntt]. */
void tpo_rlwe_ks(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* ksk,
                 uint64_t* out, const uint64_t* in);
void tpo_lwe_ks_keygen(tpo_rng* r, uint64_t q, uint64_t n_in, uint64_t n_out, uint64_t basis_log2,
                       uint64_t digits, double std_dev, const uint64_t* source_key,
                       const uint64_t* target_key, uint64_t* ksk);
void tpo_lwe_ks(uint64_t q, uint64_t n_in, uint64_t n_out, uint64_t basis_log2, uint64_t digits,
                const uint64_t* ksk, uint64_t* out, const uint64_t* in);
void tpo_make_lwe(tpo_rng* r, uint64_t q, uint64_t n, double std_dev, uint64_t* out, uint64_t msg,
                  const uint64_t* secret);

/* ---- automorphisms and packing (lib/src/utils/math_utils.cpp:70-85,
 *      lib/src/operators/automorphism_evaluation.cpp:43-63,150-206,
 *      lib/src/operators/lwe_to_rlwe_packing.cpp:46-58,129-251) ---- */
void tpo_negacyclic_automorphism(uint64_t* out, const uint64_t* in, uint64_t index, uint64_t N);
void tpo_auto_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                     uint64_t index, const uint64_t* rlwe_key, uint64_t* ksk);
/* out (NTT domain) = KS(aut_index(in)); in is [A coef | B coef]. out must be pre-zeroed. */
void tpo_auto_eval(uint64_t N, uint64_t basis_log2, uint64_t digits, uint64_t index,
                   const uint64_t* ksk, uint64_t* out, const uint64_t* in);
/* Keys for indices 2^j+1, j = 1..logN, each 2*N*digits words, concatenated. */
void tpo_pack_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                     const uint64_t* rlwe_key, uint64_t* keys);
/* Pack len LWEs (each N+1 words) into one RLWE [A|B] coefficient domain. */
int tpo_pack(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys,
             uint64_t* out, const uint64_t* in, uint64_t len);

/* PackConsecutively (lwe_to_rlwe_packing.cpp:260-393): len LWEs (2 <= len <= N) into the
 * first len coefficients of one RLWE [A|B] (coefficient domain), by the reference's stack
 * walk over a full N-leaf tree whose leaves without an input are zero and whose merges of
 * two such leaves are skipped. */
int tpo_pack_consecutive(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys,
                         uint64_t* out, const uint64_t* in, uint64_t len);

/* SampleExtract (lib/include/static/sample_extraction.h:20-36): writes nothing
 * where the source coefficient is zero (the caller pre-zeroes). */
void tpo_sample_extract(uint64_t* out_lwe, const uint64_t* rlwe, uint64_t index, uint64_t N);

/* ModulusSwitch (lib/src/static/modulus_switching.cpp:36-93), types 0 ROUND,
 * 1 FLOOR, 2 CEIL, in 80-bit long double like the reference; in place. */
int tpo_modulus_switch(uint64_t* vec, uint64_t n, uint64_t source, uint64_t target, int type);

/* ---- LWE -> RGSW scheme switching (lib/src/operators/lwe_to_rgsw_conversion.cpp) ---- */
/* The converter's accumulator m_acc = [0 | -tp | tp] (3N words; lines 120-160).
 * Returns -1 where the reference's first scale (an int shift) would overflow
 * or out_digits does not split N into even blocks. */
int tpo_ss_test_poly(uint64_t N, uint64_t out_digits, uint64_t out_basis_log2, uint64_t* acc);
/* TraceEvaluator::Eval (trace_evaluation.cpp:135-158): out = NTT of both halves of the
 * key-switched N^-1 Tr(in); in = [A | B] coefficients; keys for indices 2^j + 1. */
void tpo_trace_eval(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys, uint64_t* out,
                    const uint64_t* in);
/* Convert (lines 168-225) of one LWE (n+1 words mod 2N) into 4 N out_digits
 * words [lev_left | lev_right], NTT domain. trace_keys: automorphism keys for
 * indices 2^j + 1, j = 1..logN, concatenated; sq_key: RLWE key switch s^2 -> s. */
/* SchemeSwitchingContext::ConstructOperator (lwe_to_rgsw_conversion.cpp:72-108)
 * from one sampler stream: the rotation key, the trace's automorphism keys
 * (indices 3, 5, .., N+1), then the key switch from s^2 = INTT(NTT(s)^2) to s. */
void tpo_ss_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                   uint64_t tr_basis_log2, uint64_t tr_digits, uint64_t sq_basis_log2, uint64_t sq_digits,
                   double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk,
                   uint64_t* trace_keys, uint64_t* sq_key);
int tpo_lwe_to_rgsw(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                    const uint64_t* brk, uint64_t tr_basis_log2, uint64_t tr_digits, const uint64_t* trace_keys,
                    uint64_t sq_basis_log2, uint64_t sq_digits, const uint64_t* sq_key, uint64_t out_digits,
                    uint64_t out_basis_log2, const uint64_t* lwe, uint64_t* out);

/* ---- SAP digit decomposition (lib/src/operators/sap_decomposer.cpp) ---- */
/* The reference's IntLog2 (math_utils.cpp:11-25): ceil(log2 x), 0 for x <= 1. */
uint64_t tpo_ref_int_log2(uint64_t x);
/* SAPDecompositionContext::ConstructOperator (lines 166-186) from one sampler
 * stream: the rotation key, the trace's automorphism keys (indices 3, 5, .., N+1),
 * then the LWE key switch from the RLWE key's coefficients (N) to the LWE key (n). */
void tpo_sap_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                    uint64_t tr_basis_log2, uint64_t tr_digits, uint64_t ks_basis_log2, uint64_t ks_digits,
                    double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk,
                    uint64_t* trace_keys, uint64_t* lwe_ksk);
/* HomTrunc (lines 189-291): out (2N, NTT domain) from in (2N, NTT domain); trace_keys
 * for indices 2^j + 1, j = 1..logN. */
int tpo_sap_homtrunc(uint64_t N, uint64_t tr_basis_log2, uint64_t tr_digits, const uint64_t* trace_keys,
                     uint64_t radix, uint64_t* out, const uint64_t* in);
/* ResetAccumulator (lines 293-351) on acc (2N, NTT domain, in place), with the LWE key
 * switch N -> n of a fresh converter (its accumulator cleared). */
int tpo_sap_reset(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                  const uint64_t* brk, uint64_t ks_basis_log2, uint64_t ks_digits, const uint64_t* lwe_ksk,
                  uint64_t radix, uint64_t* acc);
/* Decompose (lines 353-464): digits of `in` (n+1 words) written to out + d (N+1) (only
 * nonzero words, the caller zeroes out), at most out_digits; returns the digit count,
 * or -1 on bad parameters / too small an output. */
int tpo_sap_decompose(int variant, uint64_t N, uint64_t n, uint64_t br_basis_log2, uint64_t br_digits,
                      const uint64_t* brk, uint64_t tr_basis_log2, uint64_t tr_digits, const uint64_t* trace_keys,
                      uint64_t ks_basis_log2, uint64_t ks_digits, const uint64_t* lwe_ksk, uint64_t radix,
                      uint64_t beta, uint64_t restart, const uint64_t* in, uint64_t* out, uint64_t out_digits);

#ifdef __cplusplus
}
#endif

#endif
