/*
 * toothpaste_gpu.h — C ABI of the B200 (sm_100a) blind-rotation engine.
 *
 * Plain C types only: device and host buffers are uint64_t pointers, streams are
 * passed as `void*` (a cudaStream_t, NULL = the legacy default stream). Every
 * entry point returns a tp_status; tp_last_error() gives a message for the
 * calling thread. No exception crosses this boundary.
 *
 * Arithmetic is over the Goldilocks prime p = 2^64 - 2^32 + 1. All ciphertext
 * words are canonical residues in [0, p); polynomials have N coefficients with
 * N a power of two in [128, 65536]; above 4096 one rotation, key switch or
 * transform runs on a cluster of CTAs that exchange through distributed shared
 * memory: 2, 4, 8 and 16 CTAs of 4096 coefficients at N = 8192, 16384, 32768 and
 * 65536. "NTT domain" means the reference's
 * evaluation order: slot k holds a(psi^(2*brv(k)+1)), psi = 7^((p-1)/2N)
 * (lib/src/backend/solinas.cpp:168-313 of the reference).
 *
 * Each declaration names the reference interface it replaces (file:line in the
 * reference project).
 */
#ifndef TOOTHPASTE_GPU_H
#define TOOTHPASTE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TP_OK = 0,
    TP_ERR_PARAM = 1,   /* invalid argument or unsupported parameter set */
    TP_ERR_OOM = 2,     /* device allocation failed */
    TP_ERR_CUDA = 3,    /* a CUDA call failed (message in tp_last_error) */
    TP_ERR_TIMEOUT = 4, /* a bounded host-side wait ran out (serving: a result or a drain) */
    TP_ERR_LAYOUT = 5,  /* key size or layout does not match the context */
    TP_ERR_STATE = 6    /* call order: e.g. rotate before a key was uploaded */
} tp_status;

/* Blind-rotation variants (reference: KeyDistribution BINARY/TERNARY for
 * CGGIBlindRotationContext, lib/include/operators/cggi_blind_rotation.h:24;
 * BMMPBlindRotationContext with step_size 2, lib/include/operators/bmmp_blind_rotation.h:23). */
typedef enum {
    TP_BR_CGGI_BINARY = 0,
    TP_BR_CGGI_TERNARY = 1,
    TP_BR_BMMP_BINARY = 2
} tp_br_variant;

/* Parameters of CGGIBlindRotationContext(distr, modulus, ring_dim, lwe_dim,
 * basis, digits, std) (lib/src/operators/cggi_blind_rotation.cpp:14-25). `std`
 * only matters for key generation, which stays on the host. */
typedef struct {
    int32_t variant;     /* tp_br_variant */
    uint64_t modulus;    /* must be 0xFFFFFFFF00000001 */
    uint32_t ring_dim;   /* N */
    uint32_t lwe_dim;    /* n (even for BMMP) */
    uint64_t basis;      /* gadget base, a power of two 2^beta, beta in [1, 30] */
    uint32_t digits;     /* l, 1..8 */
} tp_br_params;

typedef struct tp_br_ctx tp_br_ctx;

/* Creates a context on `device` (its tables are built there). Replaces the
 * operator construction of CGGIBlindRotationContext::ConstructOperator
 * (lib/src/operators/cggi_blind_rotation.cpp:184-199) minus key generation. */
tp_status tp_br_create(const tp_br_params* params, int device, tp_br_ctx** out);
tp_status tp_br_destroy(tp_br_ctx* ctx);

/* Number of uint64 words of the blind-rotation key in the reference layout
 * (the m_brk of KeyGenBinary/KeyGenTernary, cggi_blind_rotation.cpp:264-311,
 * or BMMP KeyGenBinary, bmmp_blind_rotation.cpp:229-262). */
uint64_t tp_br_key_words(const tp_br_ctx* ctx);

/* Uploads a key in that reference layout from host memory (`words` must equal
 * tp_br_key_words) and re-lays it out on the device. Synchronous. */
tp_status tp_br_upload_key(tp_br_ctx* ctx, const uint64_t* brk_host, uint64_t words);

/* Drop-in for BlindRotator::BlindRotate(result, lwe, acc, output_as_coefficients)
 * (lib/include/interfaces/blindrotation_operator.h:39-40; CGGI body
 * cggi_blind_rotation.cpp:236-262, BMMP body bmmp_blind_rotation.cpp:325-335).
 * Host pointers: lwe has n+1 words [a_0..a_{n-1}, b], each in [0, 2N); acc is
 * 2N words [A | B] in the coefficient domain; result receives 2N words in the
 * NTT domain, or coefficients when out_coef != 0. result may equal acc.
 * Synchronous; one rotation per launch (the plain form). */
tp_status tp_br_blind_rotate(tp_br_ctx* ctx, uint64_t* result, const uint64_t* lwe, const uint64_t* acc,
                             int out_coef);

/* Batched form of the same call on device buffers: rotation b reads
 * lwes + b*lwe_stride and accs + b*acc_stride (acc_stride 0 = one accumulator
 * shared by the whole batch) and writes results + b*2N. Asynchronous on
 * `stream`; runs as one persistent launch whose accumulators stay on chip for
 * all n iterations. Inputs outside [0, 2N) are reduced mod 2N and flagged;
 * tp_br_check flags them. No reference counterpart (the reference rotates
 * one ciphertext per call). */
tp_status tp_br_blind_rotate_batch(tp_br_ctx* ctx, uint64_t batch, uint64_t* results_dev,
                                   const uint64_t* lwes_dev, uint64_t lwe_stride, const uint64_t* accs_dev,
                                   uint64_t acc_stride, int out_coef, void* stream);

/* The batched call on host buffers: copies in, rotates, copies out, waits. */
tp_status tp_br_blind_rotate_batch_host(tp_br_ctx* ctx, uint64_t batch, uint64_t* results,
                                        const uint64_t* lwes, uint64_t lwe_stride, const uint64_t* accs,
                                        uint64_t acc_stride, int out_coef, void* stream);

/* Tile of the rotation kernel: coefficients per thread (8: N/8 threads per
 * rotation with radix-8 NTT passes; 4: N/4 threads, radix-4 passes, fewer
 * registers per thread so more warps per SM). Changing it after the key is
 * uploaded re-lays the key out on the device (twice the key's memory while it
 * runs). Not thread-safe against concurrent launches on the same context. No
 * reference counterpart (tiling is a property of the GPU kernel). */
tp_status tp_br_set_tile(tp_br_ctx* ctx, uint32_t coef_per_thread);
uint32_t tp_br_get_tile(const tp_br_ctx* ctx);

/* Thread blocks per rotation: 1 (default), 2 or 4. With 2, a cluster of two
 * blocks on two SMs rotates each ciphertext, each block owning one accumulator
 * half and its gadget rows and exchanging partial sums with the other through
 * distributed shared memory: about half the latency per rotation, for batches
 * smaller than the number of SMs (large batches run faster with 1). With 4, two
 * blocks per half split that half's gadget digits between them and combine
 * their sums in a second exchange (for batches up to a quarter of the SMs).
 * Needs the tile of 4 coefficients per thread; TP_ERR_PARAM if the parameter
 * set does not fit the chosen kernel on this device (the four-block kernel
 * needs (2 + 2G) N + 1024 words of shared memory with one NTT exchange buffer,
 * G = RGSWs per iteration: not for BMMP at N = 4096). Same output words either
 * way. No reference counterpart. */
tp_status tp_br_set_split(tp_br_ctx* ctx, uint32_t blocks_per_rotation);
uint32_t tp_br_get_split(const tp_br_ctx* ctx);

/* Multiply-accumulate form of the one-block kernel at 4 coefficients per thread.
 * TP_MAC_ROWWISE keeps a canonical running sum per output word, one gadget row at
 * a time (the next key row staged in shared memory while the digit is transformed);
 * TP_MAC_DIGIT_STAGED transforms all 2l digits first and sums each output word over
 * the 2l rows exactly before one reduction (digits 3 or 4, N <= 2048, one CTA per
 * rotation, where shared memory allows; the default there). Both give the same words. Project-specific tuning (no
 * reference counterpart); tp_br_autotune chooses between them. */
enum { TP_MAC_ROWWISE = 0, TP_MAC_DIGIT_STAGED = 1 };
tp_status tp_br_set_mac_form(tp_br_ctx* ctx, uint32_t form);
uint32_t tp_br_get_mac_form(const tp_br_ctx* ctx);

/* NTT passes of the one-block kernel at 4 coefficients per thread: radix 2
 * (butterflies, the default) or 4 (fused radix-4 passes: three products and a
 * power-of-two shift per two levels). Built for N = 1024 .. 4096; same words
 * either way. Project-specific tuning (no reference counterpart); tp_br_autotune
 * chooses it with the other launch settings. */
tp_status tp_br_set_radix(tp_br_ctx* ctx, uint32_t radix);
uint32_t tp_br_get_radix(const tp_br_ctx* ctx);

/* Times every launch form (8 or 4 coefficients per thread; at 4 also the
 * digit-staged multiply-accumulate, the fused radix-4 passes and two or four
 * blocks per rotation) on up to two waves of `batch` synthetic rotations with the
 * uploaded key, keeps the fastest and reports it (either output may be NULL; the
 * split, form and radix are read back with tp_br_get_split / tp_br_get_mac_form /
 * tp_br_get_radix). Blocks until done; the context must be idle. */
tp_status tp_br_autotune(tp_br_ctx* ctx, uint64_t batch, uint32_t* best_coef_per_thread,
                         double* best_rotations_per_s);

/* Waits for the context's work on `stream` and reports device-side input
 * errors seen since the last check (TP_ERR_PARAM for out-of-range LWE words). */
tp_status tp_br_check(tp_br_ctx* ctx, void* stream);

/* SampleExtract at index 0 of a batch of RLWE ciphertexts in the coefficient
 * domain (lib/include/static/sample_extraction.h:20-36), device buffers: out
 * b gets N+1 words at out + b*(N+1). The reference leaves a word untouched
 * where the source coefficient is 0; this kernel writes 0 there, which equals
 * the reference's result on a pre-zeroed buffer. */
tp_status tp_sample_extract_batch(uint32_t ring_dim, uint64_t batch, uint64_t* out_dev, const uint64_t* rlwe_dev,
                                  void* stream);

/* A batch launch recorded once as a CUDA graph and replayed many times, for
 * loops that rotate fresh ciphertexts through the same device buffers (the
 * graph reads the buffers' contents at replay time). With extract_out != NULL
 * the graph also runs SampleExtract (index 0) on every result into
 * extract_out (batch x (N+1) words), which needs out_coef = 1: rotation and
 * extraction then cost one graph launch. No reference counterpart (the
 * reference runs one rotation per call). Capture happens on a private stream;
 * the context's key must be uploaded first. */
typedef struct tp_graph tp_graph;
tp_status tp_br_batch_graph_create(tp_br_ctx* ctx, uint64_t batch, uint64_t* results_dev, const uint64_t* lwes_dev,
                                   uint64_t lwe_stride, const uint64_t* accs_dev, uint64_t acc_stride, int out_coef,
                                   uint64_t* extract_out_dev, tp_graph** out);
tp_status tp_graph_launch(tp_graph* graph, void* stream);
tp_status tp_graph_destroy(tp_graph* graph);

/* Batched negacyclic NTT on device buffers, `count` polynomials of N words,
 * in-place allowed. Replaces SolinasWorker::ForwardNTT / BackwardNTT
 * (lib/src/backend/solinas.cpp:228-313); backward includes 1/N. */
tp_status tp_ntt_forward(uint32_t ring_dim, uint64_t count, uint64_t* out_dev, const uint64_t* in_dev,
                         void* stream);
tp_status tp_ntt_backward(uint32_t ring_dim, uint64_t count, uint64_t* out_dev, const uint64_t* in_dev,
                          void* stream);

/* ---- Key switching, automorphisms, packing ------------------------------ */

typedef struct tp_ks_ctx tp_ks_ctx;

/* RLWE -> RLWE key switching context, RLWEConversionContext(distr, modulus, N,
 * basis, digits, std) (lib/include/operators/endo_glwe_conversion.h:256).
 * Key: the converter's m_ksk, l rows of [A | B] in the NTT domain (KeyGen,
 * lib/src/operators/rlwe_conversion.cpp:187-218). */
tp_status tp_rlwe_ks_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, int device, tp_ks_ctx** out);

/* Automorphism X -> X^index followed by the key switch s(X^index) -> s(X),
 * AutomorphismContext(..., automorphism_index) (lib/include/operators/automorphism_evaluation.h:25);
 * index odd and below 2N. Key: the inner converter's m_ksk. */
tp_status tp_auto_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, uint32_t index, int device,
                         tp_ks_ctx** out);

/* n-LWE -> RLWE packing, LWEtoRLWEPackingContext(distr, modulus, N, basis,
 * digits, std) (lib/include/operators/lwe_to_rlwe_packing.h:18). Keys: the
 * automorphism keys for indices 2^j + 1, j = 1..log2 N, each l x 2N words,
 * concatenated in that order (the evaluators of ConstructOperator,
 * lib/src/operators/lwe_to_rlwe_packing.cpp:46-58). */
tp_status tp_pack_create(uint32_t ring_dim, uint64_t basis, uint32_t digits, int device, tp_ks_ctx** out);

tp_status tp_ks_destroy(tp_ks_ctx* ctx);
uint64_t tp_ks_key_words(const tp_ks_ctx* ctx);
/* Host key in the reference layout above; re-laid out on the device. Synchronous. */
tp_status tp_ks_upload_key(tp_ks_ctx* ctx, const uint64_t* key_host, uint64_t words);

/* Coefficients per thread of the key-switching kernels (4 or 8; default 4):
 * N/4 or N/8 threads per ciphertext. The resident key is re-laid out for the
 * new tile. Results do not depend on it. */
tp_status tp_ks_set_tile(tp_ks_ctx* ctx, uint32_t coef_per_thread);
uint32_t tp_ks_get_tile(const tp_ks_ctx* ctx);

/* Batched RLWEtoRLWEConverter::Convert(out, in) (rlwe_conversion.cpp:224-249),
 * device buffers of 2N words per ciphertext: in = [A coefficients | B NTT];
 * out -= KS(in.A) and out.B += in.B, like the reference (which expects a
 * pre-zeroed out). out may equal in. Asynchronous. */
tp_status tp_rlwe_ks_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev, void* stream);

/* Batched AutomorphismEvaluator::Eval(out, in) (automorphism_evaluation.cpp:150-159):
 * in = [A | B] coefficients, out (NTT domain) -= KS(aut(A)), out.B += NTT(aut(B)).
 * out must not alias in. Asynchronous. */
tp_status tp_auto_eval_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev,
                             void* stream);

/* Batched LWEtoRLWEPacker::Pack(out, in, len) (lwe_to_rlwe_packing.cpp:129-236):
 * `packs` packings of `len` LWEs each (len a power of two in [2, N]; LWE e of
 * pack p at in + (p*len + e)*(N+1)), out + p*2N gets the packed RLWE in the
 * coefficient domain. The tree runs level by level over all packs, one launch
 * per level, in a context-owned work area of packs*len*2N words. Asynchronous. */
tp_status tp_pack_batch(tp_ks_ctx* ctx, uint64_t packs, uint64_t len, uint64_t* out_dev, const uint64_t* in_dev,
                        void* stream);
/* The packing tree split into shards, for a packing spread over several devices (no
 * counterpart call in the reference: Pack (lwe_to_rlwe_packing.cpp:129-236) runs the
 * whole tree in one call). A level-L merge depends only on L, so the subtree of leaf
 * positions [r m, (r + 1) m) (m = len / W, W shards) is a pack of m inputs taken with
 * stride W: input j W + s of pack p, s = (W - 1) ^ brv_{log2 W}(r), becomes that
 * subtree's input j. tp_pack_subtree_batch runs the L0 set-up and merges of levels
 * 1 .. log2 len of `packs` such subtrees (len = m inputs each, laid out as for
 * tp_pack_batch, 1 <= len <= N) and writes each root (2N coefficient words, no
 * traces) to out + p*2N. tp_pack_merge_batch continues a tree: nodes holds `packs`
 * groups of `count` roots of level `level0` in position order (count a power of two,
 * level0 + log2 count <= log2 N); it merges each group at levels level0 + 1 ..
 * level0 + log2 count and, with `finish` != 0, applies the trailing traces, so
 * out + p*2N gets what tp_pack_batch gives for the whole tree. Scratch: the
 * context's work area (packs x len or count x 2N words). Asynchronous. */
tp_status tp_pack_subtree_batch(tp_ks_ctx* ctx, uint64_t packs, uint64_t len, uint64_t* out_dev,
                                const uint64_t* in_dev, void* stream);
tp_status tp_pack_merge_batch(tp_ks_ctx* ctx, uint64_t packs, uint64_t count, uint32_t level0, int finish,
                              uint64_t* out_dev, const uint64_t* nodes_dev, void* stream);
/* LWEtoRLWEPacker::PackConsecutively(out, in, len) (lwe_to_rlwe_packing.cpp:260-393)
 * for `packs` packings of len inputs each (2 <= len <= N, any length): the inputs
 * land on the first len coefficients. Runs the reference's full N-leaf tree with
 * the empty subtrees cut away: per level one launch over the nodes that have an
 * input below them (an empty sibling reads as zero). Device buffers as for
 * tp_pack_batch; scratch 2 x packs x len x 2N words. Asynchronous. */
tp_status tp_pack_consecutive_batch(tp_ks_ctx* ctx, uint64_t packs, uint64_t len, uint64_t* out_dev,
                                    const uint64_t* in_dev, void* stream);
/* TraceEvaluator::Eval(out, in) (lib/src/operators/trace_evaluation.cpp:135-158) on a
 * packing context (its keys are the trace's, indices 3, 5, .., N+1): in = [A | B]
 * coefficients; out = NTT of both halves of N^-1 Tr(in), the key-switched trace the
 * reference computes. out may equal in. Asynchronous. */
tp_status tp_trace_eval_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev,
                              void* stream);
/* TraceEvaluator::EvalAuto(out, in, auto_index) (lines 172-179, the pointer overload):
 * the automorphism X -> X^auto_index, auto_index = 2^j + 1, with the trace's key for it;
 * AutomorphismEvaluator::Eval semantics (out -= ..., NTT domain; out zeroed by the caller). */
tp_status tp_trace_eval_auto_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev,
                                   uint32_t auto_index, void* stream);

/* tp_pack_batch for callers that cannot allocate device memory when they call:
 * a process whose HBM is owned by another allocator's pool, or a latency-bound
 * loop that must not risk cudaMalloc/cudaFree blocking or synchronising the
 * device. The packing-tree nodes live in a fixed device array of 16 MiB
 * (2^21 words) instead of a cudaMalloc'd work area; calls with
 * packs * len * 2N above 2^21 words fail with TP_ERR_PARAM. The call itself
 * allocates nothing. Its first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture; that address stays valid while the device's
 * primary context lives (do not call it again on a device after cudaDeviceReset).
 * Like every call on a context it holds the context's lock while it reads the
 * key and enqueues its launches. Every GPU that loads the library holds the
 * array until the process exits. All calls on a device share the one array:
 * calls whose work overlaps on the GPU (different streams, or different
 * contexts on the same device) race and corrupt each other, so order them.
 * Nothing carries over between calls: the set-up kernel rewrites every node
 * word a call reads. No counterpart in the reference, which always packs on
 * host buffers it allocates itself. */
tp_status tp_pack_batch_noalloc(tp_ks_ctx* ctx, uint64_t packs, uint64_t len, uint64_t* out_dev,
                                const uint64_t* in_dev, void* stream);

typedef struct tp_lwe_ks_ctx tp_lwe_ks_ctx;

/* LWE -> LWE key switching, LWEConversionContext(distr, modulus, n_in, n_out,
 * basis, digits, std) (lib/include/operators/endo_glwe_conversion.h:28), on the
 * Goldilocks modulus. Key: the converter's m_ksk, n_in x digits x (n_out+1)
 * (KeyGen, lib/src/operators/lwe_conversion.cpp:174-203), used as laid out. */
tp_status tp_lwe_ks_create(uint64_t modulus, uint32_t n_in, uint32_t n_out, uint64_t basis, uint32_t digits,
                           int device, tp_lwe_ks_ctx** out);
tp_status tp_lwe_ks_destroy(tp_lwe_ks_ctx* ctx);
uint64_t tp_lwe_ks_key_words(const tp_lwe_ks_ctx* ctx);
tp_status tp_lwe_ks_upload_key(tp_lwe_ks_ctx* ctx, const uint64_t* key_host, uint64_t words);

/* Batched LWEtoLWEConverter::Convert(out, in) (lwe_conversion.cpp:205-239):
 * in b has n_in+1 words, out b has n_out+1 words; out[n_out] = in[n_in] and
 * out -= sum of signed digits times key rows (the reference expects out[0..n_out)
 * pre-zeroed). Asynchronous. */
tp_status tp_lwe_ks_batch(tp_lwe_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev, void* stream);

/* ModulusSwitch (lib/src/static/modulus_switching.cpp:36-93) in place on a
 * device vector: source must be the Goldilocks prime p, target a power of two
 * up to 2^32 (2N), type ROUND, FLOOR or CEIL (RANDOM, which draws from an
 * unseeded generator, is not offered). Each word equals the reference's 80-bit
 * long-double result (roundl / floorl / ceill of (target * v) / p, then minus
 * target where it reaches target), computed exactly with integers. */
#define TP_MS_ROUND 0
#define TP_MS_FLOOR 1
#define TP_MS_CEIL 2
tp_status tp_modulus_switch_batch(uint64_t count, uint64_t* vec_dev, uint64_t source_modulus,
                                  uint64_t target_modulus, int type, void* stream);

/* The bootstrap epilogue, fused: SampleExtract at index 0 of each RLWE
 * (coefficient domain, batch x 2N words), LWE->LWE key switch with `ks`
 * (n_in = N, fresh output), then the FLOOR switch to `target_modulus` (2N to
 * feed the next blind rotation): out gets batch x (n_out + 1) words. This is
 * the refresh step of SAPDecomposer (lib/src/operators/sap_decomposer.cpp:353-
 * 369: SampleExtract, LWEtoLWEConverter::Convert, ModulusSwitch FLOOR to 2N)
 * for Qks = Q. */
tp_status tp_pbs_epilogue_batch(tp_lwe_ks_ctx* ks, uint64_t batch, uint64_t* out_lwe_dev,
                                const uint64_t* rlwe_coef_dev, uint64_t target_modulus, void* stream);

/* One graph for a whole bootstrap batch: blind rotation (coefficient output
 * into rlwe_scratch_dev, batch x 2N words) followed by tp_pbs_epilogue_batch
 * to 2N. The output LWEs (dimension n_out of `ks`) feed the next rotation with
 * a context whose lwe_dim is n_out. Replay with tp_graph_launch. No reference
 * counterpart as one call. */
tp_status tp_pbs_graph_create(tp_br_ctx* br, tp_lwe_ks_ctx* ks, uint64_t batch, uint64_t* rlwe_scratch_dev,
                              const uint64_t* lwes_dev, const uint64_t* accs_dev, uint64_t acc_stride,
                              uint64_t* out_lwe_dev, tp_graph** out);


/* ---- Serving loop -------------------------------------------------------- */
/* Continuous batching of single bootstrap requests over several resident
 * parameter sets (no reference counterpart: the reference rotates one
 * ciphertext per call on the calling thread). */
typedef struct tp_server tp_server;

/* max_queue bounds the requests waiting for a launch buffer; further submits
 * are rejected (admission control). 0 = 2^20. */
tp_status tp_server_create(int device, uint64_t max_queue, tp_server** out);

/* Registers a parameter set served by `ctx` (created and keyed by the caller,
 * kept alive until the server is destroyed): `buffers` launch buffers of
 * `max_batch` requests each are reserved on the device and in pinned host
 * memory now, which bounds how many of the set's requests are on the GPU at
 * once. Results are NTT domain, or coefficients when out_coef != 0. */
tp_status tp_server_add_set(tp_server* srv, tp_br_ctx* ctx, uint32_t ring_dim, uint32_t lwe_dim, uint32_t max_batch,
                            uint32_t buffers, int out_coef, uint32_t* set_id);

/* Device-memory admission. Every admitted request reserves its device bytes
 * ((n+1) + 4N words: its LWE, test polynomial and result in a launch buffer)
 * from the server's budget until its result is back in host memory; a submit
 * that would exceed the budget is rejected with TP_ERR_OOM (and counted). The
 * budget defaults to the device memory still free at tp_server_start (keys and
 * launch buffers resident); tp_server_set_memory_budget sets it explicitly, at
 * any time. tp_server_memory reads the budget, the bytes reserved now and the
 * number of requests refused for memory (any output may be NULL). */
tp_status tp_server_set_memory_budget(tp_server* srv, uint64_t bytes);
tp_status tp_server_memory(tp_server* srv, uint64_t* budget, uint64_t* in_use, uint64_t* rejected_memory);

/* Starts the scheduler thread (after every tp_server_add_set). */
tp_status tp_server_start(tp_server* srv);

/* Queues one rotation of set `set_id`: lwe (n+1 words) and acc (2N words) are
 * read and result (2N words) written by the scheduler, so the host buffers
 * must stay valid until tp_server_wait returns for the ticket. Returns
 * TP_ERR_STATE when the queue is full and TP_ERR_OOM when the device-memory
 * budget is (the request is not admitted either way). */
tp_status tp_server_submit(tp_server* srv, uint32_t set_id, const uint64_t* lwe, const uint64_t* acc,
                           uint64_t* result, uint64_t* ticket);
tp_status tp_server_wait(tp_server* srv, uint64_t ticket, uint32_t timeout_ms);
/* Waits until no request is queued or in flight. */
tp_status tp_server_drain(tp_server* srv, uint32_t timeout_ms);
/* stats8 = {completed, rejected, launches, seconds from first submit to last
 * completion, p50, p99, p99.9, max latency (ms, submit to result in host memory)}. */
tp_status tp_server_stats(tp_server* srv, double* stats8);
tp_status tp_server_reset_stats(tp_server* srv);
tp_status tp_server_destroy(tp_server* srv);
const char* tp_server_last_error(void);

/* Open-loop load generator for the serving benchmark: Poisson arrivals at
 * `rate` requests/s for `seconds`; set i with probability mix[i]; inputs taken
 * round-robin from per-set pools (pool_n[i] rows). Waits for every admitted
 * request to finish. */
tp_status tp_server_run_poisson(tp_server* srv, double rate, double seconds, const double* mix, uint32_t nsets,
                                const uint64_t* const* pool_lwe, const uint64_t* const* pool_acc,
                                const uint64_t* pool_n, uint64_t seed);

/* Diagnostic: element-wise Goldilocks primitives of the kernels on device
 * buffers, for testing them against exact integer arithmetic. op: 0 a+b,
 * 1 a-b, 2 a*b (a, b canonical); 3 c + a*b (any 64-bit a, b, c); 4 reduction
 * of the 128-bit value a + 2^64 b; 5 canonical form of a; 6 op 4 through the
 * canonical reduction (its own output, not re-canonicalised); 7 lazy a+b,
 * 8 a+b, 9 a-b (any 64-bit a, b canonical). Results canonical.
 * No reference counterpart (internal arithmetic check). */
tp_status tp_debug_arith(int op, uint64_t count, uint64_t* out_dev, const uint64_t* a_dev, const uint64_t* b_dev,
                         const uint64_t* c_dev, void* stream);

/* Measures, on `device`, the throughput of the 64x64 -> 128-bit integer
 * product every Goldilocks modmul needs (32-bit IMAD chains, as in the
 * kernels) and of plain 32-bit mad.lo, in operations per second. The
 * benchmark uses the product rate as the INT32 roof. No reference
 * counterpart. */
tp_status tp_measure_int_peak(int device, double* products_per_s, double* imad_per_s);

/* ---- LWE -> RGSW scheme switching -------------------------------------------
 * LWEtoRGSWConverter::Convert (lib/src/operators/lwe_to_rgsw_conversion.cpp:168-
 * 225) of a SchemeSwitchingContext(rotation, trace, squaring, out_digits,
 * out_basis) on the Goldilocks modulus. Lines 10-110 build the context from a
 * rotation context of any variant, a TraceEvaluationContext and an
 * RLWEConversionContext, each with its own gadget. Per LWE: a blind rotation of the context's test polynomial, Lev extraction,
 * a trace over the automorphisms N+1 .. 3 and a key switch from s^2 to s per
 * row. Keys in the reference's layouts: the blind-rotation key (m_brk), the
 * trace's automorphism keys for indices 3, 5, 9, .., N+1 concatenated (as the
 * packer takes them), and the squaring converter's m_ksk. Output per LWE:
 * 4 N out_digits words [lev_left rows | lev_right rows], NTT domain.
 * out_digits must divide N into even blocks. */
typedef struct tp_ss_ctx tp_ss_ctx;
tp_status tp_ss_create(const tp_br_params* rotation, uint64_t trace_basis, uint32_t trace_digits,
                       uint64_t square_basis, uint32_t square_digits, uint32_t out_digits, uint64_t out_basis,
                       int device, tp_ss_ctx** out);
tp_status tp_ss_destroy(tp_ss_ctx* ctx);
/* which: 0 blind-rotation key, 1 trace keys, 2 squaring key */
uint64_t tp_ss_key_words(const tp_ss_ctx* ctx, int which);
tp_status tp_ss_upload_keys(tp_ss_ctx* ctx, const uint64_t* brk, uint64_t brk_words, const uint64_t* trace_keys,
                            uint64_t trace_words, const uint64_t* square_key, uint64_t square_words);
/* The converter's accumulator (3N words: [0 | -tp | tp]), for checks. */
tp_status tp_ss_accumulator(const tp_ss_ctx* ctx, uint64_t* out_host);
tp_status tp_lwe_to_rgsw_batch(tp_ss_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* lwes_dev,
                               void* stream);

/* ---- SAP digit decomposition ---------------------------------------------
 * SAPDecomposer::Decompose (lib/src/operators/sap_decomposer.cpp:353-464) of a
 * SAPDecompositionContext(rotation, trace, LWE conversion N -> n, radix) on the
 * Goldilocks modulus, for a batch of LWEs per call. Per digit: a blind rotation
 * of the LWE's running accumulator by its next radix digit, the digit's
 * SampleExtract, optionally ResetAccumulator (lines 293-351: overflow
 * extraction, LWE key switch, FLOOR switch to 2N, a fresh rotation), and
 * HomTrunc (lines 189-291: partial trace and the truncation tree of automorphism
 * key switches). Keys in the reference's layouts: the rotator's m_brk, the trace
 * evaluators' m_ksk for indices 3, 5, 9, .., N+1 concatenated, and the LWE
 * converter's m_ksk (N -> n). */
typedef struct tp_sap_ctx tp_sap_ctx;
tp_status tp_sap_create(const tp_br_params* rotation, uint64_t trace_basis, uint32_t trace_digits, uint64_t ks_basis,
                        uint32_t ks_digits, int device, tp_sap_ctx** out);
tp_status tp_sap_destroy(tp_sap_ctx* ctx);
/* which: 0 blind-rotation key, 1 trace keys, 2 LWE key switch */
uint64_t tp_sap_key_words(const tp_sap_ctx* ctx, int which);
tp_status tp_sap_upload_keys(tp_sap_ctx* ctx, const uint64_t* brk, uint64_t brk_words, const uint64_t* trace_keys,
                             uint64_t trace_words, const uint64_t* lwe_ksk, uint64_t lwe_ksk_words);
/* Decomposes `batch` LWEs (device, rows of n+1 words; the input modulus of each
 * is read from its words as the reference does) in base `radix` (a power of two
 * in [2, N]) with the LWE key's Hamming weight `hamming_weight` (the reference's
 * m_beta) and the accumulator reset every `restart_period` digits (the
 * context's GetRestartIteration(); UINT64_MAX: never). Output (device): LWE b's
 * digit d at out + (b out_digits + d)(N+1), an LWE of dimension N mod Q; words
 * past an LWE's digit count are left untouched. digits_host (optional, batch
 * entries) receives each LWE's digit count. Reads the input moduli back once
 * (synchronising `stream`); the rest is asynchronous. Refuses the call if an LWE
 * needs more than out_digits digits. */
tp_status tp_sap_decompose_batch(tp_sap_ctx* ctx, uint64_t batch, uint64_t* out_dev, uint64_t out_digits,
                                 const uint64_t* lwes_dev, uint64_t radix, uint64_t hamming_weight,
                                 uint64_t restart_period, uint32_t* digits_host, void* stream);
/* SAPDecomposer::HomTrunc(output, input, radix) (lines 189-291) on `batch` RLWEs
 * (device, 2N words each, NTT domain in and out); radix a power of two in [2, N]. */
tp_status tp_sap_homtrunc_batch(tp_sap_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev,
                                uint64_t radix, void* stream);
/* SAPDecomposer::ResetAccumulator(acc, radix) (lines 293-351) on `batch` RLWEs in
 * place (device, NTT domain); radix 0 (as Decompose passes it) or a power of two.
 * The LWE key switch runs as on a fresh converter. */
tp_status tp_sap_reset_batch(tp_sap_ctx* ctx, uint64_t batch, uint64_t* acc_dev, uint64_t radix, void* stream);

/* ---- Key files ------------------------------------------------------------
 * The reference keeps keys only in memory (no serialization). A key file holds
 * one key in the reference's own layout (the words tp_*_upload_key takes)
 * behind a 128-byte header: magic "TPKEYv1", kind, parameters, word count and
 * the SHA-256 of the payload; all fields little-endian. Reading checks the
 * magic, the layout tag and the hash (TP_ERR_LAYOUT on a mismatch); the
 * *_upload_key_file calls also check the header against the context's
 * parameters before uploading. Writing a ciphertext batch checks that the word
 * count is count x row words. Host-only, no device needed to read or write. */
typedef enum {
    TP_KEY_BLIND_ROTATION = 1, /* m_brk: variant, ring_dim N, lwe_dim n */
    TP_KEY_RLWE_SWITCH = 2,    /* RLWEtoRLWEConverter m_ksk: ring_dim */
    TP_KEY_AUTOMORPHISM = 3,   /* AutomorphismEvaluator key: ring_dim, index */
    TP_KEY_PACKING = 4,        /* LWEtoRLWEPacker: log2 N automorphism keys, ring_dim */
    TP_KEY_LWE_SWITCH = 5,     /* LWEtoLWEConverter m_ksk: ring_dim = n_in, lwe_dim = n_out */
    /* Ciphertext batches in the same container (index = number of ciphertexts): */
    TP_CT_LWE = 16,            /* rows of lwe_dim+1 words [a | b] mod `modulus` (2N before a rotation) */
    TP_CT_RLWE = 17            /* rows of 2N words [A | B]; variant 0: coefficients, 1: NTT domain */
} tp_key_kind;

typedef struct {
    uint32_t kind, variant, ring_dim, lwe_dim, digits, index;
    uint64_t modulus, basis, words;
} tp_key_info;

tp_status tp_key_file_write(const char* path, const tp_key_info* info, const uint64_t* words);
tp_status tp_key_file_info(const char* path, tp_key_info* info);
tp_status tp_key_file_read(const char* path, tp_key_info* info, uint64_t* words, uint64_t capacity);
tp_status tp_br_upload_key_file(tp_br_ctx* ctx, const char* path);
tp_status tp_ks_upload_key_file(tp_ks_ctx* ctx, const char* path);
tp_status tp_lwe_ks_upload_key_file(tp_lwe_ks_ctx* ctx, const char* path);

/* Message for the last failing call on this thread ("" if none). */
const char* tp_last_error(void);
/* Kernels this library has launched in this process so far (a replay of a
 * graph made by tp_*_graph_create counts its kernels; launches recorded into
 * such a graph count when it is replayed). For accounting in benchmarks. No
 * reference counterpart. */
uint64_t tp_kernel_launches(void);

/* Library version string. */
const char* tp_version(void);

/* ---- Short names for the blind-rotation calls ------------------------------
 * The same functions under the short names: a context is a blind-rotation
 * context, its key the rotator's m_brk (layout_tag TP_LAYOUT_REFERENCE, the
 * only layout accepted), batch rows of n+1 LWE words. */
typedef tp_br_params tp_params;
typedef tp_br_ctx tp_ctx;
#define TP_LAYOUT_REFERENCE 0
tp_status tp_ctx_create(const tp_params* params, tp_ctx** out);  /* device 0; tp_br_create for others */
tp_status tp_ctx_destroy(tp_ctx* ctx);
tp_status tp_brk_upload(tp_ctx* ctx, const uint64_t* brk, uint64_t words, int layout_tag);
tp_status tp_blind_rotate(tp_ctx* ctx, uint64_t* result, const uint64_t* lwe, const uint64_t* acc, int out_coef);
tp_status tp_blind_rotate_batch(tp_ctx* ctx, uint64_t batch, uint64_t* results_dev, const uint64_t* lwes_dev,
                                const uint64_t* accs_dev, uint64_t acc_stride, int out_coef, void* stream);
tp_status tp_auto_ks_batch(tp_ks_ctx* ctx, uint64_t batch, uint64_t* out_dev, const uint64_t* in_dev, void* stream);
const char* tp_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif
