// Prints the shared-memory plan of the rotation kernels for every ring size and
// variant (host code only: no kernel runs, no GPU needed). One line per
// (logn, variant): logn variant one_block_words pair_words quad_fits quad_words
// quad_xbufs pair_prefetch quad_prefetch, for n = 1023 LWE words; then for the ring
// sizes that rotate on CTA clusters one line "C logn variant logs one_block_words
// ks_words" (the per-CTA plans of the rotation and key-switching kernels).
// Used by tests/test_smem_plan_cpu.py.
#include <cstdio>

#include "br_pair_kernel.cuh"
#include "ks_kernels.cuh"

int main() {
    const unsigned n = 1023;
    for (int logn = 7; logn <= 12; ++logn)
        for (int v = 0; v <= 2; ++v)
            std::printf("%d %d %zu %zu %d %zu %d %d %d\n", logn, v, tp::br_smem_words(logn, v, n, 2),
                        tp::br_pair_smem_words(logn, v, n, 2, 2), tp::br_quad_fits(logn, v) ? 1 : 0,
                        tp::br_pair_smem_words(logn, v, n, 2, 4), tp::br_split_xbufs(logn, v, 4),
                        tp::br_pair_key_prefetch(logn, v, 2) ? 1 : 0, tp::br_pair_key_prefetch(logn, v, 4) ? 1 : 0);
    for (int logn = 13; logn <= 16; ++logn)
        for (int v = 0; v <= 2; ++v) {
            const int logs = tp::br_cluster_logs(logn);
            std::printf("C %d %d %d %zu %d\n", logn, v, logs, tp::br_smem_words(logn, v, n, 2, 0, logs),
                        tp::ks_smem_words(1 << logn, 1 << logs));
        }
    return 0;
}
