// Library-internal helpers shared between translation units: the rotation
// launch with an explicit split (the serving loop chooses the kernel per
// launch) and the error recorder. Not part of the C ABI.
#pragma once

#include "toothpaste_gpu.h"

namespace tp {

// split 0: the context's setting; 1: one block per rotation; 2 / 4: the two- /
// four-block cluster kernel when the context's tile and the device allow it
// (else the next smaller form).
tp_status br_batch_launch(tp_br_ctx* c, uint64_t batch, uint64_t* results, const uint64_t* lwes,
                          uint64_t lwe_stride, const uint64_t* accs, uint64_t acc_stride, int out_coef, void* stream,
                          int split);

// Records an error message for tp_last_error() (the calling thread's) and
// returns `s`; for the library's other translation units.
tp_status set_error(tp_status s, const char* fmt, ...);

// Rotations the device runs at once with one, two or four blocks per rotation
// (split 1, 2, 4); 0 when that kernel is not available for the context.
uint64_t br_concurrency(const tp_br_ctx* c, int split);

// CTAs (SMs) one rotation occupies with one block per rotation: 1, or the cluster
// size of a ring above 4096.
int br_cluster_ctas(const tp_br_ctx* c);

}  // namespace tp
