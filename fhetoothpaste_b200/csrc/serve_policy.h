// Launch form of one serving launch: plain C++ (no CUDA types), shared by the
// scheduler in serve.cu and its CPU test.
#pragma once

#include <algorithm>
#include <cstdint>

namespace tp {

// Largest launch the scheduler runs with four blocks per rotation.
constexpr uint64_t kServeFourBlockMax = 8;

// Blocks per rotation for a launch of `take` requests. Four when the launch is
// small (at most kServeFourBlockMax requests), the set's four-block kernel holds
// it at once (take <= conc4; conc4 = 0 where that kernel does not fit) and its
// 4 * take blocks fit on the SMs that the launches in flight (`busy` blocks)
// leave free; else two when the two-block kernel holds it (take <= conc2); else
// one block per rotation.
inline int serve_split(uint64_t take, uint64_t busy, uint64_t sm_count, uint64_t conc4, uint64_t conc2) {
    if (take <= kServeFourBlockMax && take <= conc4 && busy + 4 * take <= sm_count) return 4;
    if (take <= conc2) return 2;
    return 1;
}

// Thread blocks a launch keeps busy: `split` per rotation, for at most the
// `conc` rotations that form runs at once.
inline uint64_t serve_blocks(int split, uint64_t take, uint64_t conc) {
    return (uint64_t)split * std::min<uint64_t>(take, std::max<uint64_t>(conc, 1));
}

}  // namespace tp
