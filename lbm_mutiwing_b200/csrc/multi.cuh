// Device side of the packed launches declared in lbm_kernels.h: the episode
// of a block, by binary search over the block offsets.
#pragma once
#include "lbm_kernels.h"

namespace lbm {

__device__ __forceinline__ int multi_episode(const MultiArgs& m, int b) {
    int lo = 0, hi = m.ne - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(m.boff + mid) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace lbm
