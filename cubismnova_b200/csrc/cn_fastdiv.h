// cn_fastdiv.h -- division of non-negative 31-bit integers by a divisor fixed
// at launch time, as one multiply-high, one add and one shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, the round-up method with a 33-bit multiplier 2^32 + m):
//   s = ceil(log2 d),  m = floor(2^32 (2^s - d) / d) + 1,
//   n / d = (umulhi(n, m) + n) >> s        for 0 <= n < 2^31, d >= 1.
// The multiplier 2^32 + m = ceil(2^(32+s) / d) exceeds 2^(32+s) / d by less
// than 2^s / d <= 1 per unit of d, which keeps the quotient exact for every
// n < 2^32; n < 2^31 keeps the 32-bit sum umulhi(n, m) + n from overflowing.
// Runtime integer division by a variable compiles to a long sequence that
// includes a multi-function-unit reciprocal; index decompositions in the
// stencil kernels use this instead.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace cn {

struct FastDiv {
    uint32_t d = 1, m = 1, s = 0;

    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div)
    {
        d = div < 1 ? 1 : div;
        s = 0;
        while ((uint64_t(1) << s) < d) ++s;
        m = (uint32_t)((((uint64_t(1) << s) - d) << 32) / d + 1);
    }
    // n in [0, 2^31)
    __host__ __device__ __forceinline__ int div(int n) const
    {
#ifdef __CUDA_ARCH__
        return (int)((__umulhi((uint32_t)n, m) + (uint32_t)n) >> s);
#else
        return (int)(((uint32_t)(((uint64_t)(uint32_t)n * m) >> 32) + (uint32_t)n) >> s);
#endif
    }
};

} // namespace cn
