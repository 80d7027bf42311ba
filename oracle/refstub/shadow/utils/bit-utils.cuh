// Stand-in for the reference's src/utils/bit-utils.cuh in the oracle/_ref host build. The
// reference header declares the popcount kernel get_1s_per_uint32 (defined, and compiled from
// the reference, in src/utils/bit-utils.cu), the next_power_of_two helper, and a host template
// count_1s that launches the kernel with <<<...>>> and sums with thrust::reduce; a host
// compiler cannot parse that launch, so this stand-in keeps the declarations and leaves
// count_1s out (ref_driver.cpp sums the per-word counts itself). The build finds this file
// ahead of the reference's by searching quoted includes through the include path only (-I-).
#pragma once

#include <cstddef>
#include <cstdint>

#include "../common.h"

TURBO_NAMESPACE_BEGIN

// Smallest power of two >= v (v >= 1).
template <typename T>
inline T next_power_of_two(T v) {
    T p = 1;
    while (p < v) p <<= 1;
    return p;
}

__global__ void get_1s_per_uint32(const size_t n_elements, const uint32_t* __restrict__ buffer,
                                  uint8_t* __restrict__ counts);

TURBO_NAMESPACE_END
