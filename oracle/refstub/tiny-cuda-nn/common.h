// Host stand-in for the parts of tiny-cuda-nn's common header that the reference's hot-path
// kernels use (oracle/_ref build only). tiny-cuda-nn is an un-vendored git submodule of the
// reference (its directory is empty); these are written here from the definitions:
//  - network_precision_t: the network's value type; float, as in the fp32 path this
//    repository implements (the reference's fp16 build would round values to half);
//  - clamp(v, lo, hi): min(max(v, lo), hi) with the reference's argument order;
//  - morton3D / morton3D_invert: 3 x 10-bit Z-order interleave, x in bit 0, y in bit 1, z in
//    bit 2 of every triple (the reference's inverse at occupancy-grid.cuh:173-175 fixes the
//    order), written as a plain bit loop;
//  - CUDA_CHECK_THROW and the namespace macros.
#pragma once

#include <cstdint>
#include <sstream>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#define TCNN_NAMESPACE_BEGIN namespace tcnn {
#define TCNN_NAMESPACE_END }
#define TCNN_HOST_DEVICE

#define CUDA_CHECK_THROW(x)                                                              \
    do {                                                                                 \
        cudaError_t tn_ref_status = (x);                                                 \
        if (tn_ref_status != cudaSuccess) throw std::runtime_error("host stand-in: " #x); \
    } while (0)

namespace tcnn {

using network_precision_t = float;

template <typename T>
inline T clamp(T v, T lo, T hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

inline uint32_t morton3D(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t m = 0;
    for (int b = 0; b < 10; ++b) {
        m |= ((x >> b) & 1u) << (3 * b);
        m |= ((y >> b) & 1u) << (3 * b + 1);
        m |= ((z >> b) & 1u) << (3 * b + 2);
    }
    return m;  // coordinates use 10 bits; higher bits never occur on a 128^3 grid
}

inline uint32_t morton3D_invert(uint32_t m) {
    uint32_t x = 0;
    for (int b = 0; b < 10; ++b) x |= ((m >> (3 * b)) & 1u) << b;
    return x;
}

inline uint32_t n_blocks_linear(uint32_t n, uint32_t threads = 128) { return (n + threads - 1) / threads; }

}  // namespace tcnn
