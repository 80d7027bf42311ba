// Host stand-in for the CUDA runtime header, used only to compile the reference's own kernel
// sources on the CPU (oracle/_ref). It is written for this oracle, not taken from CUDA:
//  - the execution-space qualifiers are empty, so a __global__ kernel is a plain function;
//  - threadIdx / blockIdx / blockDim / gridDim are thread-local variables that the driver
//    (oracle/ref_driver.cpp) sets before it calls a kernel once per CUDA thread;
//  - the vector types carry the members the reference reads;
//  - the few device intrinsics the reference's hot-path kernels call are defined from their
//    documented meaning: __fdiv_ru is IEEE division rounded toward +infinity (computed exactly,
//    see below), __popc counts set bits, and the fast approximations __expf / __powf /
//    __fdividef are the C library's expf / powf and an IEEE division (so float outputs that
//    depend on them agree with the GPU only to a few ulp, never bit for bit);
//  - the memory calls a reference workspace makes (cudaMallocAsync, cudaMemsetAsync, ...) are
//    served from host memory. Every allocation carries 16 MiB of zeroed guard bytes after its
//    end: the reference indexes its bitfield with an unclamped Morton code, which on the
//    bounding box's max face lands up to 7 * 2^21 bytes past a 128^3 grid.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __align__(n) alignas(n)

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x = 1, y = 1, z = 1;
    dim3() = default;
    dim3(unsigned int x_, unsigned int y_ = 1, unsigned int z_ = 1) : x(x_), y(y_), z(z_) {}
};
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };

inline float2 make_float2(float x, float y) { return float2{x, y}; }
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

// Division rounded toward +infinity. The double quotient of two floats is never within half
// a double ulp of a float unless it equals it (the exact quotient a/b differs from any other
// float f by at least |a - f*b| / |b|, a multiple of 2^-48 relative), so rounding the double
// quotient to the nearest float and stepping up when that is below it gives the exact result.
inline float __fdiv_ru(float a, float b) {
    const double q = (double)a / (double)b;
    float f = (float)q;
    if ((double)f < q) f = std::nextafter(f, INFINITY);
    return f;
}
inline float __expf(float x) { return std::exp(x); }
inline float __powf(float x, float y) { return std::pow(x, y); }
inline float __fdividef(float a, float b) { return a / b; }
inline int __popc(unsigned int v) { return __builtin_popcount(v); }

typedef int cudaError_t;
typedef void* cudaStream_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
                      cudaMemcpyDeviceToDevice = 3, cudaMemcpyDefault = 4 };

constexpr size_t TN_REF_GUARD_BYTES = size_t(16) << 20;

template <typename T>
inline cudaError_t cudaMallocAsync(T** p, size_t bytes, cudaStream_t) {
    void* q = std::calloc(bytes + TN_REF_GUARD_BYTES, 1);
    if (!q) return 2;
    *p = static_cast<T*>(q);
    return cudaSuccess;
}
template <typename T>
inline cudaError_t cudaMalloc(T** p, size_t bytes) { return cudaMallocAsync(p, bytes, nullptr); }
inline cudaError_t cudaFreeAsync(void* p, cudaStream_t) { std::free(p); return cudaSuccess; }
inline cudaError_t cudaFree(void* p) { std::free(p); return cudaSuccess; }
inline cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t) { std::memset(p, v, n); return cudaSuccess; }
inline cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) {
    std::memcpy(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { std::memcpy(d, s, n); return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline const char* cudaGetErrorString(cudaError_t) { return "host stand-in error"; }
