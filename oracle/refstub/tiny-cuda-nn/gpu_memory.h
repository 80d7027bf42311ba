// Host stand-in (oracle/_ref build): the reference's Adam class names tiny-cuda-nn's device
// buffer type in members the oracle never instantiates; only ngp_adam_step is run.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <tiny-cuda-nn/common.h>
namespace tcnn {
template <typename T>
class GPUMemory {
public:
    void resize(size_t n) { v_.resize(n); }
    void memset(int) {}
    T* data() { return v_.data(); }
    size_t size() const { return v_.size(); }

private:
    std::vector<T> v_;
};
}  // namespace tcnn
