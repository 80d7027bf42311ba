// Host stand-in (oracle/_ref build): the base class of the reference's Adam optimizer. The
// class template is never instantiated by the oracle (it runs ngp_adam_step directly), so only
// the names have to exist.
#pragma once
#include <json/json.hpp>
#include <tiny-cuda-nn/common.h>
namespace tcnn {
using json = nlohmann::json;
template <typename T>
class Optimizer {
public:
    virtual ~Optimizer() = default;
};
template <typename K, typename... Args>
inline void linear_kernel(K, uint32_t, cudaStream_t, uint32_t, Args...) {}
}  // namespace tcnn
