// Host stand-in (oracle/_ref build): the reference's bit-count header includes thrust's reduce
// for a host-side helper the oracle does not call (it sums the per-word counts itself).
#pragma once
#include <cstdint>
namespace thrust {
template <typename T>
struct plus {
    T operator()(const T& a, const T& b) const { return a + b; }
};
}  // namespace thrust
