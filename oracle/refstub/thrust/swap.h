// Host stand-in (oracle/_ref build): thrust::swap as used by the reference's box slab test.
#pragma once
#include <utility>
namespace thrust {
using std::swap;
}
