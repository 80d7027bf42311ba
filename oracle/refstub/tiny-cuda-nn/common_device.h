// Host stand-in (oracle/_ref build): everything the reference uses from tiny-cuda-nn's device
// header is in the stand-in common.h.
#pragma once
#include <tiny-cuda-nn/common.h>
