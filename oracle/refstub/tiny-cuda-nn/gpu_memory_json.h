// Host stand-in (oracle/_ref build): see gpu_memory.h.
#pragma once
#include <tiny-cuda-nn/gpu_memory.h>
