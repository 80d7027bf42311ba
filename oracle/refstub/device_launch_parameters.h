// Host stand-in (oracle/_ref build): the launch variables are declared in cuda_runtime.h.
#pragma once
#include <cuda_runtime.h>
