// Host stand-in (oracle/_ref build): the reference's batch kernels only name the byte type.
#pragma once
typedef unsigned char stbi_uc;
