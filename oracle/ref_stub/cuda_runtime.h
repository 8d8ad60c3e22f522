/* Empty stand-in for <cuda_runtime.h>: lets the host compiler read the
 * reference's header-only MurmurHash3 (kernels/MurmurHash.cuh) as plain C++
 * when building the known-answer generator in oracle/_ref. */
#pragma once
