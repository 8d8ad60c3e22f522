/* Forced-include header for building the reference's own `spgemm` driver in
 * oracle/_ref: reads the reference's include/Common.h (found through -I on the
 * reference's include/ directory; `#pragma once` keeps its later inclusions
 * empty), then sets the SM count to the B200's 148. Common.h defines NUM_SM
 * without a guard and uses it only inside other macros, which expand at their
 * use sites, so every use in the reference's kernels and wrappers sees 148. */
#pragma once
#include "Common.h"
#undef NUM_SM
#define NUM_SM 148
