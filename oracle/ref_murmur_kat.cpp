// Known-answer generator built FROM THE REFERENCE'S OWN SOURCE — test infrastructure.
//
// Compiles the reference's kernels/MurmurHash.cuh (a header of plain C plus
// __device__/__forceinline__ qualifiers) on the host with those qualifiers
// defined away, and prints "key hash" lines for the keys given on stdin. The
// output pins the oracle's and the GPU kernel's MurmurHash3 to the reference's
// exact function (seed MURMUR3_SEED = 1234, include/Common.h:73).
#define __device__
#define __forceinline__ inline
#include <cstdio>
#include <cstdint>
#include "MurmurHash.cuh"

int main() {
  unsigned long long key;
  while (std::scanf("%llu", &key) == 1) {
    const uint32_t h = somespgemm::murmurHash3_32((index_t)key);
    std::printf("%llu %u\n", key, (unsigned)h);
  }
  return 0;
}
