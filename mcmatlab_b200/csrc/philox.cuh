// Philox-4x32-10 counter-based RNG (device side).
//
// Published method: J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11. Ten rounds of two 32x32->64 multiplies (0xD2511F53,
// 0xCD9E8D57) with the key bumped by the Weyl constants 0x9E3779B9 / 0xBB67AE85.
//
// Stream convention of the transport kernels: packet p (local id within its instance) of
// wavelength iL in batch slot `stream` draws its k-th uniform from counter
// (k/4, p_lo32, p_hi16 | iL<<16, stream) under key (seed_lo32, seed_hi32), word k%4.
// A uniform in (0,1] is ((word >> 8) + 1) * 2^-24, exact in float.
#pragma once
#include <cstdint>

namespace mcb {

struct Philox4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return Philox4{c0, c1, c2, c3};
}

#ifdef __CUDACC__
// One out-of-line copy for the device: the transport inlines its ~60 draw sites, and a Philox
// block inlined at each of them made the kernel large enough to stall on instruction fetch
// (measured 5% more packets/s with this single copy).
static __device__ __noinline__ Philox4 philox_block(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                    uint32_t k1) {
  return philox4x32_10(c0, c1, c2, c3, k0, k1);
}
#endif

__host__ __device__ __forceinline__ float u01_from_word(uint32_t w) {
  return (float)((w >> 8) + 1u) * (1.0f / 16777216.0f);
}

}  // namespace mcb
