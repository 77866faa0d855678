/*
 * philox.h — Philox-4x32-10 counter-based RNG for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. Restated from the published method: J. K. Salmon,
 * M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11. Round function: two 32x32->64 multiplies by 0xD2511F53 and 0xCD9E8D57,
 * outputs permuted and xored with the key; the key is bumped by the Weyl constants
 * 0x9E3779B9 and 0xBB67AE85 between rounds; 10 rounds.
 *
 * Stream convention shared with the transport kernel: packet p of wavelength iL in
 * instance `inst` uses counter (k/4, p_lo32, p_hi16 | iL<<16, inst) for its k-th draw
 * and key (seed_lo32, seed_hi32); draw k takes word k%4. A uniform in (0,1] is
 * ((word >> 8) + 1) * 2^-24.
 */
#ifndef ORC_PHILOX_H
#define ORC_PHILOX_H
#include <stdint.h>

static inline void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline double orc_u01(uint32_t w) { return ((double)(w >> 8) + 1.0) * (1.0 / 16777216.0); }

#endif
