/*
 * oracle/philox_ref.h -- TEST INFRASTRUCTURE (the oracle).
 *
 * CPU statement of the counter-based random stream that the GPU transport
 * kernel draws, written from the published Philox4x32-10 algorithm
 * (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11): ten rounds of two 32x32->64 multiplies with the multipliers
 * 0xD2511F53 / 0xCD9E8D57 and a Weyl key schedule 0x9E3779B9 / 0xBB67AE85.
 *
 * Stream contract (shared with the product kernel; both sides must agree):
 *   key      = (seed & 0xffffffff, seed >> 32)
 *   counter  = (block, 0, photon & 0xffffffff, photon >> 32)
 *   "u53"    2 draws per block: w0 = x1:x0, w1 = x3:x2 (64-bit),
 *            u = (2*(w >> 12) + 1) * 2^-53, an odd multiple of 2^-53 in (0,1)
 *   "u24"    4 draws per block: u_i = (2*(x_i >> 9) + 1) * 2^-24, exactly
 *            representable in binary32, in (0,1)
 * Draw j of a photon lives in block j/2 (u53) or j/4 (u24).  The reference's
 * own uniform() (src/rng.cpp:12-16) is (x >> 11) * 2^-53 in [0,1); the stream
 * above is a documented replacement, never zero, so -log(u) stays finite.
 */
#ifndef LMC_ORACLE_PHILOX_REF_H
#define LMC_ORACLE_PHILOX_REF_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LMC_STREAM_U53 = 0, LMC_STREAM_U24 = 1 };

static inline void lmc_ref_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                         uint32_t out[4])
{
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Draw number `draw` of photon `photon` under `seed`, in the given format. */
static inline double lmc_ref_stream_uniform(uint64_t seed, uint64_t photon, uint64_t draw,
                                            int format)
{
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t x[4];
  if (format == LMC_STREAM_U24) {
    const uint32_t ctr[4] = {(uint32_t)(draw >> 2), 0u, (uint32_t)photon, (uint32_t)(photon >> 32)};
    lmc_ref_philox4x32_10(ctr, key, x);
    const uint32_t w = x[draw & 3u];
    return (double)(2u * (w >> 9) + 1u) * (1.0 / 16777216.0);
  }
  const uint32_t ctr[4] = {(uint32_t)(draw >> 1), 0u, (uint32_t)photon, (uint32_t)(photon >> 32)};
  lmc_ref_philox4x32_10(ctr, key, x);
  const uint64_t w = (draw & 1u) ? (((uint64_t)x[3] << 32) | x[2]) : (((uint64_t)x[1] << 32) | x[0]);
  return (double)(2u * (w >> 12) + 1u) * (1.0 / 9007199254740992.0);
}

#ifdef __cplusplus
}
#endif
#endif
