/* spiffe_b200_rng.h
 *
 * The project's counter-based uniform generator, used for cathode emission
 * on the host and on the device.  Draw k (k = 1, 2, ...) of the stream seeded
 * with `seed` is the SplitMix64 finaliser (Steele, Lea & Flood, "Fast
 * splittable pseudorandom number generators", OOPSLA 2014; mixing constants of
 * Stafford's variant 13) applied to key + k*0x9E3779B97F4A7C15, keeping the
 * top 53 bits as a double in [0, 1).  Being a pure function of (key, k), any
 * thread can produce any draw, so births are generated in parallel while
 * consuming the stream in the reference's serial order (random_1(1) calls in
 * cathode.c:409, :420, :470, :539).  The reference's own generator lives in
 * the SDDS library, which is not part of its source tree.
 */
#ifndef SPIFFE_B200_RNG_H
#define SPIFFE_B200_RNG_H

#include <stdint.h>

#ifdef __CUDACC__
#define SPIFFE_HD __host__ __device__ __forceinline__
#else
#define SPIFFE_HD static inline
#endif

SPIFFE_HD uint64_t spiffe_rng_mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* stream key of a seed, as random_1(-seed) sets it (cathode.c:90) */
SPIFFE_HD uint64_t spiffe_rng_key(uint64_t seed)
{
  return spiffe_rng_mix64(seed * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL);
}

/* stream key of a seed for the second generator, as random_2(-seed) sets it
 * (emitter.c:63; the surface emitters draw from it) */
SPIFFE_HD uint64_t spiffe_rng_key2(uint64_t seed)
{
  return spiffe_rng_mix64(seed * 0x9E3779B97F4A7C15ULL + 0xD1B54A32D192ED03ULL);
}

/* draw number k >= 1 of the stream */
SPIFFE_HD double spiffe_rng_uniform(uint64_t key, uint64_t k)
{
  return (double)(spiffe_rng_mix64(key + k * 0x9E3779B97F4A7C15ULL) >> 11) * 0x1.0p-53;
}

#endif
