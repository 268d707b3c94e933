/*
 * cleo_b200_rng.h — the injected random stream shared by every implementation of the hot path.
 *
 * CLEO draws its collision randoms from a Kokkos Random_XorShift64_Pool whose per-thread state
 * acquisition makes the sequence depend on the backend and thread count
 * (libs/superdrops/kokkosaliases_sd.hpp:60, collisions/collisions.hpp:152-155,
 * collisions/shuffle.cpp:43-49). To compare implementations draw-for-draw, every draw is instead
 * a pure function of (seed, t_sdm, gbxindex, slot):
 *
 *   key  = mix64(mix64(seed + G) ^ (t_sdm << 32 | gbxindex))
 *   u64  = mix64(key + (slot + 1) * G)                 (splitmix64 output step, G = 0x9E37...)
 *   drand(0,1)      = (u64 >> 11) * 2^-53              in [0, 1)
 *   urand(lo, hi)   = lo + floor(u64 * (hi - lo) / 2^64) in [lo, hi)
 *
 * Slot order inside one collision event of a gridbox holding n superdroplets follows the order in
 * which the reference consumes draws on one thread: the Fisher-Yates shuffle takes slots
 * 0 .. n-2 (slot n-1-i for the swap at position i = n-1 .. 1, shuffle.hpp:80-87); pair jj then
 * takes slots (n-1) + 2*jj (phi_coll) and (n-1) + 2*jj + 1 (phi_out) (collisions.hpp:152-155).
 * Further collision events inside the same SDM step continue the slot count.
 */
#ifndef CLEO_B200_RNG_H_
#define CLEO_B200_RNG_H_

#include <stdint.h>

#if defined(__CUDACC__)
#define CLEO_HD __host__ __device__ __forceinline__
#else
#define CLEO_HD static inline
#endif

#define CLEO_RNG_GOLDEN 0x9E3779B97F4A7C15ull

CLEO_HD uint64_t cleo_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

CLEO_HD uint64_t cleo_rng_key(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex) {
  const uint64_t k = cleo_mix64(seed + CLEO_RNG_GOLDEN);
  return cleo_mix64(k ^ (((uint64_t)t_sdm << 32) | (uint64_t)gbxindex));
}

CLEO_HD uint64_t cleo_rng_u64(uint64_t key, uint64_t slot) {
  return cleo_mix64(key + (slot + 1u) * CLEO_RNG_GOLDEN);
}

CLEO_HD double cleo_rng_to_unit(uint64_t u) {
  return (double)(u >> 11) * (1.0 / 9007199254740992.0); /* 2^-53 */
}

CLEO_HD uint64_t cleo_rng_mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

CLEO_HD uint64_t cleo_rng_range(uint64_t u, uint64_t start, uint64_t end) {
  return start + cleo_rng_mulhi(u, end - start);
}

#endif /* CLEO_B200_RNG_H_ */
