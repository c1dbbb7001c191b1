/* vl/random.h -- VLFeat's random number generator (MT19937) on the host.
 *
 * Same state layout, functions and outputs as the reference's vl/random.h
 * (VLFeat 0.9.21): the Mersenne Twister MT19937 of Matsumoto and Nishimura,
 * seeded on first use with 5489 when no seed was set (vl/random.c:202-203).
 * Each host thread owns one generator (vl_get_rand, vl/generic.h:110); the
 * Rand initialisation of VlGMM draws from it exactly as the reference does. */
#ifndef VL_RANDOM_H
#define VL_RANDOM_H

#include "host.h"

/* Generator state, vl/random.h:20-24. */
typedef struct _VlRand {
  vl_uint32 mt[624];
  vl_uint32 mti;
} VlRand;

/* vl/random.h:29-33. */
VL_EXPORT void vl_rand_init(VlRand *self);
VL_EXPORT void vl_rand_seed(VlRand *self, vl_uint32 s);
VL_EXPORT void vl_rand_seed_by_array(VlRand *self, vl_uint32 const key[], vl_size keySize);

/* vl/random.h:41, 50. */
VL_EXPORT vl_uint32 vl_rand_uint32(VlRand *self);
VL_EXPORT void vl_rand_permute_indexes(VlRand *self, vl_index *array, vl_size size);

/* The derived draws, defined inline like the reference (vl/random.h:64-160). */

/* Index in [0, range-1]: a 32-bit draw modulo range (64-bit above 2^32). */
VL_INLINE vl_uint64 vl_rand_uint64(VlRand *self)
{
  vl_uint64 hi = vl_rand_uint32(self);
  vl_uint64 lo = vl_rand_uint32(self);
  return (hi << 32) | lo;
}

VL_INLINE vl_uindex vl_rand_uindex(VlRand *self, vl_uindex range)
{
  if (range <= 0xffffffff) return (vl_uindex)(vl_rand_uint32(self) % (vl_uint32)range);
  return (vl_uindex)(vl_rand_uint64(self) % range);
}

VL_INLINE vl_int64 vl_rand_int63(VlRand *self) { return (vl_int64)(vl_rand_uint64(self) >> 1); }
VL_INLINE vl_int32 vl_rand_int31(VlRand *self) { return (vl_int32)(vl_rand_uint32(self) >> 1); }

/* [0, 1]: the draw divided by 2^32 - 1. */
VL_INLINE double vl_rand_real1(VlRand *self) { return vl_rand_uint32(self) * (1.0 / 4294967295.0); }
/* [0, 1): divided by 2^32. */
VL_INLINE double vl_rand_real2(VlRand *self) { return vl_rand_uint32(self) * (1.0 / 4294967296.0); }
/* (0, 1): (draw + 1/2) / 2^32. */
VL_INLINE double vl_rand_real3(VlRand *self)
{
  return (((double)vl_rand_uint32(self)) + 0.5) * (1.0 / 4294967296.0);
}
/* [0, 1) with 53-bit resolution from two draws. */
VL_INLINE double vl_rand_res53(VlRand *self)
{
  vl_uint32 a = vl_rand_uint32(self) >> 5, b = vl_rand_uint32(self) >> 6;
  return (a * 67108864.0 + b) * (1.0 / 9007199254740992.0);
}

#endif /* VL_RANDOM_H */
