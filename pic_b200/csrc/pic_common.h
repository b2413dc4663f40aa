// pic_common.h -- definitions shared by the host code, the CUDA kernels and
// the CPU oracle (plain C compatible where the oracle needs it).
#ifndef PIC_COMMON_H
#define PIC_COMMON_H

#include <stdint.h>

#if defined(__CUDACC__)
#define PIC_HD __host__ __device__ __forceinline__
#else
#define PIC_HD static inline
#endif

/* Physical constants of MCC_jw/code/base/Constants.f90:3-15. */
#define PIC_KB 1.3807e-23
#define PIC_QE 1.6022e-19
#define PIC_ME 9.1095e-31
#define PIC_AMU 1.660539040e-27
#define PIC_EPS0 8.8542e-12
#define PIC_JTOEV 1.6022e-19
#define PIC_EVTOK 11605.0
#define PIC_MINREAL 1.0e-15
#define PIC_PI 3.141592653589793238

/* Fixed-point scales of the deposit: charge weight 2^-40 per unit, energy
 * weight*eV 2^-32 per unit.  Both accumulate in int64, so the node sums are
 * independent of particle order. */
#define PIC_Q_SCALE 1099511627776.0 /* 2^40 */
#define PIC_E_SCALE 4294967296.0    /* 2^32 */

/* Shape of every deterministic reduction (dot products, norms): blocks of
 * PIC_RED_THREADS threads, each thread summing PIC_RED_ITEMS strided items
 * sequentially, an xor-butterfly over the 32 lanes of a warp, then the warp
 * sums in order.  The oracle repeats this order exactly. */
#define PIC_RED_THREADS 256
#define PIC_RED_ITEMS 4
#define PIC_RED_CHUNK (PIC_RED_THREADS * PIC_RED_ITEMS)

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11).  Counter-based: the random numbers of a particle
 * are a pure function of (seed, particle id, step, purpose), so the GPU and
 * the oracle draw identical numbers in any execution order. */
typedef struct pic_u32x4 {
  uint32_t v[4];
} pic_u32x4;

PIC_HD void pic_mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

PIC_HD pic_u32x4 pic_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                            uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    pic_mulhilo32(M0, c0, &hi0, &lo0);
    pic_mulhilo32(M1, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  pic_u32x4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

/* Uniform double in [0, 1) with 53 random bits from two 32-bit words. */
PIC_HD double pic_u01(uint32_t a, uint32_t b) {
  uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

/* Purposes (third counter word, high byte) of the MCC draws. */
#define PIC_RNG_SELECT 1u   /* round keys of the null-collision selection */
#define PIC_RNG_RESIDUE 2u  /* Bernoulli residue of N_coll                 */
#define PIC_RNG_COLLIDE 3u  /* draws of one collision (blocks of 4)        */
#define PIC_RNG_LOAD 4u     /* particle loader                             */

#endif /* PIC_COMMON_H */
