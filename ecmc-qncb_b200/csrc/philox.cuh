// philox.cuh — Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from the paper's
// definition: 10 rounds of the 4x32 S-box with multipliers 0xD2511F53 / 0xCD9E8D57 and
// Weyl key increments 0x9E3779B9 / 0xBB67AE85.
//
// The reference draws from one sequential std::mt19937_64 per MPI rank
// (src/bin/gauge_hb_ncb.cpp:28), so its chain depends on the visiting order.  Here every
// draw is a pure function of (key = seed, counter = (link, sweep, hit/subgroup, draw)),
// so results do not depend on the launch shape or on how lattices are batched.
#pragma once
#include "fp32x.cuh"
#include <stdint.h>

namespace qcb {

struct u32x4 {
  uint32_t v[4];
};

__host__ __device__ __forceinline__ void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

__host__ __device__ __forceinline__ u32x4 philox4x32_10(u32x4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    philox_mulhilo(M0, ctr.v[0], hi0, lo0);
    philox_mulhilo(M1, ctr.v[2], hi1, lo1);
    u32x4 n;
    n.v[0] = hi1 ^ ctr.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ ctr.v[3] ^ k1;
    n.v[3] = lo0;
    ctr = n;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// Uniform in (0, 1) from one 32-bit word.  FP64: (w + 1/2) 2^-32 exactly; FP32: the
// midpoint of the word's top-24-bit bin, within 2^-25 of the FP64 value (so both
// precisions read the same stream).
template <typename R>
__device__ __forceinline__ R u01(uint32_t w);
template <>
__device__ __forceinline__ double u01<double>(uint32_t w) {
  return ((double)w + 0.5) * 2.3283064365386963e-10;
}
template <>
__device__ __forceinline__ float u01<float>(uint32_t w) {
  // ((w >> 8) + 1/2) 2^-24: exact product, one rounding in the add; never 0.
  return fmaf((float)(w >> 8), 5.9604644775390625e-08f, 2.9802322387695312e-08f);
}
template <>
__device__ __forceinline__ f1 u01<f1>(uint32_t w) {
  return f1(u01<float>(w));
}

// Counter domains (word 2 of the counter) for the different consumers of the stream.
enum : uint32_t {
  RNG_DOMAIN_HB = 0x00000000u,       // heatbath: (hit * 4 + subgroup)
  RNG_DOMAIN_HOT = 0x80000000u,      // hot start
  RNG_DOMAIN_GAUGE = 0x90000000u     // random gauge transformation
};

}  // namespace qcb
