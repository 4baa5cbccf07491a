// flow_link.cuh — one link of one fused Wilson-flow RK3 stage (shared by the
// single-lattice stage kernel and the persistent batched kernel).
//
// Reference: GradientFlow (src/flow/gradient_flow.cpp:15-114):
//   Z   = -P_TA(U A)                         (force, gradient_flow.cpp:15-34)
//   s1: X = eps/4 Z0;                acc = Z0                      (compute_w1, :37-53)
//   s2: X = 8/9 eps Z1 - 17/36 eps Z0; acc = 8/9 Z1 - 17/36 Z0    (compute_w2 + replace_force_0, :56-93)
//   s3: X = 3/4 eps Z2 - eps acc                                   (compute_w3, :96-114)
//   U' = exp(X) U   with Luescher's exponential (src/su3/utils.cpp:145-193)
#pragma once
#include "staple.cuh"

namespace qcb {

// Periodic reunitarisation of FP32 links: after the last stage of each RK3 step the new link
// is converted to FP64, its rows 0 and 1 are orthonormalised (row 2 = conj(r0 x r1)), and it
// is rounded back to FP32.  Without it the FP32 links drift off SU(3) linearly in the number
// of steps; with it the FP32-12 flow of a 32^4 configuration to t = 4 stays within
// |dQ| = 4e-6 and |dE|/E = 6e-8 of the FP64 flow (1e-4 and 2e-5 without), for 3.5% more time
// per step.  FP64 links are left as the reference leaves them.
template <typename R>
__device__ __forceinline__ void flow_reunit(m3<R>& U, int stage) {
  if constexpr (is_fp32<R>::value) {
    if (stage == 3) {
      m3<double> d = convert<double>(U);
      reunitarize_rows(d);
      U = convert<R>(d);
    }
  }
}

// U' = exp(X) U.  12-real storage keeps rows 0 and 1 only (the FP64 re-orthonormalisation of
// stage 3 also reads only those), so row 2 of the product is not formed.
template <typename F, typename R>
__device__ __forceinline__ m3<R> flow_product(const m3<R>& E, const m3<R>& U) {
  if constexpr (F::NREAL == 12)
    return mul_nn_rows01(E, U);
  else
    return mul_nn(E, U);
}

// The stage-dependent part of one link's stage: X from the force Z and the accumulator,
// and the accumulator update.
template <typename ACC, typename R, int MU>
__device__ __forceinline__ alg8<R> flow_x(const ACC& acc, const alg8<R>& Z, R eps, int stage, int par, uint32_t i) {
  alg8<R> X;
  if (stage == 1) {
    const R c = R(0.25) * eps;
#pragma unroll
    for (int k = 0; k < 8; ++k) X.a[k] = c * Z.a[k];
    acc.template store<R>(MU, par, i, Z);
  } else if (stage == 2) {
    const alg8<R> Z0 = acc.template load<R>(MU, par, i);
    const R c1 = R(8.0 / 9.0) * eps, c0 = R(17.0 / 36.0) * eps;
    alg8<R> N;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      X.a[k] = fma(c1, Z.a[k], -(c0 * Z0.a[k]));
      N.a[k] = fma(R(8.0 / 9.0), Z.a[k], -(R(17.0 / 36.0) * Z0.a[k]));
    }
    acc.template store<R>(MU, par, i, N);
  } else {
    const alg8<R> Z0 = acc.template load<R>(MU, par, i);
    const R c1 = R(0.75) * eps;
#pragma unroll
    for (int k = 0; k < 8; ++k) X.a[k] = fma(c1, Z.a[k], -(eps * Z0.a[k]));
  }
  return X;
}

// Stage `stage` (1, 2, 3) of one link U_MU(x), x = (par, i): src -> dst.  Inlined with a
// constant stage in the per-stage kernels; the persistent batch kernel passes it at run time.
template <typename F, typename ACC, typename R, int MU>
__device__ __forceinline__ void flow_link(const Geom& g, const F& src, const F& dst, const ACC& acc, R eps, int stage,
                                          int par, uint32_t i) {
  const Coord x = cb_coord(g, par, i);
  if (!own_site(g, x.c[3])) return;  // halo slice of a slab
  const m3<R> A = staple_sum_best<F, R, MU>(g, src, x, par, i);
  const m3<R> U = src.template load<R>(MU, par, i);
  // Z = P_TA(-U A) = -P_TA(U A)
  alg8<R> Z = proj_ta(mul_nn(U, A));
#pragma unroll
  for (int k = 0; k < 8; ++k) Z.a[k] = -Z.a[k];
  const alg8<R> X = flow_x<ACC, R, MU>(acc, Z, eps, stage, par, i);
  const m3<R> E = exp_su3(X);
  m3<R> Un = flow_product<F, R>(E, U);
  flow_reunit<R>(Un, stage);
  dst.template store<R>(MU, par, i, Un);
}

// Runtime-direction, runtime-stage variant (one code body for every mu and stage).
template <typename F, typename ACC, typename R>
__device__ __forceinline__ void flow_link_rt(const Geom& g, const F& src, const F& dst, const ACC& acc, R eps, int stage,
                                             int mu, int par, uint32_t i) {
  const Coord x = cb_coord(g, par, i);
  if (!own_site(g, x.c[3])) return;  // halo slice of a slab
  const m3<R> A = staple_sum_rt<F, R>(g, src, x, mu, par, i);
  const m3<R> U = src.template load<R>(mu, par, i);
  alg8<R> Z = proj_ta(mul_nn(U, A));
#pragma unroll
  for (int k = 0; k < 8; ++k) Z.a[k] = -Z.a[k];
  alg8<R> X;
  if (stage == 1) {
    const R c = R(0.25) * eps;
#pragma unroll
    for (int k = 0; k < 8; ++k) X.a[k] = c * Z.a[k];
    acc.template store<R>(mu, par, i, Z);
  } else {
    const alg8<R> Z0 = acc.template load<R>(mu, par, i);
    if (stage == 2) {
      const R c1 = R(8.0 / 9.0) * eps, c0 = R(17.0 / 36.0) * eps;
      alg8<R> N;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        X.a[k] = fma(c1, Z.a[k], -(c0 * Z0.a[k]));
        N.a[k] = fma(R(8.0 / 9.0), Z.a[k], -(R(17.0 / 36.0) * Z0.a[k]));
      }
      acc.template store<R>(mu, par, i, N);
    } else {
      const R c1 = R(0.75) * eps;
#pragma unroll
      for (int k = 0; k < 8; ++k) X.a[k] = fma(c1, Z.a[k], -(eps * Z0.a[k]));
    }
  }
  const m3<R> E = exp_su3(X);
  m3<R> Un = flow_product<F, R>(E, U);
  flow_reunit<R>(Un, stage);
  dst.template store<R>(mu, par, i, Un);
}

}  // namespace qcb
