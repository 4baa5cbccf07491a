// staple.cuh — staple sum of one link, shared by the heatbath and flow kernels.
//
// Reference: GaugeField::compute_staple (src/gauge/GaugeField.cpp:74-97):
//   A = sum_{nu != mu} [ U_nu(x+mu) (U_nu(x) U_mu(x+nu))^dagger
//                       + (U_mu(x-nu) U_nu(x+mu-nu))^dagger U_nu(x-nu) ]
// MU is a template parameter so that every coordinate index is a compile-time constant
// (no local-memory arrays).  Link parity bookkeeping: x has parity `par`; x+-nu and
// x+mu have parity 1-par; x+mu-nu has parity `par`.
#pragma once
#include "layout.cuh"

namespace qcb {

// Neighbour offsets of site x in every direction: up[d] = full-index step to x + d,
// dn[d] = step to x - d (periodic).
struct NbOff {
  int32_t up[4], dn[4];
};
__device__ __forceinline__ NbOff nb_offsets(const Geom& g, const Coord& x) {
  NbOff o;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    o.up[d] = (x.c[d] + 1 == g.L[d]) ? (1 - g.L[d]) * g.str[d] : g.str[d];
    o.dn[d] = (x.c[d] == 0) ? (g.L[d] - 1) * g.str[d] : -g.str[d];
  }
  return o;
}
__device__ __forceinline__ int32_t sel4(const int32_t* v, int k) {
  return k == 0 ? v[0] : (k == 1 ? v[1] : (k == 2 ? v[2] : v[3]));
}

// The two staple terms of one plane (mu, nu), added to A.  Site indices: i = x (parity
// par); ixmu = x+mu, ixnu = x+nu, ixmnu = x-nu (parity opp); ixmunu = x+mu-nu (parity par).
// With 12-real storage each product of links is an SU(3) matrix whose third row follows
// from its first two, so only rows 0 and 1 of a product are computed and row 2 is rebuilt by
// the cross product.  Forward: rows 0, 1 of T = U_nu(x+mu) U_mu(x+nu)^dag (from the stored
// rows of U_nu(x+mu)), then rows 0, 1 of W = T U_nu(x)^dag (from rows 0, 1 of T: T's row 2
// is never formed), W's row 2 rebuilt, A += W.  Backward: P = U_mu(x-nu) U_nu(x+mu-nu) as
// rows 0, 1 plus the rebuilt row 2, A += P^dag U_nu(x-nu) (this product needs every row of
// both factors).
template <typename F, typename R>
__device__ __forceinline__ void staple_terms(m3<R>& A, const F& f, int nu, int mu, int par, int opp, uint32_t i,
                                             uint32_t ixmu, uint32_t ixnu, uint32_t ixmunu, uint32_t ixmnu) {
  if constexpr (F::NREAL == 12) {
    {
      const m3<R> U0 = f.template load_rows01<R>(nu, opp, ixmu);
      const m3<R> U1 = f.template load<R>(mu, opp, ixnu);
      const m3<R> T = mul_na_rows01(U0, U1);
      const m3<R> U2 = f.template load<R>(nu, par, i);
      m3<R> W = mul_na_rows01(T, U2);
      reconstruct_row2(W);
      add_m3(A, W);
    }
    {
      const m3<R> V1 = f.template load_rows01<R>(mu, opp, ixmnu);
      const m3<R> V0 = f.template load<R>(nu, par, ixmunu);
      m3<R> P = mul_nn_rows01(V1, V0);
      reconstruct_row2(P);
      const m3<R> V2 = f.template load<R>(nu, opp, ixmnu);
      acc_an(A, P, V2);
    }
  } else {
    {
      // forward: U_nu(x+mu) U_mu(x+nu)^dagger U_nu(x)^dagger
      const m3<R> U0 = f.template load<R>(nu, opp, ixmu);
      const m3<R> U1 = f.template load<R>(mu, opp, ixnu);
      const m3<R> T = mul_na(U0, U1);
      const m3<R> U2 = f.template load<R>(nu, par, i);
      acc_na(A, T, U2);
    }
    {
      // backward: U_nu(x+mu-nu)^dagger U_mu(x-nu)^dagger U_nu(x-nu)
      const m3<R> V0 = f.template load<R>(nu, par, ixmunu);
      const m3<R> V1 = f.template load<R>(mu, opp, ixmnu);
      const m3<R> T = mul_aa(V0, V1);
      const m3<R> V2 = f.template load<R>(nu, opp, ixmnu);
      acc_nn(A, T, V2);
    }
  }
}

template <typename F, typename R, int MU>
__device__ __forceinline__ m3<R> staple_sum(const Geom& g, const F& f, const Coord& x, int par, uint32_t i) {
  m3<R> A;
  set_zero(A);
  const int opp = par ^ 1;
  const uint32_t xmu = nb_full(g, x, MU, +1);
#pragma unroll
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == MU) continue;
    const uint32_t xnu = nb_full(g, x, nu, +1);
    const uint32_t xmunu = nb2_full(g, x, MU, +1, nu, -1);
    const uint32_t xmnu = nb_full(g, x, nu, -1);
    staple_terms<F, R>(A, f, nu, MU, par, opp, i, cb_index(xmu), cb_index(xnu), cb_index(xmunu), cb_index(xmnu));
  }
  return A;
}

// Same staple sum with the planes in a loop that is not unrolled: nu is a run-time value, so
// the plane body appears once in the code (a third of the unrolled size).  Measured on 32^4
// FP32 12-real: heatbath pass 76.6 -> 74.5 us, RK3 step 1.364 -> 1.296 ms (the unrolled planes
// stall on instruction fetch); FP64 18-real is slower with it (pass 200.8 -> 212.0 us), so the
// FP64 kernels keep the unrolled planes.
template <typename F, typename R, int MU>
__device__ __forceinline__ m3<R> staple_sum_loop(const Geom& g, const F& f, const Coord& x, int par, uint32_t i) {
  m3<R> A;
  set_zero(A);
  const int opp = par ^ 1;
  const NbOff o = nb_offsets(g, x);
  const uint32_t xmu = (uint32_t)((int32_t)x.s + o.up[MU]);
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const int nu = k + (k >= MU);
    const int32_t upnu = sel4(o.up, nu), dnnu = sel4(o.dn, nu);
    const uint32_t xnu = (uint32_t)((int32_t)x.s + upnu);
    const uint32_t xmunu = (uint32_t)((int32_t)x.s + o.up[MU] + dnnu);
    const uint32_t xmnu = (uint32_t)((int32_t)x.s + dnnu);
    staple_terms<F, R>(A, f, nu, MU, par, opp, i, cb_index(xmu), cb_index(xnu), cb_index(xmunu), cb_index(xmnu));
  }
  return A;
}

// The staple of the single-lattice kernels: planes in a loop in FP32, unrolled in FP64.
template <typename F, typename R, int MU>
__device__ __forceinline__ m3<R> staple_sum_best(const Geom& g, const F& f, const Coord& x, int par, uint32_t i) {
  if constexpr (is_fp32<R>::value)
    return staple_sum_loop<F, R, MU>(g, f, x, par, i);
  else
    return staple_sum<F, R, MU>(g, f, x, par, i);
}

// Same staple sum with the direction mu known only at run time: one code path for all
// four directions (a quarter of the code of the four MU instantiations), for kernels in
// which neighbouring blocks handle different directions.
template <typename F, typename R>
__device__ __forceinline__ m3<R> staple_sum_rt(const Geom& g, const F& f, const Coord& x, int mu, int par,
                                               uint32_t i) {
  m3<R> A;
  set_zero(A);
  const int opp = par ^ 1;
  const NbOff o = nb_offsets(g, x);
  const int32_t upmu = sel4(o.up, mu);
  const uint32_t xmu = (uint32_t)((int32_t)x.s + upmu);
  if constexpr (is_fp32<R>::value) {
    // FP32: the planes in a loop that is not unrolled (one plane body, as staple_sum_loop)
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
      const int nu = k + (k >= mu);
      const int32_t upnu = sel4(o.up, nu), dnnu = sel4(o.dn, nu);
      const uint32_t xnu = (uint32_t)((int32_t)x.s + upnu);
      const uint32_t xmunu = (uint32_t)((int32_t)x.s + upmu + dnnu);
      const uint32_t xmnu = (uint32_t)((int32_t)x.s + dnnu);
      staple_terms<F, R>(A, f, nu, mu, par, opp, i, cb_index(xmu), cb_index(xnu), cb_index(xmunu), cb_index(xmnu));
    }
  } else {
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
      if (nu == mu) continue;
      const uint32_t xnu = (uint32_t)((int32_t)x.s + o.up[nu]);
      const uint32_t xmunu = (uint32_t)((int32_t)x.s + upmu + o.dn[nu]);
      const uint32_t xmnu = (uint32_t)((int32_t)x.s + o.dn[nu]);
      staple_terms<F, R>(A, f, nu, mu, par, opp, i, cb_index(xmu), cb_index(xnu), cb_index(xmunu), cb_index(xmnu));
    }
  }
  return A;
}

}  // namespace qcb
