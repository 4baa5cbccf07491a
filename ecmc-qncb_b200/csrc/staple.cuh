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

template <typename S, int NR, typename R, int MU>
__device__ __forceinline__ m3<R> staple_sum(const Geom& g, const Links<S, NR>& f, const Coord& x, int par,
                                            uint32_t i) {
  m3<R> A;
  set_zero(A);
  const int opp = par ^ 1;
  const uint32_t xmu = nb_full(g, x, MU, +1);
#pragma unroll
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == MU) continue;
    {
      // forward: U_nu(x+mu) U_mu(x+nu)^dagger U_nu(x)^dagger
      const uint32_t xnu = nb_full(g, x, nu, +1);
      m3<R> U0 = f.template load<R>(nu, opp, cb_index(xmu));
      m3<R> U1 = f.template load<R>(MU, opp, cb_index(xnu));
      m3<R> T = mul_na(U0, U1);
      m3<R> U2 = f.template load<R>(nu, par, i);
      acc_na(A, T, U2);
    }
    {
      // backward: U_nu(x+mu-nu)^dagger U_mu(x-nu)^dagger U_nu(x-nu)
      const uint32_t xmunu = nb2_full(g, x, MU, +1, nu, -1);
      const uint32_t xmnu = nb_full(g, x, nu, -1);
      m3<R> V0 = f.template load<R>(nu, par, cb_index(xmunu));
      m3<R> V1 = f.template load<R>(MU, opp, cb_index(xmnu));
      m3<R> T = mul_aa(V0, V1);
      m3<R> V2 = f.template load<R>(nu, opp, cb_index(xmnu));
      acc_nn(A, T, V2);
    }
  }
  return A;
}

}  // namespace qcb
