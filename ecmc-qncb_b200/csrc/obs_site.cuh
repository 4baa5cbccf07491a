// obs_site.cuh — per-site plaquette and clover (q, e) contributions, shared by the
// single-lattice and batched reductions.
//
// References: mean_plaquette_local (src/observables/observables_mpi.cpp:8-29),
// clover_site and local_q_e_clover (observables_mpi.cpp:61-107).
#pragma once
#include "layout.cuh"

namespace qcb {

// ---- plaquette ------------------------------------------------------------------------
template <typename F, typename R>
__device__ __forceinline__ R site_plaquette(const Geom& g, const F& f, const Coord& x, int par,
                                            uint32_t i) {
  const int opp = par ^ 1;
  R sum = 0;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const m3<R> Umu = f.template load<R>(mu, par, i);
    const uint32_t xmu = cb_index(nb_full(g, x, mu, +1));
#pragma unroll
    for (int nu = mu + 1; nu < 4; ++nu) {
      const uint32_t xnu = cb_index(nb_full(g, x, nu, +1));
      // T1 = U_mu(x) U_nu(x+mu), T2 = U_nu(x) U_mu(x+nu); Re tr(T1 T2^dag)
      m3<R> T1 = mul_nn(Umu, f.template load<R>(nu, opp, xmu));
      m3<R> T2 = mul_nn(f.template load<R>(nu, par, i), f.template load<R>(mu, opp, xnu));
      sum += re_tr_na(T1, T2);
    }
  }
  return sum * R(1.0 / 3.0);
}

// ---- clover Q and E -------------------------------------------------------------------
// Clover sum C_{mu nu}(x) of the four leaves, in the reference's leaf order
// (observables_mpi.cpp:70-80).
template <typename LF, typename R, int MU, int NU>
__device__ __forceinline__ m3<R> clover_F(const Geom& g, const LF& f, const Coord& x, int par,
                                          uint32_t i) {
  const int opp = par ^ 1;
  const uint32_t xpmu = cb_index(nb_full(g, x, MU, +1));            // opp
  const uint32_t xpnu = cb_index(nb_full(g, x, NU, +1));            // opp
  const uint32_t xmmu = cb_index(nb_full(g, x, MU, -1));            // opp
  const uint32_t xmnu = cb_index(nb_full(g, x, NU, -1));            // opp
  const uint32_t xmmupnu = cb_index(nb2_full(g, x, MU, -1, NU, +1));  // par
  const uint32_t xmmumnu = cb_index(nb2_full(g, x, MU, -1, NU, -1));  // par
  const uint32_t xpmumnu = cb_index(nb2_full(g, x, MU, +1, NU, -1));  // par
  const m3<R> Umu_x = f.template load<R>(MU, par, i);
  const m3<R> Unu_x = f.template load<R>(NU, par, i);
  m3<R> C;
  {
    // U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
    m3<R> T1 = mul_nn(Umu_x, f.template load<R>(NU, opp, xpmu));
    m3<R> T2 = mul_nn(Unu_x, f.template load<R>(MU, opp, xpnu));
    C = mul_na(T1, T2);
  }
  const m3<R> Umu_xmmu = f.template load<R>(MU, opp, xmmu);
  {
    // U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)
    m3<R> T1 = mul_na(Unu_x, f.template load<R>(MU, par, xmmupnu));
    m3<R> T2 = mul_an(f.template load<R>(NU, opp, xmmu), Umu_xmmu);
    acc_nn(C, T1, T2);
  }
  const m3<R> Unu_xmnu = f.template load<R>(NU, opp, xmnu);
  {
    // U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu)
    m3<R> T1 = mul_aa(Umu_xmmu, f.template load<R>(NU, par, xmmumnu));
    m3<R> T2 = mul_nn(f.template load<R>(MU, par, xmmumnu), Unu_xmnu);
    acc_nn(C, T1, T2);
  }
  {
    // U_nu(x-nu)^dag U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^dag
    m3<R> T1 = mul_an(Unu_xmnu, f.template load<R>(MU, opp, xmnu));
    m3<R> T2 = mul_na(f.template load<R>(NU, par, xpmumnu), Umu_x);
    acc_nn(C, T1, T2);
  }
  // F = (C - C^dag) / 8
  m3<R> Fm;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      Fm.e[a][b] = mk<R>(R(0.125) * (C.e[a][b].re - C.e[b][a].re), R(0.125) * (C.e[a][b].im + C.e[b][a].im));
  return Fm;
}

template <typename R>
__device__ __forceinline__ R sqnorm(const m3<R>& a) {
  R s = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s = fma(a.e[i][j].re, a.e[i][j].re, fma(a.e[i][j].im, a.e[i][j].im, s));
  return s;
}

// q and e contributions of one pair of planes, sgn * Re tr(F_{M1 N1} F_{M2 N2}) and the two
// squared norms.  Not inlined: each pair is a separate register allocation, which keeps
// the six clover evaluations of a site from being interleaved into one block that spills.
template <typename F, typename R, int M1, int N1, int M2, int N2>
__device__ __noinline__ void pair_qe(Geom g, F f, Coord x, int par, uint32_t i, R sgn, R* q, R* e) {
  const m3<R> Fa = clover_F<F, R, M1, N1>(g, f, x, par, i);
  const m3<R> Fb = clover_F<F, R, M2, N2>(g, f, x, par, i);
  *q += sgn * re_tr_nn(Fa, Fb);
  *e += sqnorm(Fa) + sqnorm(Fb);
}

// Per-site unscaled clover sums: q_site = tr F01 F23 - tr F02 F13 + tr F03 F12 and
// e_site = sum_{mu<nu} |F_mu nu|^2 (the 1/(4 pi^2) and 1/2 are applied to the totals).
template <typename F, typename R>
__device__ __forceinline__ void site_qe(const Geom& g, const F& f, const Coord& x, int par, uint32_t i, R* q, R* e) {
  pair_qe<F, R, 0, 1, 2, 3>(g, f, x, par, i, R(1), q, e);
  pair_qe<F, R, 0, 2, 1, 3>(g, f, x, par, i, R(-1), q, e);
  pair_qe<F, R, 0, 3, 1, 2>(g, f, x, par, i, R(1), q, e);
}

}  // namespace qcb
