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
__device__ __forceinline__ m3<R> clover_C(const Geom& g, const LF& f, const Coord& x, int par, uint32_t i) {
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
  return C;
}

// Anti-Hermitian 3x3 matrix in 9 reals: F_kk = i d[k], F_ij = o[.] for (i,j) = (0,1),
// (0,2), (1,2), and F_ji = -conj(F_ij).
template <typename R>
struct ah9 {
  R d[3];
  cx<R> o[3];
};

// F_{mu nu} = (C - C^dag) / 8 (observables_mpi.cpp:81-82) in compact form.
template <typename R>
__device__ __forceinline__ ah9<R> ah_from_clover(const m3<R>& C) {
  ah9<R> F;
#pragma unroll
  for (int k = 0; k < 3; ++k) F.d[k] = R(0.25) * C.e[k][k].im;
  F.o[0] = mk<R>(R(0.125) * (C.e[0][1].re - C.e[1][0].re), R(0.125) * (C.e[0][1].im + C.e[1][0].im));
  F.o[1] = mk<R>(R(0.125) * (C.e[0][2].re - C.e[2][0].re), R(0.125) * (C.e[0][2].im + C.e[2][0].im));
  F.o[2] = mk<R>(R(0.125) * (C.e[1][2].re - C.e[2][1].re), R(0.125) * (C.e[1][2].im + C.e[2][1].im));
  return F;
}

// Re tr(A B) of two anti-Hermitian matrices: -sum_k a_k b_k - 2 sum_{i<j} Re(A_ij conj B_ij).
template <typename R>
__device__ __forceinline__ R re_tr_ah(const ah9<R>& A, const ah9<R>& B) {
  R s = 0, t = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    s = fma(A.d[k], B.d[k], s);
    t = fma(A.o[k].re, B.o[k].re, fma(A.o[k].im, B.o[k].im, t));
  }
  return -s - R(2) * t;
}

// |F|^2 = sum_ij |F_ij|^2 = sum_k d_k^2 + 2 sum_{i<j} |F_ij|^2.
template <typename R>
__device__ __forceinline__ R sqnorm_ah(const ah9<R>& A) {
  R s = 0, t = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    s = fma(A.d[k], A.d[k], s);
    t = fma(A.o[k].re, A.o[k].re, fma(A.o[k].im, A.o[k].im, t));
  }
  return s + R(2) * t;
}

// One clover plane.  Not inlined: each plane is its own register allocation (the 9-real
// result crosses the call), which keeps the six planes of a site from being interleaved
// into one block that spills.
template <typename LF, typename R, int MU, int NU>
__device__ __noinline__ void clover_plane(Geom g, LF f, Coord x, int par, uint32_t i, ah9<R>* out) {
  *out = ah_from_clover(clover_C<LF, R, MU, NU>(g, f, x, par, i));
}

// Per-site unscaled clover sums: q_site = tr F01 F23 - tr F02 F13 + tr F03 F12 and
// e_site = sum_{mu<nu} |F_mu nu|^2 (the 1/(4 pi^2) and 1/2 are applied to the totals).
template <typename F, typename R>
__device__ __forceinline__ void site_qe(const Geom& g, const F& f, const Coord& x, int par, uint32_t i, R* q, R* e) {
  ah9<R> a, b;
  clover_plane<F, R, 0, 1>(g, f, x, par, i, &a);
  clover_plane<F, R, 2, 3>(g, f, x, par, i, &b);
  R qs = re_tr_ah(a, b), es = sqnorm_ah(a) + sqnorm_ah(b);
  clover_plane<F, R, 0, 2>(g, f, x, par, i, &a);
  clover_plane<F, R, 1, 3>(g, f, x, par, i, &b);
  qs -= re_tr_ah(a, b);
  es += sqnorm_ah(a) + sqnorm_ah(b);
  clover_plane<F, R, 0, 3>(g, f, x, par, i, &a);
  clover_plane<F, R, 1, 2>(g, f, x, par, i, &b);
  qs += re_tr_ah(a, b);
  es += sqnorm_ah(a) + sqnorm_ah(b);
  *q += qs;
  *e += es;
}

}  // namespace qcb
