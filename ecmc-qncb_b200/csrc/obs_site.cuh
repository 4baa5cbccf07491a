// obs_site.cuh — per-site plaquette and clover (q, e) contributions, shared by the
// single-lattice and batched reductions.
//
// References: mean_plaquette_local (src/observables/observables_mpi.cpp:8-29),
// clover_site and local_q_e_clover (observables_mpi.cpp:61-107).
#pragma once
#include "staple.cuh"

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

// Sum of Re tr P_ij(x) over the spatial planes i < j < 3 (no 1/3), for the measuring
// heatbath pass.
template <typename F, typename R>
__device__ __forceinline__ R site_plaquette_spatial(const Geom& g, const F& f, const Coord& x, int par,
                                                    uint32_t i) {
  const int opp = par ^ 1;
  R sum = 0;
#pragma unroll
  for (int mu = 0; mu < 2; ++mu) {
    const m3<R> Umu = f.template load<R>(mu, par, i);
    const uint32_t xmu = cb_index(nb_full(g, x, mu, +1));
#pragma unroll
    for (int nu = mu + 1; nu < 3; ++nu) {
      const uint32_t xnu = cb_index(nb_full(g, x, nu, +1));
      m3<R> T1 = mul_nn(Umu, f.template load<R>(nu, opp, xmu));
      m3<R> T2 = mul_nn(f.template load<R>(nu, par, i), f.template load<R>(mu, opp, xnu));
      sum += re_tr_na(T1, T2);
    }
  }
  return sum;
}

// ---- clover Q and E -------------------------------------------------------------------
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
  return fma(R(-2), t, -s);
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
  return fma(R(2), t, s);
}

// Product helpers for the clover leaves.  With 12-real storage a product of two SU(3)
// matrices is formed from the stored rows 0 and 1 of its first factor (no reconstruction of
// that link) and its row 2 is rebuilt by the cross product; with 18-real storage the full
// product is formed.
template <typename LF, typename R>
__device__ __forceinline__ m3<R> lead(const LF& f, int mu, int par, uint32_t i) {
  if constexpr (LF::NREAL == 12) return f.template load_rows01<R>(mu, par, i);
  else return f.template load<R>(mu, par, i);
}
template <typename LF, typename R>
__device__ __forceinline__ m3<R> prod_nn(const m3<R>& a, const m3<R>& b) {
  if constexpr (LF::NREAL == 12) {
    m3<R> c = mul_nn_rows01(a, b);
    reconstruct_row2(c);
    return c;
  } else {
    return mul_nn(a, b);
  }
}
template <typename LF, typename R>
__device__ __forceinline__ m3<R> prod_na(const m3<R>& a, const m3<R>& b) {
  if constexpr (LF::NREAL == 12) {
    m3<R> c = mul_na_rows01(a, b);
    reconstruct_row2(c);
    return c;
  } else {
    return mul_na(a, b);
  }
}

// Clover plane (mu, nu) at site x with the plane chosen at run time, so that the six planes
// of a site run through one copy of this code (one body in the instruction cache).  The four
// leaves, in the reference's order (observables_mpi.cpp:70-80), each grouped as products of
// SU(3) matrices whose first factor is a stored link:
//   L1 = [U_mu(x) U_nu(x+mu)] [U_nu(x) U_mu(x+nu)]^dag
//   L2 = U_nu(x) [U_nu(x-mu) U_mu(x-mu+nu)]^dag U_mu(x-mu)
//   L3 = [U_nu(x-mu-nu) U_mu(x-mu)]^dag [U_mu(x-mu-nu) U_nu(x-nu)]
//   L4 = U_nu(x-nu)^dag [U_mu(x-nu) U_nu(x+mu-nu)] U_mu(x)^dag
// xs is the full index of x; o its neighbour offsets.
template <typename LF, typename R>
__device__ __noinline__ void clover_plane_rt(LF f, uint32_t xs, NbOff o, int mu, int nu, int par, uint32_t i,
                                             ah9<R>* out) {
  const int opp = par ^ 1;
  const int32_t upmu = sel4(o.up, mu), upnu = sel4(o.up, nu), dnmu = sel4(o.dn, mu), dnnu = sel4(o.dn, nu);
  const int32_t s = (int32_t)xs;
  const uint32_t xpmu = (uint32_t)(s + upmu) >> 1, xpnu = (uint32_t)(s + upnu) >> 1;       // opp
  const uint32_t xmmu = (uint32_t)(s + dnmu) >> 1, xmnu = (uint32_t)(s + dnnu) >> 1;       // opp
  const uint32_t xmmupnu = (uint32_t)(s + dnmu + upnu) >> 1;                               // par
  const uint32_t xmmumnu = (uint32_t)(s + dnmu + dnnu) >> 1;                               // par
  const uint32_t xpmumnu = (uint32_t)(s + upmu + dnnu) >> 1;                               // par
  m3<R> C;
  {
    const m3<R> P1 = prod_nn<LF, R>(lead<LF, R>(f, mu, par, i), f.template load<R>(nu, opp, xpmu));
    const m3<R> P2 = prod_nn<LF, R>(lead<LF, R>(f, nu, par, i), f.template load<R>(mu, opp, xpnu));
    C = mul_na(P1, P2);
  }
  {
    const m3<R> S = prod_nn<LF, R>(lead<LF, R>(f, nu, opp, xmmu), f.template load<R>(mu, par, xmmupnu));
    const m3<R> T = prod_na<LF, R>(lead<LF, R>(f, nu, par, i), S);
    acc_nn(C, T, f.template load<R>(mu, opp, xmmu));
  }
  {
    const m3<R> S1 = prod_nn<LF, R>(lead<LF, R>(f, nu, par, xmmumnu), f.template load<R>(mu, opp, xmmu));
    const m3<R> S2 = prod_nn<LF, R>(lead<LF, R>(f, mu, par, xmmumnu), f.template load<R>(nu, opp, xmnu));
    acc_an(C, S1, S2);
  }
  {
    // rows 0 and 1 of S suffice for T = S U_mu(x)^dag
    m3<R> S;
    if constexpr (LF::NREAL == 12)
      S = mul_nn_rows01(f.template load_rows01<R>(mu, opp, xmnu), f.template load<R>(nu, par, xpmumnu));
    else
      S = mul_nn(f.template load<R>(mu, opp, xmnu), f.template load<R>(nu, par, xpmumnu));
    const m3<R> T = prod_na<LF, R>(S, f.template load<R>(mu, par, i));
    acc_an(C, f.template load<R>(nu, opp, xmnu), T);
  }
  *out = ah_from_clover(C);
}

// Per-site unscaled clover sums: q_site = tr F01 F23 - tr F02 F13 + tr F03 F12 and
// e_site = sum_{mu<nu} |F_mu nu|^2 (the 1/(4 pi^2) and 1/2 are applied to the totals).
template <typename F, typename R>
__device__ __forceinline__ void site_qe(const Geom& g, const F& f, const Coord& x, int par, uint32_t i, R* q, R* e) {
  const NbOff o = nb_offsets(g, x);
  R qs = 0, es = 0;
#pragma unroll 1
  for (int p = 0; p < 3; ++p) {
    // pairs (01, 23), (02, 13), (03, 12) with signs +, -, +
    const int nu1 = p + 1;
    const int mu2 = (p == 0) ? 2 : 1;
    const int nu2 = (p == 2) ? 2 : 3;
    ah9<R> a, b;
    clover_plane_rt<F, R>(f, x.s, o, 0, nu1, par, i, &a);
    clover_plane_rt<F, R>(f, x.s, o, mu2, nu2, par, i, &b);
    const R t = re_tr_ah(a, b);
    qs += (p == 1) ? -t : t;
    es += sqnorm_ah(a) + sqnorm_ah(b);
  }
  *q += qs;
  *e += es;
}

}  // namespace qcb
