// hb_link.cuh — one Cabibbo-Marinari heatbath update of one link (shared by the
// single-lattice pass kernel and the persistent batched kernel).
//
// Reference path: mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:11-34) with
// heatbath::su2_step and generate_su2_kp (src/heatbath/heatbath.cpp:8-44).
#pragma once
#include "philox.cuh"
#include "staple.cuh"

namespace qcb {

// Kennedy-Pendleton attempts per SU(2) draw before the update is skipped and counted
// in the status word (the reference loops without bound, heatbath.cpp:54-66).
constexpr uint32_t KP_CAP = 4096;

// Transcendentals of the KP draw.  FP64: the accurate library functions (parity with the
// FP64 oracle).  FP32: the hardware approximations (relative error ~2^-21 on the ranges used
// here, below the FP32 rounding of the stored links).
template <typename R>
struct KpMath;
template <>
struct KpMath<double> {
  static __device__ __forceinline__ double log(double x) { return ::log(x); }
  // cos(2 pi u)
  static __device__ __forceinline__ double cos2pi(double u) { return cospi(2.0 * u); }
  // sin, cos of 2 pi u
  static __device__ __forceinline__ void sincos2pi(double u, double* s, double* c) { sincospi(2.0 * u, s, c); }
};
template <>
struct KpMath<f1> {
  static __device__ __forceinline__ f1 log(f1 x) { return f1(__logf(x.v)); }
  // 2 pi u = 2 pi (u - 1/2) + pi keeps the hardware argument in (-pi, pi).
  static __device__ __forceinline__ f1 cos2pi(f1 u) {
    return f1(-__cosf(__fmul_rn(6.28318530717958648f, __fsub_rn(u.v, 0.5f))));
  }
  static __device__ __forceinline__ void sincos2pi(f1 u, f1* s, f1* c) {
    float sn, cs;
    __sincosf(__fmul_rn(6.28318530717958648f, __fsub_rn(u.v, 0.5f)), &sn, &cs);
    *s = f1(-sn);
    *c = f1(-cs);
  }
};

// The SU(2) draw of one subgroup update: a0 from the Kennedy-Pendleton density
// sqrt(1-a0^2) exp(alpha a0), then (a1, a2, a3) uniform on the sphere of radius
// sqrt(1-a0^2).  Returns false when the KP attempts hit the cap.  FP64 calls one
// out-of-line copy for the three subgroups (measured 4% faster per pass on 32^4, the
// smaller code); FP32 inlines it (no difference measured).
template <typename R>
__device__ __forceinline__ bool kp_draw_inline(R alpha, uint32_t link, uint32_t sweep, uint32_t hsg, uint32_t k0,
                                               uint32_t k1, R* x) {
  R mhalf_over_alpha = R(-0.5) / alpha;
  // Kennedy-Pendleton draw of a0 with density sqrt(1-a0^2) exp(alpha a0).
  R a0 = 0;
  bool ok = false;
  for (uint32_t att = 0; att < KP_CAP; ++att) {
    u32x4 c;
    c.v[0] = link;
    c.v[1] = sweep;
    c.v[2] = hsg;
    c.v[3] = att;
    u32x4 r = philox4x32_10(c, k0, k1);
    R delta = u01<R>(r.v[0]);
    R r1 = u01<R>(r.v[1]);
    R r2 = u01<R>(r.v[2]);
    R r3 = u01<R>(r.v[3]);
    R cs = KpMath<R>::cos2pi(r2);
    R lam2 = mhalf_over_alpha * fma(cs * cs, KpMath<R>::log(r3), KpMath<R>::log(r1));
    if (delta * delta <= R(1) - lam2) {
      a0 = fma(R(-2), lam2, R(1));
      ok = true;
      break;
    }
  }
  if (!ok) return false;
  // Uniform direction on S^2 for (a1, a2, a3).
  u32x4 c;
  c.v[0] = link;
  c.v[1] = sweep;
  c.v[2] = hsg;
  c.v[3] = 0xFFFFFFFFu;
  u32x4 r = philox4x32_10(c, k0, k1);
  R uphi = u01<R>(r.v[0]);
  R cth = fma(R(2), u01<R>(r.v[1]), R(-1));
  R sth = sqrt(fmax(R(0), fma(-cth, cth, R(1))));
  R rs = sqrt(fmax(R(0), fma(-a0, a0, R(1))));
  R sphi, cphi;
  KpMath<R>::sincos2pi(uphi, &sphi, &cphi);
  x[0] = a0;
  x[1] = rs * sth * cphi;
  x[2] = rs * sth * sphi;
  x[3] = rs * cth;
  return true;
}

template <typename R>
__device__ __noinline__ bool kp_draw(R alpha, uint32_t link, uint32_t sweep, uint32_t hsg, uint32_t k0, uint32_t k1,
                                     R* x) {
  return kp_draw_inline<R>(alpha, link, sweep, hsg, k0, k1, x);
}

// One SU(2) subgroup update of U for subgroup (a, b), block entries of W = U A.
template <typename R, int A_, int B_>
__device__ __forceinline__ bool cm_subgroup(m3<R>& U, const m3<R>& A, R beta, uint32_t link, uint32_t sweep,
                                            uint32_t hsg, uint32_t k0, uint32_t k1) {
  // W_ij = sum_k U_ik A_kj for the four block entries.
  cx<R> Waa = mk<R>(0, 0), Wab = mk<R>(0, 0), Wba = mk<R>(0, 0), Wbb = mk<R>(0, 0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Waa = cfma(U.e[A_][k], A.e[k][A_], Waa);
    Wab = cfma(U.e[A_][k], A.e[k][B_], Wab);
    Wba = cfma(U.e[B_][k], A.e[k][A_], Wba);
    Wbb = cfma(U.e[B_][k], A.e[k][B_], Wbb);
  }
  // Quaternion of [[Waa, Wab], [Wba, Wbb]].
  R w0 = (Waa.re + Wbb.re) * R(0.5);
  R w1 = (Wab.im + Wba.im) * R(0.5);
  R w2 = (Wab.re - Wba.re) * R(0.5);
  R w3 = (Waa.im - Wbb.im) * R(0.5);
  R kk = sqrt(fma(w0, w0, fma(w1, w1, fma(w2, w2, w3 * w3))));
  R ik = R(1) / kk;
  R v0 = w0 * ik, v1 = w1 * ik, v2 = w2 * ik, v3 = w3 * ik;
  R alpha = beta * kk * R(2.0) / R(3.0);
  R x0, x1, x2, x3;
  if constexpr (std::is_same<R, double>::value) {
    R xq[4];
    if (!kp_draw<R>(alpha, link, sweep, hsg, k0, k1, xq)) return false;
    x0 = xq[0], x1 = xq[1], x2 = xq[2], x3 = xq[3];
  } else {
    R xq[4];
    if (!kp_draw_inline<R>(alpha, link, sweep, hsg, k0, k1, xq)) return false;
    x0 = xq[0], x1 = xq[1], x2 = xq[2], x3 = xq[3];
  }
  // r = x * adj(v), adj(v) = (v0, -v1, -v2, -v3).
  R q0 = fma(x0, v0, fma(x1, v1, fma(x2, v2, x3 * v3)));
  R q1 = fma(-x0, v1, fma(x1, v0, fma(-x2, v3, x3 * v2)));
  R q2 = fma(-x0, v2, fma(x1, v3, fma(x2, v0, -(x3 * v1))));
  R q3 = fma(-x0, v3, fma(-x1, v2, fma(x2, v1, x3 * v0)));
  // Embedding: X_aa = q0 + i q3, X_bb = q0 - i q3, X_ab = q2 + i q1, X_ba = -q2 + i q1.
  cx<R> Xaa = mk<R>(q0, q3), Xbb = mk<R>(q0, -q3), Xab = mk<R>(q2, q1), Xba = mk<R>(-q2, q1);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    cx<R> ua = U.e[A_][k], ub = U.e[B_][k];
    U.e[A_][k] = cfma(Xab, ub, Xaa * ua);
    U.e[B_][k] = cfma(Xbb, ub, Xba * ua);
  }
  return true;
}

// n_hits Cabibbo-Marinari hits on link (MU, par, i) of field f, at site x; returns the number
// of KP draws that hit the attempt cap.  With MEAS, *retr receives Re tr(U A) of the updated
// (stored) link U and its staple A: the sum of Re tr of the six plaquettes that contain U.
template <typename F, typename R, int NR, int MU, bool MEAS = false>
__device__ __forceinline__ uint32_t hb_update_at(const Geom& g, const F& f, const Coord& x, int par, uint32_t i,
                                                 R beta, uint32_t k0, uint32_t k1, uint32_t sweep, int n_hits,
                                                 R* retr = nullptr) {
  const m3<R> A = staple_sum_best<F, R, MU>(g, f, x, par, i);
  m3<R> U = f.template load<R>(MU, par, i);
  const uint32_t link = (uint32_t)MU * g.Vg + (x.s + g.soff);
  uint32_t fails = 0;
  for (int h = 0; h < n_hits; ++h) {
    const uint32_t hb = RNG_DOMAIN_HB | ((uint32_t)h << 2);
    fails += !cm_subgroup<R, 0, 1>(U, A, beta, link, sweep, hb | 0u, k0, k1);
    fails += !cm_subgroup<R, 1, 2>(U, A, beta, link, sweep, hb | 1u, k0, k1);
    fails += !cm_subgroup<R, 0, 2>(U, A, beta, link, sweep, hb | 2u, k0, k1);
  }
  if (NR == 12) {
    // Only rows 0 and 1 are stored: keep them orthonormal (in the storage precision) so
    // that the rebuilt row 2 stays the SU(3) completion.
    reunitarize_rows(U);
  }
  f.template store<R>(MU, par, i, U);
  if constexpr (MEAS) *retr = re_tr_nn(U, A);
  return fails;
}

template <typename F, typename R, int NR, int MU>
__device__ __forceinline__ uint32_t hb_update_link(const Geom& g, const F& f, int par, uint32_t i, R beta,
                                                   uint32_t k0, uint32_t k1, uint32_t sweep, int n_hits) {
  const Coord x = cb_coord(g, par, i);
  if (!own_site(g, x.c[3])) return 0;  // halo slice of a slab
  return hb_update_at<F, R, NR, MU>(g, f, x, par, i, beta, k0, k1, sweep, n_hits);
}

// Runtime-direction variant of hb_update_link (one code path for every mu), for the
// persistent batched kernel whose neighbouring blocks handle different directions.
template <typename F, typename R, int NR>
__device__ __forceinline__ uint32_t hb_update_link_rt(const Geom& g, const F& f, int mu, int par, uint32_t i, R beta,
                                                      uint32_t k0, uint32_t k1, uint32_t sweep, int n_hits) {
  const Coord x = cb_coord(g, par, i);
  if (!own_site(g, x.c[3])) return 0;  // halo slice of a slab
  const m3<R> A = staple_sum_rt<F, R>(g, f, x, mu, par, i);
  m3<R> U = f.template load<R>(mu, par, i);
  const uint32_t link = (uint32_t)mu * g.Vg + (x.s + g.soff);
  uint32_t fails = 0;
  for (int h = 0; h < n_hits; ++h) {
    const uint32_t hb = RNG_DOMAIN_HB | ((uint32_t)h << 2);
    fails += !cm_subgroup<R, 0, 1>(U, A, beta, link, sweep, hb | 0u, k0, k1);
    fails += !cm_subgroup<R, 1, 2>(U, A, beta, link, sweep, hb | 1u, k0, k1);
    fails += !cm_subgroup<R, 0, 2>(U, A, beta, link, sweep, hb | 2u, k0, k1);
  }
  if (NR == 12) reunitarize_rows(U);
  f.template store<R>(mu, par, i, U);
  return fails;
}

}  // namespace qcb
