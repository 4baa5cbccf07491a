// k_hb.cu — checkerboarded Cabibbo-Marinari heatbath pass.
//
// Reference path: mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:11-34) with
// heatbath::su2_step and generate_su2_kp (src/heatbath/heatbath.cpp:8-44), applied by
// mpi::heatbathcb::sweep (heatbath_mpi.cpp:37-56) to every non-frozen link in
// lexicographic order.  Here one pass updates all links U_mu(x) with x of one parity:
// their staples only touch links of other directions or of U_mu at the opposite parity,
// so the updates of a pass are independent and run one thread per link.
//
// Per link: staple A once (it does not change between hits), then for each hit and each
// subgroup (0,1), (1,2), (0,2):
//   W = U A restricted to the 2x2 block, w = quaternion of the block (su2_to_quaternion,
//   src/su3/utils.cpp:47-50), k = |w|, v = w/k; x ~ KP(alpha = 2 beta k / 3);
//   r = x v^dagger (utils.cpp:53-63); U <- embed_ij(r) U (utils.cpp:33-44), touching rows
//   i and j only.
#include "dispatch.cuh"
#include "philox.cuh"
#include "staple.cuh"

namespace qcb {

// Kennedy-Pendleton attempts per SU(2) draw before the update is skipped and counted
// in the status word (the reference loops without bound, heatbath.cpp:54-66).
constexpr uint32_t KP_CAP = 4096;

template <typename R>
__device__ __forceinline__ R kp_log(R x);
template <>
__device__ __forceinline__ double kp_log<double>(double x) {
  return log(x);
}
template <>
__device__ __forceinline__ float kp_log<float>(float x) {
  return logf(x);
}

template <typename R>
__device__ __forceinline__ void kp_sincospi(R x, R* s, R* c);
template <>
__device__ __forceinline__ void kp_sincospi<double>(double x, double* s, double* c) {
  sincospi(x, s, c);
}
template <>
__device__ __forceinline__ void kp_sincospi<float>(float x, float* s, float* c) {
  sincospif(x, s, c);
}
template <typename R>
__device__ __forceinline__ R kp_cospi(R x);
template <>
__device__ __forceinline__ double kp_cospi<double>(double x) {
  return cospi(x);
}
template <>
__device__ __forceinline__ float kp_cospi<float>(float x) {
  return cospif(x);
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
  R kk = sqrt(w0 * w0 + w1 * w1 + w2 * w2 + w3 * w3);
  R ik = R(1) / kk;
  R v0 = w0 * ik, v1 = w1 * ik, v2 = w2 * ik, v3 = w3 * ik;
  R alpha = beta * kk * R(2.0) / R(3.0);
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
    R cs = kp_cospi<R>(R(2) * r2);
    R lam2 = mhalf_over_alpha * (kp_log<R>(r1) + cs * cs * kp_log<R>(r3));
    if (delta * delta <= R(1) - lam2) {
      a0 = R(1) - R(2) * lam2;
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
  R cth = R(2) * u01<R>(r.v[1]) - R(1);
  R sth = sqrt(fmax(R(0), R(1) - cth * cth));
  R rs = sqrt(fmax(R(0), R(1) - a0 * a0));
  R sphi, cphi;
  kp_sincospi<R>(R(2) * uphi, &sphi, &cphi);
  R x0 = a0, x1 = rs * sth * cphi, x2 = rs * sth * sphi, x3 = rs * cth;
  // r = x * adj(v), adj(v) = (v0, -v1, -v2, -v3).
  R q0 = x0 * v0 + x1 * v1 + x2 * v2 + x3 * v3;
  R q1 = -x0 * v1 + x1 * v0 - x2 * v3 + x3 * v2;
  R q2 = -x0 * v2 + x1 * v3 + x2 * v0 - x3 * v1;
  R q3 = -x0 * v3 - x1 * v2 + x2 * v1 + x3 * v0;
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

template <typename S, int NR, int MU>
__global__ void __launch_bounds__(128) k_hb_pass(Geom g, Links<S, NR> f, int par, S beta, uint32_t k0,
                                                 uint32_t k1, uint32_t sweep, int n_hits, uint32_t* status) {
  typedef S R;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const Coord x = cb_coord(g, par, i);
  const m3<R> A = staple_sum<S, NR, R, MU>(g, f, x, par, i);
  m3<R> U = f.template load<R>(MU, par, i);
  const uint32_t link = (uint32_t)MU * g.V + x.s;
  uint32_t fails = 0;
  for (int h = 0; h < n_hits; ++h) {
    const uint32_t hb = RNG_DOMAIN_HB | ((uint32_t)h << 2);
    fails += !cm_subgroup<R, 0, 1>(U, A, beta, link, sweep, hb | 0u, k0, k1);
    fails += !cm_subgroup<R, 1, 2>(U, A, beta, link, sweep, hb | 1u, k0, k1);
    fails += !cm_subgroup<R, 0, 2>(U, A, beta, link, sweep, hb | 2u, k0, k1);
  }
  if (NR == 12) {
    // Only rows 0 and 1 are stored: keep them orthonormal so that the rebuilt row 2
    // stays the SU(3) completion.
    m3<double> Ud = convert<double>(U);
    reunitarize_rows(Ud);
    U = convert<R>(Ud);
  }
  f.template store<R>(MU, par, i, U);
  if (fails) atomicAdd(status, fails);
}

template <typename S, int NR>
static cudaError_t hb_pass_impl(const LatDev& L, int mu, int par, double beta, uint64_t seed, uint32_t sweep,
                                int n_hits, uint32_t* status, cudaStream_t s, int block) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  dim3 grid(grid_for(L.g.Vh, block));
  switch (mu) {
    case 0:
      k_hb_pass<S, NR, 0><<<grid, block, 0, s>>>(L.g, f, par, S(beta), k0, k1, sweep, n_hits, status);
      break;
    case 1:
      k_hb_pass<S, NR, 1><<<grid, block, 0, s>>>(L.g, f, par, S(beta), k0, k1, sweep, n_hits, status);
      break;
    case 2:
      k_hb_pass<S, NR, 2><<<grid, block, 0, s>>>(L.g, f, par, S(beta), k0, k1, sweep, n_hits, status);
      break;
    default:
      k_hb_pass<S, NR, 3><<<grid, block, 0, s>>>(L.g, f, par, S(beta), k0, k1, sweep, n_hits, status);
      break;
  }
  return cudaGetLastError();
}

cudaError_t launch_hb_pass(const LatDev& L, int mu, int parity, double beta, uint64_t seed, uint32_t sweep,
                           int n_hits, uint32_t* status, cudaStream_t s, int block) {
  if (block <= 0) block = 128;
  QCB_DISPATCH_STORE(L, hb_pass_impl, L, mu, parity, beta, seed, sweep, n_hits, status, s, block);
}

}  // namespace qcb
