// k_obs.cu — mean plaquette and clover Q/E reductions.
//
// References:
//   mean_plaquette_local / _global (src/observables/observables_mpi.cpp:8-43): serial sum of
//   Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag)/3 over x and mu < nu, / (6V).
//   clover_site / local_q_e_clover / topo_q_e_clover(_global) (observables_mpi.cpp:61-150):
//   F_{mu nu} = (C - C^dag)/8 with C the sum of the four leaves at x,
//   q = (tr F01 F23 - tr F02 F13 + tr F03 F12) / (4 pi^2), e = 1/2 sum_{mu<nu} |F|^2.
// Here: one thread per site (both parities), per-site value in the lattice's arithmetic
// type, converted to FP64; FP64 tree reduction inside each block; the block partials are
// summed in a fixed order with Neumaier compensation by a single-block kernel.  The grid
// is a fixed multiple of the SM count (grid-stride loop), so the scratch is bounded.
#include "dispatch.cuh"

namespace qcb {

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 148 * 8;

int reduce_blocks() { return RED_BLOCKS; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of v (valid in thread 0).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (w == 0) {
    r = (lane < NT / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

// Neumaier-compensated sum of n partials (one block), written to out[0].
__global__ void k_finalize(const double* __restrict__ parts, int n, int nq, double* __restrict__ out) {
  // thread q sums quantity q sequentially (n is ~1k): fixed order, compensated.
  const int q = threadIdx.x;
  if (q >= nq) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n; ++k) {
    double v = parts[q * n + k];
    double t = s + v;
    if (fabs(s) >= fabs(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  out[q] = s + c;
}

// ---- plaquette ------------------------------------------------------------------------
template <typename S, int NR, typename R>
__device__ __forceinline__ R site_plaquette(const Geom& g, const Links<S, NR>& f, const Coord& x, int par,
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

template <typename S, int NR>
__global__ void __launch_bounds__(RED_THREADS) k_plaquette(Geom g, Links<S, NR> f, double* __restrict__ parts) {
  __shared__ double sh[RED_THREADS / 32];
  double acc = 0.0;
  const uint64_t n = (uint64_t)g.V;
  for (uint64_t t = (uint64_t)blockIdx.x * RED_THREADS + threadIdx.x; t < n; t += (uint64_t)gridDim.x * RED_THREADS) {
    const int par = (t >= g.Vh) ? 1 : 0;
    const uint32_t i = (uint32_t)(t - (par ? g.Vh : 0));
    const Coord x = cb_coord(g, par, i);
    acc += (double)site_plaquette<S, NR, S>(g, f, x, par, i);
  }
  double b = block_sum<RED_THREADS>(acc, sh);
  if (threadIdx.x == 0) parts[blockIdx.x] = b;
}

template <typename S, int NR>
static cudaError_t plaquette_impl(const LatDev& L, double* scratch, double* out, cudaStream_t s, int) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  k_plaquette<S, NR><<<RED_BLOCKS, RED_THREADS, 0, s>>>(L.g, f, scratch);
  k_finalize<<<1, 32, 0, s>>>(scratch, RED_BLOCKS, 1, out);
  return cudaGetLastError();
}

cudaError_t launch_plaquette(const LatDev& L, double* scratch, double* out, cudaStream_t s, int block) {
  QCB_DISPATCH_STORE(L, plaquette_impl, L, scratch, out, s, block);
}

// Same reduction with a caller-chosen number of blocks (partials written to scratch[0..nblocks)).
template <typename S, int NR>
static cudaError_t plaquette_partials_impl(const LatDev& L, int nblocks, double* scratch, double* out,
                                           cudaStream_t s) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  k_plaquette<S, NR><<<nblocks, RED_THREADS, 0, s>>>(L.g, f, scratch);
  k_finalize<<<1, 32, 0, s>>>(scratch, nblocks, 1, out);
  return cudaGetLastError();
}

cudaError_t launch_plaquette_partials(const LatDev& L, int nblocks, double* scratch, double* out, cudaStream_t s) {
  if (nblocks < 1) return cudaErrorInvalidValue;
  QCB_DISPATCH_STORE(L, plaquette_partials_impl, L, nblocks, scratch, out, s);
}

int reduce_threads() { return RED_THREADS; }

// ---- clover Q and E -------------------------------------------------------------------
// Clover sum C_{mu nu}(x) of the four leaves, in the reference's leaf order
// (observables_mpi.cpp:70-80).
template <typename S, int NR, typename R, int MU, int NU>
__device__ __forceinline__ m3<R> clover_F(const Geom& g, const Links<S, NR>& f, const Coord& x, int par,
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
  m3<R> F;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      F.e[a][b] = mk<R>(R(0.125) * (C.e[a][b].re - C.e[b][a].re), R(0.125) * (C.e[a][b].im + C.e[b][a].im));
  return F;
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
template <typename S, int NR, typename R, int M1, int N1, int M2, int N2>
__device__ __noinline__ void pair_qe(Geom g, Links<S, NR> f, Coord x, int par, uint32_t i, R sgn, R* q, R* e) {
  const m3<R> Fa = clover_F<S, NR, R, M1, N1>(g, f, x, par, i);
  const m3<R> Fb = clover_F<S, NR, R, M2, N2>(g, f, x, par, i);
  *q += sgn * re_tr_nn(Fa, Fb);
  *e += sqnorm(Fa) + sqnorm(Fb);
}

template <typename S, int NR>
__global__ void __launch_bounds__(RED_THREADS) k_clover_qe(Geom g, Links<S, NR> f, double* __restrict__ parts) {
  typedef S R;
  __shared__ double sh[RED_THREADS / 32];
  double accq = 0.0, acce = 0.0;
  const uint64_t n = (uint64_t)g.V;
  for (uint64_t t = (uint64_t)blockIdx.x * RED_THREADS + threadIdx.x; t < n; t += (uint64_t)gridDim.x * RED_THREADS) {
    const int par = (t >= g.Vh) ? 1 : 0;
    const uint32_t i = (uint32_t)(t - (par ? g.Vh : 0));
    const Coord x = cb_coord(g, par, i);
    R q = 0, e = 0;
    pair_qe<S, NR, R, 0, 1, 2, 3>(g, f, x, par, i, R(1), &q, &e);
    pair_qe<S, NR, R, 0, 2, 1, 3>(g, f, x, par, i, R(-1), &q, &e);
    pair_qe<S, NR, R, 0, 3, 1, 2>(g, f, x, par, i, R(1), &q, &e);
    accq += (double)q;
    acce += (double)e;
  }
  double bq = block_sum<RED_THREADS>(accq, sh);
  double be = block_sum<RED_THREADS>(acce, sh);
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = bq;
    parts[RED_BLOCKS + blockIdx.x] = be;
  }
}

// out2[0] = Q = sum q / (4 pi^2); out2[1] = E = sum e / 2 / V.
__global__ void k_qe_scale(double* out2, double inv_vol) {
  out2[0] = out2[0] * (1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846));
  out2[1] = 0.5 * out2[1] * inv_vol;
}

template <typename S, int NR>
static cudaError_t clover_impl(const LatDev& L, double* scratch, double* out2, cudaStream_t s, int) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  k_clover_qe<S, NR><<<RED_BLOCKS, RED_THREADS, 0, s>>>(L.g, f, scratch);
  k_finalize<<<1, 32, 0, s>>>(scratch, RED_BLOCKS, 2, out2);
  k_qe_scale<<<1, 1, 0, s>>>(out2, 1.0 / (double)L.g.V);
  return cudaGetLastError();
}

cudaError_t launch_clover_qe(const LatDev& L, double* scratch, double* out2, cudaStream_t s, int block) {
  QCB_DISPATCH_STORE(L, clover_impl, L, scratch, out2, s, block);
}

}  // namespace qcb
