// k_obs.cu — mean plaquette and clover Q/E reductions.
//
// References:
//   mean_plaquette_local / _global (src/observables/observables_mpi.cpp:8-43): serial sum of
//   Re tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag)/3 over x and mu < nu, / (6V).
//   clover_site / local_q_e_clover / topo_q_e_clover(_global) (observables_mpi.cpp:61-150):
//   F_{mu nu} = (C - C^dag)/8 with C the sum of the four leaves at x,
//   q = (tr F01 F23 - tr F02 F13 + tr F03 F12) / (4 pi^2), e = 1/2 sum_{mu<nu} |F|^2.
// Here: one thread per site (the two parities of a checkerboard index adjacent; a slab
// skips its halo slices), per-site value in the lattice's arithmetic type, converted to FP64; FP64 tree reduction inside each block; the block partials are
// summed in a fixed order with Neumaier compensation by a single-block kernel.  The grid
// is a fixed multiple of the SM count (grid-stride loop), so the scratch is bounded.
#include "dispatch.cuh"
#include "obs_site.cuh"
#include "reduce.cuh"

namespace qcb {

constexpr int RED_THREADS = 128;
constexpr int RED_BLOCKS = 148 * 8;

// Minimum resident blocks per SM of the reduction kernels: the clover site evaluation is
// the largest per-thread body; the bound keeps FP32 at 4 x 128 threads (128 registers) and
// FP64 at 2 x 128 threads per SM.
template <typename S>
struct RedMinBlocks {
  static constexpr int value = sizeof(S) == 4 ? 4 : 2;
};

int reduce_blocks() { return RED_BLOCKS; }

// Neumaier-compensated sums of nq quantities of n partials each (parts[q*n + k]), one warp
// per quantity: lane j sums k = j, j+32, ...; lane 0 then adds the 32 lane sums in lane
// order.  The order is fixed, so the result is deterministic.  out[q] = sum.
__global__ void k_finalize(const double* __restrict__ parts, int n, int nq, double* __restrict__ out) {
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (q >= nq) return;
  double s = 0.0, c = 0.0;
  for (int k = lane; k < n; k += 32) neumaier_add(s, c, parts[q * n + k]);
  __shared__ double ls[4][32], lc[4][32];
  ls[q][lane] = s;
  lc[q][lane] = c;
  __syncwarp();
  if (lane == 0) {
    double S = 0.0, Cc = 0.0;
    for (int j = 0; j < 32; ++j) {
      neumaier_add(S, Cc, ls[q][j]);
      Cc += lc[q][j];
    }
    out[q] = S + Cc;
  }
}

// Reduction grid: one block per RED_THREADS sites, at most RED_BLOCKS.
static int red_grid(const Geom& g) {
  const uint64_t want = ((uint64_t)g.V + RED_THREADS - 1) / RED_THREADS;
  return (int)(want < (uint64_t)RED_BLOCKS ? want : (uint64_t)RED_BLOCKS);
}

template <typename S, int NR>
__global__ void __launch_bounds__(RED_THREADS, RedMinBlocks<S>::value) k_plaquette(Geom g, Links<S, NR> f, double* __restrict__ parts) {
  __shared__ double sh[RED_THREADS / 32];
  double acc = 0.0;
  const uint64_t n = (uint64_t)g.V;
  for (uint64_t t = (uint64_t)blockIdx.x * RED_THREADS + threadIdx.x; t < n; t += (uint64_t)gridDim.x * RED_THREADS) {
    // both parities of a checkerboard index together: a site's neighbours (opposite
    // parity) are then read close in time, from L2
    const int par = (int)(t & 1);
    const uint32_t i = (uint32_t)(t >> 1);
    const Coord x = cb_coord(g, par, i);
    if (own_site(g, x.c[3])) acc += (double)site_plaquette<Links<S, NR>, arith_t<S>>(g, f, x, par, i);
  }
  double b = block_sum<RED_THREADS>(acc, sh);
  if (threadIdx.x == 0) parts[blockIdx.x] = b;
}

template <typename S, int NR>
static cudaError_t plaquette_impl(const LatDev& L, double* scratch, double* out, cudaStream_t s, int) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  const int nb = red_grid(L.g);
  k_plaquette<S, NR><<<nb, RED_THREADS, 0, s>>>(L.g, f, scratch);
  k_finalize<<<1, 32, 0, s>>>(scratch, nb, 1, out);
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

// First level of a deterministic sum of nq quantities of n partials each (quantity q at
// parts[q * n ..]): block (b, q) sums the chunk [b * chunk, min((b + 1) * chunk, n)) of quantity
// q (thread-strided in index order, then the block tree) into out[q * gridDim.x + b].
__global__ void __launch_bounds__(RED_THREADS) k_sum_chunks(const double* __restrict__ parts, int n, int chunk,
                                                           double* __restrict__ out) {
  __shared__ double sh[RED_THREADS / 32];
  const double* p = parts + (size_t)blockIdx.y * n;
  const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
  double s = 0.0, c = 0.0;
  for (int k = lo + threadIdx.x; k < hi; k += RED_THREADS) neumaier_add(s, c, p[k]);
  const double b = block_sum<RED_THREADS>(s + c, sh);
  if (threadIdx.x == 0) out[blockIdx.y * gridDim.x + blockIdx.x] = b;
}

// out[q] = sum of parts[q * n .. q * n + n) for q < nq (nq <= 4), in a fixed order whatever the
// device: chunks of at most 256 x 128 partials per block, then the single-warp Neumaier
// finalize.  tmp holds 256 * nq doubles.
static cudaError_t sum_parts(const double* parts, int n, int nq, double* tmp, double* out, cudaStream_t s) {
  if (n < 1 || nq < 1 || nq > 4) return cudaErrorInvalidValue;
  const int nb = min(256, (n + RED_THREADS - 1) / RED_THREADS);
  const int chunk = (n + nb - 1) / nb;
  k_sum_chunks<<<dim3(nb, nq), RED_THREADS, 0, s>>>(parts, n, chunk, tmp);
  k_finalize<<<1, 32 * nq, 0, s>>>(tmp, nb, nq, out);
  return cudaGetLastError();
}

cudaError_t launch_sum_parts(const double* parts, int n, double* tmp, double* out, cudaStream_t s) {
  return sum_parts(parts, n, 1, tmp, out, s);
}

template <typename S, int NR>
__global__ void __launch_bounds__(RED_THREADS, RedMinBlocks<S>::value) k_clover_qe(Geom g, Links<S, NR> f, double* __restrict__ parts) {
  typedef S R;
  __shared__ double sh[RED_THREADS / 32];
  double accq = 0.0, acce = 0.0;
  const uint64_t n = (uint64_t)g.V;
  for (uint64_t t = (uint64_t)blockIdx.x * RED_THREADS + threadIdx.x; t < n; t += (uint64_t)gridDim.x * RED_THREADS) {
    // both parities of a checkerboard index together: a site's neighbours (opposite
    // parity) are then read close in time, from L2
    const int par = (int)(t & 1);
    const uint32_t i = (uint32_t)(t >> 1);
    const Coord x = cb_coord(g, par, i);
    if (!own_site(g, x.c[3])) continue;
    R q = 0, e = 0;
    site_qe<Links<S, NR>, R>(g, f, x, par, i, &q, &e);
    accq += (double)q;
    acce += (double)e;
  }
  double bq = block_sum<RED_THREADS>(accq, sh);
  double be = block_sum<RED_THREADS>(acce, sh);
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = bq;
    parts[gridDim.x + blockIdx.x] = be;
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
  const int nb = red_grid(L.g);
  k_clover_qe<S, NR><<<nb, RED_THREADS, 0, s>>>(L.g, f, scratch);
  k_finalize<<<1, 64, 0, s>>>(scratch, nb, 2, out2);
  k_qe_scale<<<1, 1, 0, s>>>(out2, 1.0 / (double)L.g.Vg);
  return cudaGetLastError();
}

cudaError_t launch_qe_from_parts(const double* parts, int n, double* tmp, double* out2, double inv_vol,
                                 cudaStream_t s) {
  cudaError_t e = sum_parts(parts, n, 2, tmp, out2, s);
  if (e != cudaSuccess) return e;
  k_qe_scale<<<1, 1, 0, s>>>(out2, inv_vol);
  return cudaGetLastError();
}

cudaError_t launch_clover_qe(const LatDev& L, double* scratch, double* out2, cudaStream_t s, int block) {
  QCB_DISPATCH_STORE(L, clover_impl, L, scratch, out2, s, block);
}

}  // namespace qcb
