// k_batch.cu — persistent kernels that advance many independent lattices in one launch.
//
// The reference runs one lattice per process (src/bin/gauge_hb_ncb.cpp:18-201).  Here a
// batch of lattices of different sizes and couplings shares one cooperative launch: the
// work of every lattice is cut into levels (one checkerboard heatbath pass, or one RK3
// stage) and each level into tiles of sites.  Work items are ordered level-major across
// lattices, item j = (level, lattice, tile), and block b processes items b, b+G, b+2G, ...
// in order.  Before an item of level k of lattice l starts, all tiles of level k-1 of the
// same lattice must be finished: a per-lattice counter done[l] counts finished tiles, and
// the block waits (acquire) until done[l] >= k * ntiles[l].  Levels of different lattices
// overlap freely, so small lattices do not serialise the GPU.
//
// Progress: every item's dependencies have smaller indices, blocks take their items in
// increasing order, and the cooperative launch makes all blocks co-resident; so the
// smallest unfinished item always has its dependencies done.  Every wait is bounded by
// wall-clock time (WAIT_NS); a block that gives up raises an abort flag that makes every
// other block return, and the host reports the error.  Links and accumulators are read
// with L2-coherent loads (LD_CG), because blocks read links that other blocks wrote in the
// same launch.
#include "batch.h"
#include "dispatch.cuh"
#include "flow_link.cuh"
#include "flow_site.cuh"
#include "hb_link.cuh"
#include "obs_site.cuh"
#include "sync.cuh"

// Resident blocks of 128 threads per SM in FP32 (the register bound): 5 measured 10% (heatbath)
// and 19% (flow) faster than 4 on the 64-lattice batch, 3 slower.
#ifndef QCB_BATCH_MINB32
#define QCB_BATCH_MINB32 5
#endif

namespace qcb {

// Decode item r (within one level) into (lattice, tile) by binary search of prefix[].
__device__ __forceinline__ int find_lattice(const uint32_t* __restrict__ prefix, int nlat, uint32_t r) {
  int lo = 0, hi = nlat;  // prefix[lo] <= r < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= r)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Thread 0 waits until done[l] >= target; returns false (for the whole block) on abort
// or timeout (limit_ns of wall-clock time or WAIT_MAX_ITERS polls).  status[1] counts
// timeouts, status[2] is the abort flag.
__device__ __forceinline__ bool block_wait(const uint32_t* done, uint32_t target, uint32_t* status,
                                           uint64_t limit_ns = WAIT_NS) {
  __shared__ int ok;
  if (threadIdx.x == 0) ok = wait_geq(done, target, status, limit_ns) ? 1 : 0;
  __syncthreads();
  const bool r = ok != 0;
  __syncthreads();
  return r;
}

// Publish one finished tile of lattice l.
__device__ __forceinline__ void block_release(uint32_t* done) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(done, 1u);
}

// ---- one work item ----------------------------------------------------------------------
// Heatbath level k: pass k % 8 (mu = pass / 2, parity = pass % 2) of sweep sweep0 + k / 8;
// item tile = a tile of that pass's sites.
template <typename S, int NR>
__device__ __forceinline__ uint32_t hb_item(const BatchRun& run, const BatchLat& B, uint32_t level, uint32_t tile) {
  typedef Links<S, NR, LD_CG> F;
  const uint32_t sweep = B.sweep0 + level / 8;
  const int pass = (int)(level & 7), mu = pass >> 1, par = pass & 1;
  F f;
  f.p = reinterpret_cast<typename F::V*>(B.links);
  f.stride = B.g.stride;
  const arith_t<S> beta = arith_t<S>(S(B.beta));
  const int n_hits = B.n_hits > 0 ? B.n_hits : run.n_hits;
  uint32_t fails = 0;
  for (uint32_t k = threadIdx.x; k < B.tile; k += blockDim.x) {
    const uint32_t i = tile * B.tile + k;
    if (i >= B.g.Vh) break;
    fails += hb_update_link_rt<F, arith_t<S>, NR>(B.g, f, mu, par, i, beta, B.k0, B.k1, sweep, n_hits);
  }
  return fails;
}

// Flow level j = 3 s + k is stage k of RK3 step s.  With a = links, b = work for even s
// (swapped for odd s): stage 0 a -> b, stage 1 b -> a, stage 2 a -> b.  FP32: a flow item
// covers a tile of sites of one parity, all four links of each site (the single-lattice site
// kernel's body, flow_site.cuh): item r -> parity r % 2, tile r / 2.  FP64: a flow item covers
// a tile of one (mu, parity) block, one link per thread: item r -> (mu, parity) = r % 8,
// tile = r / 8.  The direction and the stage are run-time values here (one code body for all
// twelve (mu, stage) pairs): compiled-direction bodies, with the items of a level ordered
// direction-major, measured 7% (heatbath) and 13% (flow) slower on the 64-lattice batch,
// from register spills and instruction-cache misses.
template <typename S, int NR>
__device__ __forceinline__ void flow_item(const BatchRun& run, const BatchLat& B, uint32_t level, uint32_t local,
                                          arith_t<S>* slot_mem) {
  typedef Links<S, NR, LD_CG> F;
  typedef AlgField<S, LD_CG> Z;
  const uint32_t step = level / 3, stage = level - 3 * step;
  void* a = (step & 1) ? B.work : B.links;
  void* bb = (step & 1) ? B.links : B.work;
  F src, dst;
  src.p = reinterpret_cast<typename F::V*>(stage == 1 ? bb : a);
  dst.p = reinterpret_cast<typename F::V*>(stage == 1 ? a : bb);
  src.stride = dst.stride = B.g.stride;
  Z acc;
  acc.p = reinterpret_cast<typename Z::V*>(B.acc);
  acc.stride = B.g.stride;
  const arith_t<S> eps = arith_t<S>(S(B.eps != 0.0 ? B.eps : run.eps));
  if constexpr (sizeof(S) == 4) {
    const int par = (int)(local & 1);
    const uint32_t tile = local >> 1;
    for (uint32_t k = threadIdx.x; k < B.tile; k += blockDim.x) {
      const uint32_t i = tile * B.tile + k;
      if (i >= B.g.Vh) break;
      flow_site<F, Z, arith_t<S>, NR>(B.g, src, dst, acc, eps, (int)stage + 1, par, i, slot_mem);
    }
  } else {
    const int mp8 = (int)(local & 7), mu = mp8 >> 1, par = mp8 & 1;
    const uint32_t tile = local >> 3;
    for (uint32_t k = threadIdx.x; k < B.tile; k += blockDim.x) {
      const uint32_t i = tile * B.tile + k;
      if (i >= B.g.Vh) break;
      flow_link_rt<F, Z, arith_t<S>>(B.g, src, dst, acc, eps, (int)stage + 1, mu, par, i);
    }
  }
}

// ---- the persistent kernel -----------------------------------------------------------------
// KINDS: BATCH_HB or BATCH_FLOW for a launch of one kind, BATCH_MIXED when each lattice's
// descriptor says which kind its items are.  A lattice with B.nlev != 0 takes part in its
// first B.nlev levels only; its items at later levels are skipped (no wait, no release), and
// a lattice of kind BATCH_NONE in a mixed launch takes part in none.
template <typename S, int NR, int KINDS>
__global__ void __launch_bounds__(128, sizeof(S) == 4 ? QCB_BATCH_MINB32 : 2) k_batch(BatchRun run) {
  extern __shared__ __align__(16) unsigned char kb_smem[];  // FP32 flow: the T slots of flow_site
  const uint64_t total = (uint64_t)run.nlevels * run.per_level;
  uint32_t fails = 0;
  for (uint64_t item = blockIdx.x; item < total; item += gridDim.x) {
    const uint32_t level = (uint32_t)(item / run.per_level);
    const uint32_t r = (uint32_t)(item - (uint64_t)level * run.per_level);
    const int l = find_lattice(run.prefix, run.nlat, r);
    const BatchLat& B = run.lats[l];
    if (B.nlev != 0 && level >= B.nlev) continue;
    if (KINDS == BATCH_MIXED && B.kind == BATCH_NONE) continue;
    const uint32_t local = r - run.prefix[l];
    if (level > 0 && !block_wait(&run.done[l], level * B.ntiles, run.status)) return;
    const int kind = (KINDS == BATCH_MIXED) ? B.kind : KINDS;
    if (kind == BATCH_HB)
      fails += hb_item<S, NR>(run, B, level, local);
    else
      flow_item<S, NR>(run, B, level, local, reinterpret_cast<arith_t<S>*>(kb_smem));
    block_release(&run.done[l]);
  }
  if (fails) atomicAdd(&run.status[0], fails);
}

// ---- launch -------------------------------------------------------------------------------
template <typename S, int NR>
static cudaError_t batch_launch_impl(int kind, const BatchRun& run, int block, int max_blocks, cudaStream_t s) {
  void* fn = (kind == BATCH_HB) ? (void*)k_batch<S, NR, BATCH_HB>
             : (kind == BATCH_FLOW) ? (void*)k_batch<S, NR, BATCH_FLOW> : (void*)k_batch<S, NR, BATCH_MIXED>;
  const size_t smem = (sizeof(S) == 4 && kind != BATCH_HB) ? flow_site_smem<arith_t<S>, NR>() : 0;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem);
  if (e != cudaSuccess) return e;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const uint64_t total = (uint64_t)run.nlevels * run.per_level;
  uint64_t grid = (uint64_t)per_sm * (uint64_t)sms;
  if (max_blocks > 0 && (uint64_t)max_blocks < grid) grid = (uint64_t)max_blocks;
  if (grid > total) grid = total;
  if (grid == 0) return cudaSuccess;
  BatchRun r = run;
  void* args[] = {&r};
  return cudaLaunchCooperativeKernel(fn, dim3((unsigned)grid), dim3(block), args, smem, s);
}

cudaError_t launch_batch(int kind, const BatchRun& run, int prec, int nr, int block, int max_blocks,
                         cudaStream_t s) {
  LatDev probe;
  probe.prec = prec;
  probe.nr = nr;
  if (block <= 0) block = 128;
  if (block > 128 || (block & 31)) return cudaErrorInvalidValue;
  QCB_DISPATCH_STORE(probe, batch_launch_impl, kind, run, block, max_blocks, s);
}

// ---- wait self-test -------------------------------------------------------------------------
// Block 0 waits for flag[0] >= 1, which nothing sets, until its limit; it then counts a
// timeout and raises the abort flag.  The other blocks wait for the same flag with a longer
// limit and return when they see the abort flag.  Exercises the bounded wait and abort path
// of the persistent kernels without a fault.
__global__ void k_wait_probe(const uint32_t* flag, uint32_t* status, uint64_t limit_ns) {
  const uint64_t lim = blockIdx.x == 0 ? limit_ns : 4 * limit_ns;
  if (!block_wait(flag, 1u, status, lim)) return;
  if (threadIdx.x == 0) atomicAdd(&status[3], 1u);  // a wait that succeeded (not expected)
}

cudaError_t launch_wait_probe(const uint32_t* flag, uint32_t* status, uint64_t limit_ns, int blocks,
                              cudaStream_t s) {
  void* args[] = {(void*)&flag, (void*)&status, (void*)&limit_ns};
  return cudaLaunchCooperativeKernel((void*)k_wait_probe, dim3(blocks), dim3(32), args, 0, s);
}

// ---- batched observables --------------------------------------------------------------------
// One reduction item per (lattice, tile of RED_SITES sites, both parities: item site t is
// checkerboard index t >> 1 of parity t & 1); partial sums parts[item] (and parts[nitems + item] for the
// second quantity), then one warp per lattice adds its partials in a fixed order with
// Neumaier compensation.
constexpr int RED_SITES = 128;
int batch_red_sites() { return RED_SITES; }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
template <int NQ>
__device__ __forceinline__ void block_sums(double* v, double* out) {
  __shared__ double sh[NQ][RED_SITES / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double s = warp_sum_d(v[q]);
    if (lane == 0) sh[q][w] = s;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double r = (lane < RED_SITES / 32) ? sh[q][lane] : 0.0;
      r = warp_sum_d(r);
      if (lane == 0) out[q] = r;
    }
  }
}

template <typename S, int NR, int WHAT>
__global__ void __launch_bounds__(RED_SITES, sizeof(S) == 4 ? 4 : 2) k_batch_red(const BatchLat* __restrict__ lats,
                                                         const uint32_t* __restrict__ rprefix, int nlat,
                                                         uint32_t nitems, double* __restrict__ parts) {
  const uint32_t item = blockIdx.x;
  const int l = find_lattice(rprefix, nlat, item);
  const BatchLat& B = lats[l];
  const uint32_t t = (item - rprefix[l]) * RED_SITES + threadIdx.x;
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(B.links);
  f.stride = B.g.stride;
  double v[2] = {0.0, 0.0};
  if (t < B.g.V) {
    const int par = (int)(t & 1);  // both parities of a checkerboard index together
    const uint32_t i = t >> 1;
    const Coord x = cb_coord(B.g, par, i);
    if (WHAT == 0) {
      v[0] = (double)site_plaquette<Links<S, NR>, arith_t<S>>(B.g, f, x, par, i);
    } else {
      arith_t<S> q = 0, e = 0;
      site_qe<Links<S, NR>, arith_t<S>>(B.g, f, x, par, i, &q, &e);
      v[0] = (double)q;
      v[1] = (double)e;
    }
  }
  __shared__ double res[2];
  block_sums<2>(v, res);
  if (threadIdx.x == 0) {
    parts[item] = res[0];
    parts[nitems + item] = res[1];
  }
}

__device__ __forceinline__ void neumaier(double& s, double& c, double v) {
  const double t = s + v;
  if (fabs(s) >= fabs(v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

// One warp per lattice: lane j sums items j, j+32, ... of the lattice; lane 0 adds the 32
// lane sums in lane order.  WHAT 0: out[l] = sum / (6 V); WHAT 1: out[2l] = Q, out[2l+1] = E.
template <int WHAT>
__global__ void k_batch_red_finalize(const BatchLat* __restrict__ lats, const uint32_t* __restrict__ rprefix,
                                     int nlat, uint32_t nitems, const double* __restrict__ parts,
                                     double* __restrict__ out) {
  const int l = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (l >= nlat) return;
  const uint32_t a = rprefix[l], b = rprefix[l + 1];
  const double V = (double)lats[l].g.V;
  for (int q = 0; q < (WHAT == 0 ? 1 : 2); ++q) {
    double s = 0.0, c = 0.0;
    for (uint32_t k = a + lane; k < b; k += 32) neumaier(s, c, parts[(size_t)q * nitems + k]);
    double S = 0.0, Cc = 0.0;
    for (int j = 0; j < 32; ++j) {
      const double sj = __shfl_sync(0xffffffffu, s, j), cj = __shfl_sync(0xffffffffu, c, j);
      neumaier(S, Cc, sj);
      Cc += cj;
    }
    if (lane == 0) {
      const double tot = S + Cc;
      if (WHAT == 0)
        out[l] = tot / (6.0 * V);
      else if (q == 0)
        out[2 * l] = tot * (1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846));
      else
        out[2 * l + 1] = 0.5 * tot / V;
    }
  }
}

template <typename S, int NR>
static cudaError_t batch_red_impl(int what, const BatchLat* lats, const uint32_t* rprefix, int nlat,
                                  uint32_t nitems, double* scratch, double* out, cudaStream_t s) {
  if (nitems == 0) return cudaSuccess;
  if (what == 0) {
    k_batch_red<S, NR, 0><<<nitems, RED_SITES, 0, s>>>(lats, rprefix, nlat, nitems, scratch);
    k_batch_red_finalize<0><<<(nlat + 3) / 4, 128, 0, s>>>(lats, rprefix, nlat, nitems, scratch, out);
  } else {
    k_batch_red<S, NR, 1><<<nitems, RED_SITES, 0, s>>>(lats, rprefix, nlat, nitems, scratch);
    k_batch_red_finalize<1><<<(nlat + 3) / 4, 128, 0, s>>>(lats, rprefix, nlat, nitems, scratch, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_plaquette(const BatchLat* lats, const uint32_t* rprefix, int nlat, uint32_t nitems,
                                   int prec, int nr, double* scratch, double* out, cudaStream_t s) {
  LatDev probe;
  probe.prec = prec;
  probe.nr = nr;
  QCB_DISPATCH_STORE(probe, batch_red_impl, 0, lats, rprefix, nlat, nitems, scratch, out, s);
}
cudaError_t launch_batch_qe(const BatchLat* lats, const uint32_t* rprefix, int nlat, uint32_t nitems, int prec,
                            int nr, double* scratch, double* out2, cudaStream_t s) {
  LatDev probe;
  probe.prec = prec;
  probe.nr = nr;
  QCB_DISPATCH_STORE(probe, batch_red_impl, 1, lats, rprefix, nlat, nitems, scratch, out2, s);
}

}  // namespace qcb
