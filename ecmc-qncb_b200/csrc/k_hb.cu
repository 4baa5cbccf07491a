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
#include "hb_link.cuh"
#include "obs_site.cuh"
#include "reduce.cuh"
#include "sync.cuh"

namespace qcb {

// Blocks of 128 threads.  Resident blocks per SM (the register bound): FP32 5 (96
// registers, measured 2.6% faster than 4 on 32^4), FP64 3 (2.6% faster than 4, 2 slower).
#ifndef QCB_HB_MINB32
#define QCB_HB_MINB32 5
#endif
#ifndef QCB_HB_MINB64
#define QCB_HB_MINB64 3
#endif
template <typename S>
struct HbMinBlocks {
  static constexpr int value = sizeof(S) == 4 ? QCB_HB_MINB32 : QCB_HB_MINB64;
};

// Frozen links of the reference's block decomposition (src/geometry/GeometryCB.cpp:33-56)
// after a cumulative translation of the field by `shift`: link (x, mu) with
// (x_d + shift_d) % lcore == 0 for some d != mu is not updated.  lcore == 0: none frozen.
struct FrozenMask {
  int lcore;
  int shift[4];  // each in [0, lcore)
};

template <int MU>
__device__ __forceinline__ bool is_frozen(const Coord& x, const FrozenMask& m) {
#pragma unroll
  for (int d = 0; d < 4; ++d)
    if (d != MU && (x.c[d] + m.shift[d]) % m.lcore == 0) return true;
  return false;
}

template <typename S, int NR, int MU, bool FROZEN>
__global__ void __launch_bounds__(128, HbMinBlocks<S>::value) k_hb_pass(Geom g, Links<S, NR> f, int par, S beta, uint32_t k0,
                                                 uint32_t k1, uint32_t sweep, int n_hits, uint32_t* status,
                                                 FrozenMask fm) {
  // programmatic dependent launch: the next pass may be scheduled during this one's last
  // wave; this pass reads nothing before the previous kernel has completed
  pdl_launch_dependents();
  pdl_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  if (FROZEN && is_frozen<MU>(cb_coord(g, par, i), fm)) return;
  const uint32_t fails = hb_update_link<Links<S, NR>, arith_t<S>, NR, MU>(g, f, par, i, arith_t<S>(beta), k0, k1, sweep, n_hits);
  if (fails) atomicAdd(status, fails);
}

// Launch with programmatic stream serialization: the pass's blocks become resident while the
// previous kernel drains and wait in pdl_wait().  Measured per pass: 32^4 FP32-12 74.7 -> 72.9
// us, 64^4 1211 -> 1144 us, 32^4 FP64-18 200.7 -> 197.4 us.
template <typename S, int NR, int MU>
static cudaError_t hb_pass_launch(dim3 grid, int block, cudaStream_t s, const Geom& g, const Links<S, NR>& f, int par,
                                  S beta, uint32_t k0, uint32_t k1, uint32_t sweep, int n_hits, uint32_t* status,
                                  const FrozenMask& fm) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(block);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (fm.lcore > 0)
    return cudaLaunchKernelEx(&cfg, k_hb_pass<S, NR, MU, true>, g, f, par, beta, k0, k1, sweep, n_hits, status, fm);
  return cudaLaunchKernelEx(&cfg, k_hb_pass<S, NR, MU, false>, g, f, par, beta, k0, k1, sweep, n_hits, status, fm);
}

template <typename S, int NR>
static cudaError_t hb_pass_impl(const LatDev& L, int mu, int par, double beta, uint64_t seed, uint32_t sweep,
                                int n_hits, uint32_t* status, cudaStream_t s, int block, FrozenMask fm) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  dim3 grid(grid_for(L.g.Vh, block));
  switch (mu) {
    case 0: return hb_pass_launch<S, NR, 0>(grid, block, s, L.g, f, par, S(beta), k0, k1, sweep, n_hits, status, fm);
    case 1: return hb_pass_launch<S, NR, 1>(grid, block, s, L.g, f, par, S(beta), k0, k1, sweep, n_hits, status, fm);
    case 2: return hb_pass_launch<S, NR, 2>(grid, block, s, L.g, f, par, S(beta), k0, k1, sweep, n_hits, status, fm);
    default: return hb_pass_launch<S, NR, 3>(grid, block, s, L.g, f, par, S(beta), k0, k1, sweep, n_hits, status, fm);
  }
}

// Pass (mu = 3, par) of a measured sweep (whole lattices only): the updates of k_hb_pass, and
// per block the FP64 sum of the spatial plaquettes of its sites (parity par), plus for par = 1
// Re tr(U_3 A_3) of each updated link.  After the pass of parity 0 the spatial links and the
// even U_3 links are final, so the pass of parity 1 sees final staples; every temporal
// plaquette holds exactly one odd U_3 link, so Re tr(U_3(x) A_3(x)) over odd x counts each
// temporal plaquette once, and the spatial plaquettes of both parities count each spatial one
// once.
template <typename S, int NR>
__global__ void __launch_bounds__(128, HbMinBlocks<S>::value) k_hb_pass_meas(Geom g, Links<S, NR> f, int par, S beta,
                                                                            uint32_t k0, uint32_t k1, uint32_t sweep,
                                                                            int n_hits, uint32_t* status,
                                                                            double* __restrict__ parts) {
  __shared__ double sh[4];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  uint32_t fails = 0;
  if (i < g.Vh) {
    const Coord x = cb_coord(g, par, i);
    arith_t<S> retr = 0;
    fails = hb_update_at<Links<S, NR>, arith_t<S>, NR, 3, true>(g, f, x, par, i, arith_t<S>(beta), k0, k1, sweep, n_hits, &retr);
    v = (double)site_plaquette_spatial<Links<S, NR>, arith_t<S>>(g, f, x, par, i);
    if (par) v += (double)retr;
  }
  if (fails) atomicAdd(status, fails);
  const double b = block_sum<128>(v, sh);
  if (threadIdx.x == 0) parts[blockIdx.x] = b;
}

template <typename S, int NR>
static cudaError_t hb_meas_impl(const LatDev& L, int par, double beta, uint64_t seed, uint32_t sweep, int n_hits,
                                uint32_t* status, double* parts, cudaStream_t s) {
  Links<S, NR> f;
  f.p = reinterpret_cast<typename Links<S, NR>::V*>(L.links);
  f.stride = L.g.stride;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  k_hb_pass_meas<S, NR><<<grid_for(L.g.Vh, 128), 128, 0, s>>>(L.g, f, par, S(beta), k0, k1, sweep, n_hits, status,
                                                              parts);
  return cudaGetLastError();
}

int hb_meas_blocks(const LatDev& L) { return (int)grid_for(L.g.Vh, 128); }

cudaError_t launch_hb_pass_meas(const LatDev& L, int parity, double beta, uint64_t seed, uint32_t sweep, int n_hits,
                                uint32_t* status, double* parts, cudaStream_t s) {
  if (L.g.tlo != 0 || L.g.thi != L.g.L[3] - 1) return cudaErrorInvalidValue;  // whole lattices only
  QCB_DISPATCH_STORE(L, hb_meas_impl, L, parity, beta, seed, sweep, n_hits, status, parts, s);
}

cudaError_t launch_hb_pass(const LatDev& L, int mu, int parity, double beta, uint64_t seed, uint32_t sweep,
                           int n_hits, uint32_t* status, cudaStream_t s, int block, const int* frozen) {
  if (block <= 0) block = 128;
  FrozenMask fm = {0, {0, 0, 0, 0}};
  if (frozen) {
    fm.lcore = frozen[0];
    for (int d = 0; d < 4; ++d) fm.shift[d] = frozen[1 + d];
  }
  QCB_DISPATCH_STORE(L, hb_pass_impl, L, mu, parity, beta, seed, sweep, n_hits, status, s, block, fm);
}

}  // namespace qcb
