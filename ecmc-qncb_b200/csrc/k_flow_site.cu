// k_flow_site.cu — one fused Wilson-flow RK3 stage with one thread per site (all four links).
//
// Reference: GradientFlow (src/flow/gradient_flow.cpp:15-114), as in k_flow.cu; the stage
// arithmetic per link is the same (flow_link.cuh), only the work is grouped by site.
//
// One thread per site; the per-site body (flow_site.cuh) forms the product shared by the two
// forward staples of each plane once and keeps the links around x in L1/L2.
#include "dispatch.cuh"
#include "flow_site.cuh"
#include "obs_site.cuh"
#include "reduce.cuh"
#include "sync.cuh"

namespace qcb {

#ifndef QCB_FLOW_SITE_MINB
#define QCB_FLOW_SITE_MINB 5
#endif

template <typename S, int NR, int STAGE>
__global__ void __launch_bounds__(FS_THREADS, QCB_FLOW_SITE_MINB) k_flow_site(Geom g, Links<S, NR> src,
                                                                             Links<S, NR> dst, AlgField<S> acc,
                                                                             S eps) {
  extern __shared__ __align__(16) unsigned char fs_smem[];
  pdl_launch_dependents();  // launched with programmatic stream serialization
  pdl_wait();
  const int par = blockIdx.x & 1;
  const uint32_t i = (blockIdx.x >> 1) * FS_THREADS + threadIdx.x;
  if (i >= g.Vh) return;
  flow_site<Links<S, NR>, AlgField<S>, arith_t<S>, NR>(g, src, dst, acc, arith_t<S>(eps), STAGE, par, i,
                                                     reinterpret_cast<arith_t<S>*>(fs_smem));
}

// Stage 1 of a measured RK3 step: the site's four links as k_flow_site, and the clover q and e
// of the site from the same source links (site_qe, the arithmetic of k_clover_qe), summed per
// block in FP64.  The clover's links are the stage's own neighbourhood, read from L1/L2.
// Four resident blocks (128 registers): the clover planes spill at the flow kernel's bound of 96.
template <typename S, int NR>
__global__ void __launch_bounds__(FS_THREADS, 4) k_flow_site_qe(Geom g, Links<S, NR> src,
                                                                                Links<S, NR> dst, AlgField<S> acc,
                                                                                S eps, double* __restrict__ parts) {
  extern __shared__ __align__(16) unsigned char fs_smem[];
  __shared__ double sh[FS_THREADS / 32];
  const int par = blockIdx.x & 1;
  const uint32_t i = (blockIdx.x >> 1) * FS_THREADS + threadIdx.x;
  double q = 0.0, e = 0.0;
  if (i < g.Vh) {
    flow_site<Links<S, NR>, AlgField<S>, arith_t<S>, NR>(g, src, dst, acc, arith_t<S>(eps), 1, par, i,
                                                         reinterpret_cast<arith_t<S>*>(fs_smem));
    const Coord x = cb_coord(g, par, i);
    arith_t<S> qs = 0, es = 0;
    site_qe<Links<S, NR>, arith_t<S>>(g, src, x, par, i, &qs, &es);
    q = (double)qs;
    e = (double)es;
  }
  const double bq = block_sum<FS_THREADS>(q, sh);
  const double be = block_sum<FS_THREADS>(e, sh);
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = bq;
    parts[gridDim.x + blockIdx.x] = be;
  }
}

template <typename S, int NR>
static cudaError_t flow_site_qe_impl(const LatDev& Ls, const LatDev& Ld, const AlgDev& z, double eps, double* parts,
                                     cudaStream_t s) {
  Links<S, NR> src, dst;
  src.p = reinterpret_cast<typename Links<S, NR>::V*>(Ls.links);
  src.stride = Ls.g.stride;
  dst.p = reinterpret_cast<typename Links<S, NR>::V*>(Ld.links);
  dst.stride = Ld.g.stride;
  AlgField<S> acc;
  acc.p = reinterpret_cast<typename AlgField<S>::V*>(z.p);
  acc.stride = Ls.g.stride;
  const size_t smem = flow_site_smem<arith_t<S>, NR>();
  k_flow_site_qe<S, NR><<<dim3(grid_for(Ls.g.Vh, FS_THREADS) * 2), FS_THREADS, smem, s>>>(Ls.g, src, dst, acc, S(eps),
                                                                                        parts);
  return cudaGetLastError();
}

int flow_site_blocks(const LatDev& L) { return (int)grid_for(L.g.Vh, FS_THREADS) * 2; }

cudaError_t launch_flow_site_qe(const LatDev& src, const LatDev& dst, const AlgDev& z, double eps, double* parts,
                                cudaStream_t s) {
  if (src.prec != dst.prec || src.nr != dst.nr || src.prec != QCB_PREC_FP32) return cudaErrorInvalidValue;
  if (src.g.tlo != 0 || src.g.thi != src.g.L[3] - 1) return cudaErrorInvalidValue;  // whole lattices only
  if (src.nr == 12) return flow_site_qe_impl<float, 12>(src, dst, z, eps, parts, s);
  if (src.nr == 18) return flow_site_qe_impl<float, 18>(src, dst, z, eps, parts, s);
  return cudaErrorInvalidValue;
}

template <typename S, int NR>
static cudaError_t flow_site_impl(int stage, const LatDev& Ls, const LatDev& Ld, const AlgDev& z, double eps,
                                  cudaStream_t s) {
  Links<S, NR> src, dst;
  src.p = reinterpret_cast<typename Links<S, NR>::V*>(Ls.links);
  src.stride = Ls.g.stride;
  dst.p = reinterpret_cast<typename Links<S, NR>::V*>(Ld.links);
  dst.stride = Ld.g.stride;
  AlgField<S> acc;
  acc.p = reinterpret_cast<typename AlgField<S>::V*>(z.p);
  acc.stride = Ls.g.stride;
  const size_t smem = flow_site_smem<arith_t<S>, NR>();
  void (*kern)(Geom, Links<S, NR>, Links<S, NR>, AlgField<S>, S) =
      stage == 1 ? k_flow_site<S, NR, 1> : (stage == 2 ? k_flow_site<S, NR, 2> : k_flow_site<S, NR, 3>);
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // programmatic stream serialization: the stage's blocks become resident while the previous
  // kernel drains (the kernel waits for it before reading)
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for(Ls.g.Vh, FS_THREADS) * 2);
  cfg.blockDim = dim3(FS_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, kern, Ls.g, src, dst, acc, S(eps));
  return e != cudaSuccess ? e : cudaGetLastError();
}

// FP32 storages only (the FP64 kernels keep one thread per link: at three resident blocks per SM
// of the FP64 register budget this kernel would spill).
cudaError_t launch_flow_site(int stage, const LatDev& src, const LatDev& dst, const AlgDev& z, double eps,
                             cudaStream_t s) {
  if (src.prec != dst.prec || src.nr != dst.nr || src.prec != QCB_PREC_FP32) return cudaErrorInvalidValue;
  if (src.nr == 12) return flow_site_impl<float, 12>(stage, src, dst, z, eps, s);
  if (src.nr == 18) return flow_site_impl<float, 18>(stage, src, dst, z, eps, s);
  return cudaErrorInvalidValue;
}

}  // namespace qcb
