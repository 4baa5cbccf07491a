// k_flow_site.cu — one fused Wilson-flow RK3 stage with one thread per site (all four links).
//
// Reference: GradientFlow (src/flow/gradient_flow.cpp:15-114), as in k_flow.cu; the stage
// arithmetic per link is the same (flow_link.cuh), only the work is grouped by site.
//
// One thread per site; the per-site body (flow_site.cuh) forms the product shared by the two
// forward staples of each plane once and keeps the links around x in L1/L2.
#include "dispatch.cuh"
#include "flow_site.cuh"

namespace qcb {

#ifndef QCB_FLOW_SITE_MINB
#define QCB_FLOW_SITE_MINB 5
#endif

template <typename S, int NR, int STAGE>
__global__ void __launch_bounds__(FS_THREADS, QCB_FLOW_SITE_MINB) k_flow_site(Geom g, Links<S, NR> src,
                                                                             Links<S, NR> dst, AlgField<S> acc,
                                                                             S eps) {
  extern __shared__ __align__(16) unsigned char fs_smem[];
  const int par = blockIdx.x & 1;
  const uint32_t i = (blockIdx.x >> 1) * FS_THREADS + threadIdx.x;
  if (i >= g.Vh) return;
  flow_site<Links<S, NR>, AlgField<S>, S, NR>(g, src, dst, acc, eps, STAGE, par, i, reinterpret_cast<S*>(fs_smem));
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
  const size_t smem = flow_site_smem<S, NR>();
  dim3 grid(grid_for(Ls.g.Vh, FS_THREADS) * 2);
  cudaError_t e = cudaSuccess;
  if (stage == 1) {
    if (smem > 48 * 1024)
      e = cudaFuncSetAttribute(k_flow_site<S, NR, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_flow_site<S, NR, 1><<<grid, FS_THREADS, smem, s>>>(Ls.g, src, dst, acc, S(eps));
  } else if (stage == 2) {
    if (smem > 48 * 1024)
      e = cudaFuncSetAttribute(k_flow_site<S, NR, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_flow_site<S, NR, 2><<<grid, FS_THREADS, smem, s>>>(Ls.g, src, dst, acc, S(eps));
  } else {
    if (smem > 48 * 1024)
      e = cudaFuncSetAttribute(k_flow_site<S, NR, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_flow_site<S, NR, 3><<<grid, FS_THREADS, smem, s>>>(Ls.g, src, dst, acc, S(eps));
  }
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
