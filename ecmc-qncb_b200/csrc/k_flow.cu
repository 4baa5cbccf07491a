// k_flow.cu — fused Wilson-flow RK3 stages.
//
// Reference: GradientFlow (src/flow/gradient_flow.cpp:15-128) runs five full-lattice loops
// per step (compute_force, compute_w1, compute_force, compute_w2, replace_force_0,
// compute_force, compute_w3) over three full GaugeField copies, with a halo exchange after
// every W update.  Each stage here is one kernel, one thread per link:
//   Z   = -P_TA(U A)                         (force, gradient_flow.cpp:15-34)
//   s1: X = eps/4 Z0;                acc = Z0                      (compute_w1, :37-53)
//   s2: X = 8/9 eps Z1 - 17/36 eps Z0; acc = 8/9 Z1 - 17/36 Z0    (compute_w2 + replace_force_0, :56-93)
//   s3: X = 3/4 eps Z2 - eps acc                                   (compute_w3, :96-114)
//   U' = exp(X) U   with Luescher's exponential (src/su3/utils.cpp:145-193)
// Links are double-buffered (src -> dst) because every stage reads neighbours of the
// previous stage; the force accumulator holds 8 reals per link.
#include "dispatch.cuh"
#include "flow_link.cuh"
#include "sync.cuh"

namespace qcb {

// Grid (2 * tiles, 4): blockIdx.y = mu, blockIdx.x = 2 * tile + parity.  Blocks are issued
// x-fastest, so one direction runs at a time over the whole lattice (one mu instantiation in
// the instruction cache) and both parities of a tile run together.  Measured per RK3 step on
// 32^4 FP32-12: 1.37 ms; a run-time-mu kernel with the eight (mu, parity) blocks of a tile
// adjacent: 1.58 ms; chunks of 256 / 512 / 1024 tiles with the four directions of a chunk in
// turn (to reuse the chunk's links from L2): 1.48 / 1.71 / 1.54 ms, because the direction
// changes every one or two waves of blocks and the four instantiations then compete for the
// instruction cache.  The flow is bound by instruction issue, not by DRAM.
// Resident blocks per SM (the register bound): FP32 5 (96 registers) measured 1.36 ms per RK3
// step on 32^4 FP32-12 against 1.74 ms with the compiler's own choice; FP64 3 measured
// 2.76 ms per step on 32^4 FP64-18 against 3.02 ms with the compiler's own choice or 2.
#ifndef QCB_FLOW_MINB32
#define QCB_FLOW_MINB32 5
#endif
#ifndef QCB_FLOW_MINB64
#define QCB_FLOW_MINB64 3
#endif
template <typename S, int NR, int STAGE>
__global__ void __launch_bounds__(128, sizeof(S) == 4 ? QCB_FLOW_MINB32 : QCB_FLOW_MINB64) k_flow_stage(Geom g, Links<S, NR> src, Links<S, NR> dst, AlgField<S> acc,
                                                    S eps) {
  pdl_launch_dependents();  // launched with programmatic stream serialization
  pdl_wait();
  const int mu = blockIdx.y;
  const uint32_t i = (blockIdx.x >> 1) * blockDim.x + threadIdx.x;
  const int par = blockIdx.x & 1;
  if (i >= g.Vh) return;
  switch (mu) {
    case 0: flow_link<Links<S, NR>, AlgField<S>, arith_t<S>, 0>(g, src, dst, acc, arith_t<S>(eps), STAGE, par, i); break;
    case 1: flow_link<Links<S, NR>, AlgField<S>, arith_t<S>, 1>(g, src, dst, acc, arith_t<S>(eps), STAGE, par, i); break;
    case 2: flow_link<Links<S, NR>, AlgField<S>, arith_t<S>, 2>(g, src, dst, acc, arith_t<S>(eps), STAGE, par, i); break;
    default: flow_link<Links<S, NR>, AlgField<S>, arith_t<S>, 3>(g, src, dst, acc, arith_t<S>(eps), STAGE, par, i); break;
  }
}

template <typename S, int NR>
static cudaError_t flow_impl(int stage, const LatDev& Ls, const LatDev& Ld, const AlgDev& z, double eps,
                             cudaStream_t s, int block) {
  Links<S, NR> src, dst;
  src.p = reinterpret_cast<typename Links<S, NR>::V*>(Ls.links);
  src.stride = Ls.g.stride;
  dst.p = reinterpret_cast<typename Links<S, NR>::V*>(Ld.links);
  dst.stride = Ld.g.stride;
  AlgField<S> acc;
  acc.p = reinterpret_cast<typename AlgField<S>::V*>(z.p);
  acc.stride = Ls.g.stride;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for(Ls.g.Vh, block) * 2, 4);
  cfg.blockDim = dim3(block);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  void (*kern)(Geom, Links<S, NR>, Links<S, NR>, AlgField<S>, S) =
      stage == 1 ? k_flow_stage<S, NR, 1> : (stage == 2 ? k_flow_stage<S, NR, 2> : k_flow_stage<S, NR, 3>);
  return cudaLaunchKernelEx(&cfg, kern, Ls.g, src, dst, acc, S(eps));
}

// FP32 lattices run the flow with one thread per site (k_flow_site.cu): measured per RK3 step
// 1.297 -> 1.225 ms on 32^4 and 23.4 -> 20.3 ms on 64^4 (12-real), with DRAM traffic 1.12 x the
// algorithmic bytes instead of 2.0 x.  FP64 keeps one thread per link.
#ifndef QCB_FLOW_SITE
#define QCB_FLOW_SITE 1
#endif

cudaError_t launch_flow_stage(int stage, const LatDev& src, const LatDev& dst, const AlgDev& z, double eps,
                              cudaStream_t s, int block) {
  if (block <= 0) block = 128;
  if (src.prec != dst.prec || src.nr != dst.nr) return cudaErrorInvalidValue;
  if (QCB_FLOW_SITE && src.prec == 1) return launch_flow_site(stage, src, dst, z, eps, s);
  QCB_DISPATCH_STORE(src, flow_impl, stage, src, dst, z, eps, s, block);
}

}  // namespace qcb
