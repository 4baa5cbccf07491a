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
#include "staple.cuh"

namespace qcb {

template <typename S, int NR, int STAGE, int MU>
__device__ __forceinline__ void flow_link(const Geom& g, const Links<S, NR>& src, const Links<S, NR>& dst,
                                          const AlgField<S>& acc, S eps, int par, uint32_t i) {
  typedef S R;
  const Coord x = cb_coord(g, par, i);
  const m3<R> A = staple_sum<S, NR, R, MU>(g, src, x, par, i);
  const m3<R> U = src.template load<R>(MU, par, i);
  // Z = P_TA(-U A) = -P_TA(U A)
  alg8<R> Z = proj_ta(mul_nn(U, A));
#pragma unroll
  for (int k = 0; k < 8; ++k) Z.a[k] = -Z.a[k];
  alg8<R> X;
  if (STAGE == 1) {
    const R c = R(0.25) * eps;
#pragma unroll
    for (int k = 0; k < 8; ++k) X.a[k] = c * Z.a[k];
    acc.template store<R>(MU, par, i, Z);
  } else if (STAGE == 2) {
    const alg8<R> Z0 = acc.template load<R>(MU, par, i);
    const R c1 = R(8.0 / 9.0) * eps, c0 = R(17.0 / 36.0) * eps;
    alg8<R> N;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      X.a[k] = c1 * Z.a[k] - c0 * Z0.a[k];
      N.a[k] = R(8.0 / 9.0) * Z.a[k] - R(17.0 / 36.0) * Z0.a[k];
    }
    acc.template store<R>(MU, par, i, N);
  } else {
    const alg8<R> Z0 = acc.template load<R>(MU, par, i);
    const R c1 = R(0.75) * eps;
#pragma unroll
    for (int k = 0; k < 8; ++k) X.a[k] = c1 * Z.a[k] - eps * Z0.a[k];
  }
  const m3<R> E = exp_su3(X);
  dst.template store<R>(MU, par, i, mul_nn(E, U));
}

// blockIdx.y = mu * 2 + parity
template <typename S, int NR, int STAGE>
__global__ void __launch_bounds__(128) k_flow_stage(Geom g, Links<S, NR> src, Links<S, NR> dst, AlgField<S> acc,
                                                    S eps) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Vh) return;
  const int mu = blockIdx.y >> 1, par = blockIdx.y & 1;
  switch (mu) {
    case 0:
      flow_link<S, NR, STAGE, 0>(g, src, dst, acc, eps, par, i);
      break;
    case 1:
      flow_link<S, NR, STAGE, 1>(g, src, dst, acc, eps, par, i);
      break;
    case 2:
      flow_link<S, NR, STAGE, 2>(g, src, dst, acc, eps, par, i);
      break;
    default:
      flow_link<S, NR, STAGE, 3>(g, src, dst, acc, eps, par, i);
      break;
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
  dim3 grid(grid_for(Ls.g.Vh, block), 8);
  if (stage == 1)
    k_flow_stage<S, NR, 1><<<grid, block, 0, s>>>(Ls.g, src, dst, acc, S(eps));
  else if (stage == 2)
    k_flow_stage<S, NR, 2><<<grid, block, 0, s>>>(Ls.g, src, dst, acc, S(eps));
  else
    k_flow_stage<S, NR, 3><<<grid, block, 0, s>>>(Ls.g, src, dst, acc, S(eps));
  return cudaGetLastError();
}

cudaError_t launch_flow_stage(int stage, const LatDev& src, const LatDev& dst, const AlgDev& z, double eps,
                              cudaStream_t s, int block) {
  if (block <= 0) block = 128;
  if (src.prec != dst.prec || src.nr != dst.nr) return cudaErrorInvalidValue;
  QCB_DISPATCH_STORE(src, flow_impl, stage, src, dst, z, eps, s, block);
}

}  // namespace qcb
