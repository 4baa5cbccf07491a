// noalloc.cu — mean plaquette of links already on the device, for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: a host application whose memory manager owns all of
// the device memory (a pool or caching allocator, as serving runtimes and ML frameworks
// use), or a latency-critical loop in which an allocation is not acceptable because
// cudaMalloc/cudaFree can synchronise the device and stall the work of other streams.  The
// ordinary entry points allocate through their context (qcb_ctx_create allocates its
// reduction scratch).  This one allocates nothing: the caller passes the link storage and a
// device double for the result, and the reduction's scratch (one FP64 partial sum per
// reduction block) lives in the file-scope device array below, which every GPU that loads
// the library holds until the process exits.
//
// The array's name in host code is only a host-side stand-in for the symbol, not a device
// address, so its device address is looked up once per device with cudaGetSymbolAddress
// (with that device current) on the first call there, and passed to the kernels.  Every
// call shares the array; calls whose kernels overlap on the GPU race on it.  Nothing in it
// needs to start at zero: each launch writes every partial it later reads.
#include <mutex>

#include "../../include/qcb.h"
#include "kernels.h"

namespace {

static __device__ __align__(256) double g_noalloc_scratch[QCB_NOALLOC_MAX_PARTIALS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_addr[MAX_DEVICES] = {};

__global__ void k_mean(double* out, double inv_count) { out[0] *= inv_count; }

}  // namespace

extern "C" int qcb_plaquette_noalloc(const void* links, const int dims[4], int precision, int storage, size_t stride,
                                     double* out, void* stream) {
  using namespace qcb;
  if (!links || !dims || !out) return set_error(QCB_ERR_INVALID, "null argument");
  uint64_t vol = 1;
  for (int d = 0; d < 4; ++d) {
    if (dims[d] < 2 || (dims[d] & 1)) return set_error(QCB_ERR_INVALID, "lattice extents must be even and >= 2");
    vol *= (uint64_t)dims[d];
  }
  if (vol >= (1ull << 30)) return set_error(QCB_ERR_INVALID, "lattice volume must be below 2^30");
  if (precision != QCB_FP64 && precision != QCB_FP32) return set_error(QCB_ERR_INVALID, "bad precision");
  if (storage != QCB_R18 && storage != QCB_R12) return set_error(QCB_ERR_INVALID, "bad storage");
  LatDev L;
  L.g = make_geom(dims);
  if (stride < L.g.Vh) return set_error(QCB_ERR_INVALID, "stride is smaller than half the lattice volume");
  if (stride > 0xffffffffull) return set_error(QCB_ERR_INVALID, "stride too large");
  L.g.stride = (uint32_t)stride;
  L.prec = precision;
  L.nr = storage;
  L.links = const_cast<void*>(links);

  // One partial per reduction block; the grid never exceeds the library's reduction grid.
  const uint64_t want = (vol + (uint64_t)reduce_threads() - 1) / (uint64_t)reduce_threads();
  const int nblocks = (int)(want < (uint64_t)reduce_blocks() ? want : (uint64_t)reduce_blocks());
  if (nblocks > QCB_NOALLOC_MAX_PARTIALS)
    return set_error(QCB_ERR_INVALID, "reduction needs more partial sums than the static scratch holds");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(QCB_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return set_error(QCB_ERR_INVALID, "device index above the supported range");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
      double* p = nullptr;
      e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
      if (e != cudaSuccess) return set_error(QCB_ERR_CUDA, cudaGetErrorString(e));
      g_scratch_addr[dev] = p;
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = launch_plaquette_partials(L, nblocks, scratch, out, s);
  if (e == cudaSuccess) {
    k_mean<<<1, 1, 0, s>>>(out, 1.0 / (6.0 * (double)vol));
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return set_error(QCB_ERR_CUDA, cudaGetErrorString(e));
  return QCB_OK;
}
