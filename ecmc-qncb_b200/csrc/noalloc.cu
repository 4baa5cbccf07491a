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
// address, so every call looks up its device address with cudaGetSymbolAddress (with the
// caller's device current; the lookup allocates nothing) and passes that to the kernels.
// Looking it up on every call, rather than caching it per device, keeps the address right
// when the host application resets the device and the module is loaded again.  The first
// call on a device loads the module, so it should come before any stream capture.  Every
// call shares the array; calls whose kernels overlap on the GPU race on it.  Nothing in it
// needs to start at zero: each launch writes every partial it later reads.
#include <stdint.h>

#include "../../include/qcb.h"
#include "kernels.h"

namespace {

static __device__ __align__(256) double g_noalloc_scratch[QCB_NOALLOC_MAX_PARTIALS];

__global__ void k_mean(double* out, double inv_count) { out[0] *= inv_count; }

}  // namespace

extern "C" int qcb_plaquette_noalloc(const void* links, const int dims[4], int precision, int storage, size_t stride,
                                     double* out, void* stream) {
  using namespace qcb;
  if (!links || !dims || !out) return set_error(QCB_ERR_INVALID, "null argument");
  // The kernels read a link chunk as one 16-byte vector (8 bytes for FP32 18-real storage)
  // and write one double: a sub-allocated pointer off those boundaries would fault the device.
  const uintptr_t chunk = (precision == QCB_FP32 && storage == QCB_R18) ? 8 : 16;
  if ((uintptr_t)links % chunk)
    return set_error(QCB_ERR_INVALID, "links must be aligned to the storage's chunk size (16 bytes; 8 for FP32 18-real)");
  if ((uintptr_t)out % alignof(double)) return set_error(QCB_ERR_INVALID, "out must be 8-byte aligned");
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

  double* scratch = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&scratch, g_noalloc_scratch);
  if (e != cudaSuccess) return set_error(QCB_ERR_CUDA, cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = launch_plaquette_partials(L, nblocks, scratch, out, s);
  if (e == cudaSuccess) {
    k_mean<<<1, 1, 0, s>>>(out, 1.0 / (6.0 * (double)vol));
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return set_error(QCB_ERR_CUDA, cudaGetErrorString(e));
  return QCB_OK;
}
