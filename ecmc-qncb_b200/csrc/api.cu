// api.cu — C ABI (include/qcb.h): contexts, lattices, and the drop-in entry points.
#include <errno.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/qcb.h"
#include "api_internal.h"
#include "host_io.h"
#include "kernels.h"

using namespace qcb;

// ---- error state -------------------------------------------------------------------------
namespace {
thread_local std::string t_err;

int fail(int code, const std::string& msg) {
  t_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  t_err = std::string(what) + ": " + cudaGetErrorString(e);
  return QCB_ERR_CUDA;
}
}  // namespace

int qcb::set_error(int code, const char* msg) { return fail(code, msg); }

#define CU(call, what)                               \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

namespace {
constexpr size_t STAGE_BYTES = 64ull << 20;

int set_device(qcb_ctx* c) {
  CU(cudaSetDevice(c->device), "cudaSetDevice");
  return QCB_OK;
}

}  // namespace

// Reads and clears the device status words; reports KP cap hits.
int qcb::check_status(qcb_ctx* c) {
  CU(cudaMemcpyAsync(c->h_status, c->d_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
     "status copy");
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  uint32_t kp = c->h_status[0];
  const uint32_t timeouts = c->h_status[1], aborted = c->h_status[2];
  if (timeouts || aborted) {
    CU(cudaMemsetAsync(c->d_status, 0, 4 * sizeof(uint32_t), c->stream), "status reset");
    CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return fail(QCB_ERR_CUDA, "a persistent kernel gave up waiting (" + std::to_string(timeouts) +
                                  " wait timeout(s)); the launch was abandoned");
  }
  if (kp) {
    CU(cudaMemsetAsync(c->d_status, 0, 4 * sizeof(uint32_t), c->stream), "status reset");
    CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return fail(QCB_ERR_KP_CAP, "Kennedy-Pendleton draw hit its attempt cap " + std::to_string(kp) +
                                    " time(s); those SU(2) updates were skipped");
  }
  return QCB_OK;
}

namespace {
int valid_dims(const int dims[4]) {
  if (!dims) return 0;
  uint64_t v = 1;
  for (int d = 0; d < 4; ++d) {
    if (dims[d] < 2 || (dims[d] & 1)) return 0;
    v *= (uint64_t)dims[d];
  }
  return v < (1ull << 30);  // link ids mu*V + s must fit in 32 bits
}

}  // namespace

int qcb::ensure_flow_space(qcb_lattice* L) {
  if (L->fw[0]) return QCB_OK;
  const size_t lb = link_bytes(L->dev.g, L->dev.prec, L->dev.nr);
  const size_t ab = alg_bytes(L->dev.g, L->dev.prec);
  if (cudaMalloc(&L->fw[0], lb) != cudaSuccess || cudaMalloc(&L->fw[1], lb) != cudaSuccess ||
      cudaMalloc(&L->fz, ab) != cudaSuccess) {
    cudaFree(L->fw[0]);
    cudaFree(L->fw[1]);
    cudaFree(L->fz);
    L->fw[0] = L->fw[1] = L->fz = nullptr;
    cudaGetLastError();
    return fail(QCB_ERR_NOMEM, "cannot allocate Wilson-flow work space");
  }
  return QCB_OK;
}

namespace {
LatDev with_links(const LatDev& d, void* p) {
  LatDev r = d;
  r.links = p;
  return r;
}

// One RK3 step with the three fused stages: a -> b -> a -> b.  The step's input in `a`
// is overwritten by stage 2 (stage 1 has consumed it); the result is in `b`.
int rk3(qcb_lattice* L, const LatDev& a, const LatDev& b, double eps) {
  qcb_ctx* c = L->ctx;
  AlgDev z;
  z.p = L->fz;
  CU(launch_flow_stage(1, a, b, z, eps, c->stream, c->block), "flow stage 1");
  CU(launch_flow_stage(2, b, a, z, eps, c->stream, c->block), "flow stage 2");
  CU(launch_flow_stage(3, a, b, z, eps, c->stream, c->block), "flow stage 3");
  c->launches += 3;
  return QCB_OK;
}

// Device buffer of at least `need` doubles for the partial sums of fused measurements.
int ensure_meas(qcb_lattice* L, size_t need) {
  if (L->meas_n >= need) return QCB_OK;
  cudaFree(L->meas);
  L->meas = nullptr;
  L->meas_n = 0;
  if (cudaMalloc(&L->meas, need * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(QCB_ERR_NOMEM, "cannot allocate the measurement partial sums");
  }
  L->meas_n = need;
  return QCB_OK;
}

// One RK3 step a -> b as rk3(), with the clover (Q, E) of the step's input summed inside
// stage 1 and written to dst_dev[0..1] (FP32 whole lattices: one thread per site).
int rk3_qe(qcb_lattice* L, const LatDev& a, const LatDev& b, double eps, double* dst_dev) {
  qcb_ctx* c = L->ctx;
  AlgDev z;
  z.p = L->fz;
  const int nb = flow_site_blocks(a);
  const int r_ = ensure_meas(L, 2 * (size_t)nb + 512);
  if (r_ != QCB_OK) return r_;
  CU(launch_flow_site_qe(a, b, z, eps, L->meas, c->stream), "flow stage 1 with Q/E");
  CU(launch_qe_from_parts(L->meas, nb, L->meas + 2 * nb, dst_dev, 1.0 / (double)a.g.Vg, c->stream), "Q/E sums");
  CU(launch_flow_stage(2, b, a, z, eps, c->stream, c->block), "flow stage 2");
  CU(launch_flow_stage(3, a, b, z, eps, c->stream, c->block), "flow stage 3");
  c->launches += 6;
  return QCB_OK;
}

int qe_async(qcb_lattice* L, const LatDev& d, double* dst_dev) {
  qcb_ctx* c = L->ctx;
  CU(launch_clover_qe(d, c->d_scratch, dst_dev, c->stream, c->block), "clover Q/E");
  c->launches += 3;
  return QCB_OK;
}
}  // namespace

#define CHECK_CTX(c) \
  if (!(c)) return fail(QCB_ERR_INVALID, "null context")
#define CHECK_LAT(l) \
  if (!(l)) return fail(QCB_ERR_INVALID, "null lattice")
#define LOCK(c) std::lock_guard<std::mutex> lk_((c)->mu)
#define TRY(x)                \
  do {                        \
    int r_ = (x);             \
    if (r_ != QCB_OK) return r_; \
  } while (0)

extern "C" {

int qcb_abi_version(void) { return QCB_ABI_VERSION; }
const char* qcb_last_error(void) { return t_err.c_str(); }

int qcb_device_count(int* count) {
  if (!count) return fail(QCB_ERR_INVALID, "null count");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return QCB_OK;
}

int qcb_ctx_create(int device, unsigned flags, qcb_ctx** out) {
  (void)flags;
  if (!out) return fail(QCB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(QCB_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= n) return fail(QCB_ERR_INVALID, "device index out of range");
  qcb_ctx* c = new (std::nothrow) qcb_ctx();
  if (!c) return fail(QCB_ERR_NOMEM, "host allocation failed");
  c->device = device;
  auto cleanup = [&](int code) {
    qcb_ctx_destroy(c);
    return code;
  };
  if (set_device(c) != QCB_OK) return cleanup(QCB_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_status, 4 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMallocHost(&c->h_status, 4 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->d_scratch, 4 * (size_t)reduce_blocks() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_out, 64 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&c->h_out, 64 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    t_err = "context allocation failed";
    return cleanup(QCB_ERR_NOMEM);
  }
  if (cudaMemset(c->d_status, 0, 4 * sizeof(uint32_t)) != cudaSuccess) return cleanup(QCB_ERR_CUDA);
  *out = c;
  return QCB_OK;
}

}  // extern "C"

namespace {
void ctx_free(qcb_ctx* c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_status);
  cudaFreeHost(c->h_status);
  cudaFree(c->d_scratch);
  cudaFree(c->d_out);
  cudaFreeHost(c->h_out);
  cudaFree(c->d_stage[0]);
  cudaFree(c->d_stage[1]);
  cudaFreeHost(c->h_stage);
  if (c->stream) cudaStreamDestroy(c->stream);
  cudaGetLastError();
  delete c;
}
}  // namespace

void qcb::ctx_ref(qcb_ctx* c) {
  std::lock_guard<std::mutex> lk(c->mu);
  c->refs++;
}

void qcb::ctx_unref(qcb_ctx* c) {
  bool free_now = false;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    c->refs--;
    free_now = c->doomed && c->refs == 0;
  }
  if (free_now) ctx_free(c);
}

extern "C" {

int qcb_ctx_destroy(qcb_ctx* c) {
  if (!c) return QCB_OK;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->refs > 0) {
      c->doomed = true;  // freed by the last child's destroy
      return QCB_OK;
    }
  }
  ctx_free(c);
  return QCB_OK;
}

int qcb_ctx_sync(qcb_ctx* c) {
  CHECK_CTX(c);
  LOCK(c);
  TRY(set_device(c));
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return check_status(c);
}

int qcb_ctx_launch_count(qcb_ctx* c, uint64_t* count) {
  CHECK_CTX(c);
  if (!count) return fail(QCB_ERR_INVALID, "null count");
  *count = c->launches;
  return QCB_OK;
}

int qcb_ctx_set_block(qcb_ctx* c, int threads) {
  CHECK_CTX(c);
  if (threads != 0 && (threads < 32 || threads > 1024 || (threads & 31)))
    return fail(QCB_ERR_INVALID, "block size must be 0 or a multiple of 32 in [32, 1024]");
  // the per-link kernels declare __launch_bounds__(128)
  if (threads > 128) return fail(QCB_ERR_INVALID, "block size above 128 is not supported by the link kernels");
  c->block = threads;
  return QCB_OK;
}

int qcb_ctx_stream(qcb_ctx* c, void** stream) {
  CHECK_CTX(c);
  if (!stream) return fail(QCB_ERR_INVALID, "null stream pointer");
  *stream = (void*)c->stream;
  return QCB_OK;
}

int qcb_lattice_create(qcb_ctx* c, const int dims[4], int precision, int storage, qcb_lattice** out) {
  CHECK_CTX(c);
  if (!out) return fail(QCB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!valid_dims(dims)) return fail(QCB_ERR_INVALID, "lattice extents must be even, >= 2, volume < 2^30");
  if (precision != QCB_FP64 && precision != QCB_FP32) return fail(QCB_ERR_INVALID, "bad precision");
  if (storage != QCB_R18 && storage != QCB_R12) return fail(QCB_ERR_INVALID, "bad storage");
  LOCK(c);
  TRY(set_device(c));
  qcb_lattice* L = new (std::nothrow) qcb_lattice();
  if (!L) return fail(QCB_ERR_NOMEM, "host allocation failed");
  L->ctx = c;
  L->dev.g = make_geom(dims);
  L->dev.prec = precision;
  L->dev.nr = storage;
  L->bytes = link_bytes(L->dev.g, precision, storage);
  if (cudaMalloc(&L->dev.links, L->bytes) != cudaSuccess) {
    cudaGetLastError();
    const size_t bytes = L->bytes;
    delete L;
    return fail(QCB_ERR_NOMEM, "cannot allocate " + std::to_string(bytes) + " bytes of link storage");
  }
  {
    cudaError_t e = cudaMemsetAsync(L->dev.links, 0, L->bytes, c->stream);
    if (e == cudaSuccess) e = launch_cold(L->dev, c->stream, 0);
    if (e != cudaSuccess) {
      cudaFree(L->dev.links);
      delete L;
      return cuda_fail(e, "lattice initialisation");
    }
  }
  c->launches++;
  c->refs++;  // under the context lock
  *out = L;
  return QCB_OK;
}

int qcb_lattice_create_slab(qcb_ctx* c, const int global_dims[4], int t0, int t_local, int precision, int storage,
                            qcb_lattice** out) {
  CHECK_CTX(c);
  if (!out) return fail(QCB_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (!valid_dims(global_dims)) return fail(QCB_ERR_INVALID, "lattice extents must be even, >= 2, volume < 2^30");
  if (t_local < 2 || (t_local & 1) || (t0 & 1) || t0 < 0 || t0 + t_local > global_dims[3])
    return fail(QCB_ERR_INVALID, "slab times must be even, t_local >= 2, t0 >= 0 and t0 + t_local <= Lt");
  if (precision != QCB_FP64 && precision != QCB_FP32) return fail(QCB_ERR_INVALID, "bad precision");
  if (storage != QCB_R18 && storage != QCB_R12) return fail(QCB_ERR_INVALID, "bad storage");
  LOCK(c);
  TRY(set_device(c));
  qcb_lattice* L = new (std::nothrow) qcb_lattice();
  if (!L) return fail(QCB_ERR_NOMEM, "host allocation failed");
  L->ctx = c;
  L->dev.g = make_slab_geom(global_dims, t0, t_local);
  L->dev.prec = precision;
  L->dev.nr = storage;
  for (int d = 0; d < 4; ++d) L->gdims[d] = global_dims[d];
  L->slab_t0 = t0;
  L->slab_tl = t_local;
  L->bytes = link_bytes(L->dev.g, precision, storage);
  if (cudaMalloc(&L->dev.links, L->bytes) != cudaSuccess) {
    cudaGetLastError();
    const size_t bytes = L->bytes;
    delete L;
    return fail(QCB_ERR_NOMEM, "cannot allocate " + std::to_string(bytes) + " bytes of link storage");
  }
  {
    cudaError_t e = cudaMemsetAsync(L->dev.links, 0, L->bytes, c->stream);
    if (e == cudaSuccess) e = launch_cold(L->dev, c->stream, 0);
    if (e != cudaSuccess) {
      cudaFree(L->dev.links);
      delete L;
      return cuda_fail(e, "lattice initialisation");
    }
  }
  c->launches++;
  c->refs++;
  *out = L;
  return QCB_OK;
}

int qcb_lattice_destroy(qcb_lattice* L) {
  if (!L) return QCB_OK;
  qcb_ctx* c = L->ctx;
  {
    LOCK(c);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFree(L->dev.links);
    cudaFree(L->fw[0]);
    cudaFree(L->fw[1]);
    cudaFree(L->fz);
    cudaFree(L->meas);
    cudaGetLastError();
  }
  delete L;
  ctx_unref(c);
  return QCB_OK;
}

int qcb_lattice_info(const qcb_lattice* L, int dims[4], int* precision, int* storage, size_t* device_bytes) {
  CHECK_LAT(L);
  if (dims)
    for (int d = 0; d < 4; ++d) dims[d] = L->dev.g.L[d];
  if (precision) *precision = L->dev.prec;
  if (storage) *storage = L->dev.nr;
  if (device_bytes) {
    size_t b = L->bytes;
    if (L->fw[0]) b += 2 * L->bytes + alg_bytes(L->dev.g, L->dev.prec);
    *device_bytes = b;
  }
  return QCB_OK;
}

int qcb_lattice_device_links(const qcb_lattice* L, void** dev_ptr, size_t* stride, int* nchunk, int* chunk_bytes) {
  CHECK_LAT(L);
  if (dev_ptr) *dev_ptr = L->dev.links;
  if (stride) *stride = L->dev.g.stride;
  const int es = L->dev.prec == QCB_FP64 ? 8 : 4;
  const int cw = (L->dev.prec == QCB_FP32 && L->dev.nr == 12) ? 4 : 2;
  if (nchunk) *nchunk = L->dev.nr / cw;
  if (chunk_bytes) *chunk_bytes = cw * es;
  return QCB_OK;
}

int qcb_cold_start(qcb_lattice* L) {
  CHECK_LAT(L);
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  CU(launch_cold(L->dev, c->stream, 0), "cold start");
  c->launches++;
  return QCB_OK;
}

int qcb_hot_start(qcb_lattice* L, uint64_t seed) {
  CHECK_LAT(L);
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  CU(launch_hot(L->dev, seed, c->stream, 0), "hot start");
  c->launches++;
  return QCB_OK;
}

int qcb_reunitarize(qcb_lattice* L) {
  CHECK_LAT(L);
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  CU(launch_reunitarize(L->dev, c->stream, 0), "reunitarize");
  c->launches++;
  return QCB_OK;
}

int qcb_gauge_transform(qcb_lattice* L, uint64_t seed) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  CU(launch_gauge_transform(L->dev, seed, c->stream, 0), "gauge transform");
  c->launches++;
  return QCB_OK;
}

}  // extern "C"

// ---- AoS transfers (host <-> device in site chunks through two staging buffers) ------
namespace {
constexpr uint32_t STAGE_SITES = (uint32_t)(STAGE_BYTES / (72 * sizeof(double)));

int ensure_stage(qcb_ctx* c) {
  if (c->d_stage[0]) return QCB_OK;
  if (cudaMalloc(&c->d_stage[0], STAGE_BYTES) != cudaSuccess ||
      cudaMalloc(&c->d_stage[1], STAGE_BYTES) != cudaSuccess) {
    cudaFree(c->d_stage[0]);
    c->d_stage[0] = nullptr;
    cudaGetLastError();
    return fail(QCB_ERR_NOMEM, "cannot allocate staging buffers");
  }
  c->stage_bytes = STAGE_BYTES;
  return QCB_OK;
}

int ensure_host_stage(qcb_ctx* c) {
  if (c->h_stage) return QCB_OK;
  if (cudaMallocHost(&c->h_stage, STAGE_BYTES) != cudaSuccess) {
    cudaGetLastError();
    return fail(QCB_ERR_NOMEM, "cannot allocate pinned staging buffer");
  }
  return QCB_OK;
}

// host -> device; `host` holds the whole lattice (72*V doubles).  Copies and conversions of
// consecutive chunks alternate between the two device staging buffers (stream-ordered).
int upload_aos(qcb_lattice* L, const double* host, int bswap) {
  qcb_ctx* c = L->ctx;
  TRY(ensure_stage(c));
  const uint32_t V = L->dev.g.V;
  int k = 0;
  for (uint32_t s0 = 0; s0 < V; s0 += STAGE_SITES, k ^= 1) {
    const uint32_t n = (V - s0 < STAGE_SITES) ? V - s0 : STAGE_SITES;
    CU(cudaMemcpyAsync(c->d_stage[k], host + (size_t)s0 * 72, (size_t)n * 72 * sizeof(double),
                       cudaMemcpyHostToDevice, c->stream),
       "H2D copy");
    CU(launch_aos_to_soa(L->dev, c->d_stage[k], s0, n, bswap, c->stream, 0), "AoS->SoA");
    c->launches++;
  }
  return QCB_OK;
}

int download_aos(qcb_lattice* L, double* host, int bswap) {
  qcb_ctx* c = L->ctx;
  TRY(ensure_stage(c));
  const uint32_t V = L->dev.g.V;
  int k = 0;
  for (uint32_t s0 = 0; s0 < V; s0 += STAGE_SITES, k ^= 1) {
    const uint32_t n = (V - s0 < STAGE_SITES) ? V - s0 : STAGE_SITES;
    CU(launch_soa_to_aos(L->dev, c->d_stage[k], s0, n, bswap, c->stream, 0), "SoA->AoS");
    c->launches++;
    CU(cudaMemcpyAsync(host + (size_t)s0 * 72, c->d_stage[k], (size_t)n * 72 * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream),
       "D2H copy");
  }
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return QCB_OK;
}
}  // namespace

extern "C" {

int qcb_set_links(qcb_lattice* L, const double* aos) {
  CHECK_LAT(L);
  if (!aos) return fail(QCB_ERR_INVALID, "null host buffer");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(upload_aos(L, aos, 0));
  // the caller's buffer is only borrowed for the duration of the call
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return QCB_OK;
}

int qcb_get_links(qcb_lattice* L, double* aos) {
  CHECK_LAT(L);
  if (!aos) return fail(QCB_ERR_INVALID, "null host buffer");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  return download_aos(L, aos, 0);
}

int qcb_copy_links(qcb_lattice* dst, const qcb_lattice* src) {
  CHECK_LAT(dst);
  CHECK_LAT(src);
  if (dst->ctx != src->ctx) return fail(QCB_ERR_INVALID, "lattices belong to different contexts");
  for (int d = 0; d < 4; ++d)
    if (dst->dev.g.L[d] != src->dev.g.L[d]) return fail(QCB_ERR_INVALID, "lattice extents differ");
  qcb_ctx* c = dst->ctx;
  LOCK(c);
  TRY(set_device(c));
  if (dst->dev.prec == src->dev.prec && dst->dev.nr == src->dev.nr) {
    CU(cudaMemcpyAsync(dst->dev.links, src->dev.links, dst->bytes, cudaMemcpyDeviceToDevice, c->stream), "D2D copy");
  } else {
    CU(launch_convert(dst->dev, src->dev, c->stream, 0), "convert");
    c->launches++;
  }
  return QCB_OK;
}

// ---- ILDG -----------------------------------------------------------------------------------
int qcb_ildg_probe(const char* path, uint64_t* data_offset, uint64_t* data_bytes) {
  if (!path || !data_offset || !data_bytes) return fail(QCB_ERR_INVALID, "null argument");
  FILE* fp = fopen(path, "rb");
  if (!fp) return fail(QCB_ERR_IO, std::string("cannot open ") + path + ": " + strerror(errno));
  std::string err;
  int r = lime_find(fp, "ildg-binary-data", data_offset, data_bytes, &err);
  fclose(fp);
  if (r != QCB_OK) return fail(r, std::string(path) + ": " + err);
  return QCB_OK;
}

int qcb_save_ildg(qcb_lattice* L, const char* path) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (!path) return fail(QCB_ERR_INVALID, "null path");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  const Geom& g = L->dev.g;
  const uint64_t nbytes = (uint64_t)g.V * 72 * sizeof(double);
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(QCB_ERR_IO, std::string("cannot open ") + path + " for writing: " + strerror(errno));
  const std::string xml = ildg_xml(g.L);
  bool ok = lime_write_header(fp, true, true, "ildg-format", xml.size()) &&
            fwrite(xml.data(), 1, xml.size(), fp) == xml.size() && lime_write_padding(fp, xml.size()) &&
            lime_write_header(fp, false, true, "ildg-binary-data", nbytes);
  if (!ok) {
    fclose(fp);
    return fail(QCB_ERR_IO, std::string("write failed: ") + path);
  }
  int r = ensure_stage(c);
  if (r == QCB_OK) r = ensure_host_stage(c);
  if (r != QCB_OK) {
    fclose(fp);
    return r;
  }
  for (uint32_t s0 = 0; s0 < g.V; s0 += STAGE_SITES) {
    const uint32_t n = (g.V - s0 < STAGE_SITES) ? g.V - s0 : STAGE_SITES;
    const size_t bytes = (size_t)n * 72 * sizeof(double);
    cudaError_t e = launch_soa_to_aos(L->dev, c->d_stage[0], s0, n, 1, c->stream, 0);
    c->launches++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->h_stage, c->d_stage[0], bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      fclose(fp);
      return cuda_fail(e, "ILDG download");
    }
    if (fwrite(c->h_stage, 1, bytes, fp) != bytes) {
      fclose(fp);
      return fail(QCB_ERR_IO, std::string("write failed: ") + path);
    }
  }
  if (fclose(fp) != 0) return fail(QCB_ERR_IO, std::string("close failed: ") + path);
  return QCB_OK;
}

int qcb_load_ildg(qcb_lattice* L, const char* path) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (!path) return fail(QCB_ERR_INVALID, "null path");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  const Geom& g = L->dev.g;
  const uint64_t expected = (uint64_t)g.V * 72 * sizeof(double);
  FILE* fp = fopen(path, "rb");
  if (!fp) return fail(QCB_ERR_IO, std::string("cannot open ") + path + ": " + strerror(errno));
  uint64_t off = 0, nbytes = 0;
  std::string err;
  int r = lime_find(fp, "ildg-binary-data", &off, &nbytes, &err);
  if (r != QCB_OK) {
    fclose(fp);
    return fail(r, std::string(path) + ": " + err);
  }
  if (nbytes != expected) {
    fclose(fp);
    return fail(QCB_ERR_FORMAT, std::string(path) + ": binary data size " + std::to_string(nbytes) +
                                    " does not match the lattice (" + std::to_string(expected) + " bytes)");
  }
  r = ensure_stage(c);
  if (r == QCB_OK) r = ensure_host_stage(c);
  if (r != QCB_OK || fseeko(fp, (off_t)off, SEEK_SET) != 0) {
    fclose(fp);
    return r != QCB_OK ? r : fail(QCB_ERR_IO, "seek failed");
  }
  for (uint32_t s0 = 0; s0 < g.V; s0 += STAGE_SITES) {
    const uint32_t n = (g.V - s0 < STAGE_SITES) ? g.V - s0 : STAGE_SITES;
    const size_t bytes = (size_t)n * 72 * sizeof(double);
    cudaError_t e = cudaStreamSynchronize(c->stream);  // h_stage is reused
    if (e != cudaSuccess) {
      fclose(fp);
      return cuda_fail(e, "ILDG upload");
    }
    if (fread(c->h_stage, 1, bytes, fp) != bytes) {
      fclose(fp);
      return fail(QCB_ERR_FORMAT, std::string(path) + ": truncated binary data");
    }
    e = cudaMemcpyAsync(c->d_stage[0], c->h_stage, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_aos_to_soa(L->dev, c->d_stage[0], s0, n, 1, c->stream, 0);
    c->launches++;
    if (e != cudaSuccess) {
      fclose(fp);
      return cuda_fail(e, "ILDG upload");
    }
  }
  fclose(fp);
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return QCB_OK;
}

// ---- heatbath ---------------------------------------------------------------------------------
int qcb_heatbath(qcb_lattice* L, double beta, int n_sweeps, int n_hits, uint64_t seed, uint64_t sweep_offset) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (n_sweeps < 0 || n_hits < 0) return fail(QCB_ERR_INVALID, "negative sweep or hit count");
  if (!(beta > 0.0)) return fail(QCB_ERR_INVALID, "beta must be positive");
  if (n_hits > (1 << 20)) return fail(QCB_ERR_INVALID, "too many hits");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  for (int s = 0; s < n_sweeps; ++s) {
    const uint32_t sweep = (uint32_t)(sweep_offset + (uint64_t)s);
    for (int mu = 0; mu < 4; ++mu)
      for (int par = 0; par < 2; ++par) {
        CU(launch_hb_pass(L->dev, mu, par, beta, seed, sweep, n_hits, c->d_status, c->stream, c->block),
           "heatbath pass");
        c->launches++;
      }
  }
  return QCB_OK;
}

int qcb_heatbath_plaquette(qcb_lattice* L, double beta, int n_sweeps, int n_hits, uint64_t seed,
                           uint64_t sweep_offset, double* plaq) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (!plaq) return fail(QCB_ERR_INVALID, "null output");
  if (n_sweeps < 0 || n_hits < 0) return fail(QCB_ERR_INVALID, "negative sweep or hit count");
  if (!(beta > 0.0)) return fail(QCB_ERR_INVALID, "beta must be positive");
  if (n_hits > (1 << 20)) return fail(QCB_ERR_INVALID, "too many hits");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  if (n_sweeps == 0) {
    CU(launch_plaquette(L->dev, c->d_scratch, c->d_out, c->stream, c->block), "plaquette");
    c->launches += 2;
  } else {
    const int nb = hb_meas_blocks(L->dev);
    TRY(ensure_meas(L, 2 * (size_t)nb + 256));
    for (int s = 0; s < n_sweeps; ++s) {
      const uint32_t sweep = (uint32_t)(sweep_offset + (uint64_t)s);
      const bool last = s == n_sweeps - 1;
      for (int mu = 0; mu < 4; ++mu)
        for (int par = 0; par < 2; ++par) {
          if (last && mu == 3) {
            CU(launch_hb_pass_meas(L->dev, par, beta, seed, sweep, n_hits, c->d_status, L->meas + (size_t)par * nb,
                                   c->stream),
               "measuring heatbath pass");
          } else {
            CU(launch_hb_pass(L->dev, mu, par, beta, seed, sweep, n_hits, c->d_status, c->stream, c->block),
               "heatbath pass");
          }
          c->launches++;
        }
    }
    CU(launch_sum_parts(L->meas, 2 * nb, L->meas + 2 * nb, c->d_out, c->stream), "plaquette sum");
    c->launches += 2;
  }
  CU(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
  TRY(check_status(c));
  // the measuring passes sum Re tr P; the plaquette kernel sums Re tr P / 3
  const double scale = n_sweeps == 0 ? 1.0 : 1.0 / 3.0;
  *plaq = c->h_out[0] * scale / (6.0 * (double)L->dev.g.Vg);
  return QCB_OK;
}

int qcb_heatbath_frozen(qcb_lattice* L, double beta, int n_sweeps, int n_hits, uint64_t seed, uint64_t sweep_offset,
                        int l_core, const int shift[4]) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (n_sweeps < 0 || n_hits < 0) return fail(QCB_ERR_INVALID, "negative sweep or hit count");
  if (!(beta > 0.0)) return fail(QCB_ERR_INVALID, "beta must be positive");
  if (n_hits > (1 << 20)) return fail(QCB_ERR_INVALID, "too many hits");
  if (!shift) return fail(QCB_ERR_INVALID, "null shift");
  if (l_core < 1) return fail(QCB_ERR_INVALID, "l_core must be positive");
  for (int d = 0; d < 4; ++d)
    if (L->dev.g.L[d] % l_core != 0) return fail(QCB_ERR_INVALID, "l_core must divide every extent");
  int fr[5] = {l_core, 0, 0, 0, 0};
  for (int d = 0; d < 4; ++d) fr[1 + d] = ((shift[d] % l_core) + l_core) % l_core;
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  for (int s = 0; s < n_sweeps; ++s) {
    const uint32_t sweep = (uint32_t)(sweep_offset + (uint64_t)s);
    for (int mu = 0; mu < 4; ++mu)
      for (int par = 0; par < 2; ++par) {
        CU(launch_hb_pass(L->dev, mu, par, beta, seed, sweep, n_hits, c->d_status, c->stream, c->block, fr),
           "heatbath pass");
        c->launches++;
      }
  }
  return QCB_OK;
}

int qcb_translate(qcb_lattice* L, const int shift[4]) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (!shift) return fail(QCB_ERR_INVALID, "null shift");
  int sh[4];
  for (int d = 0; d < 4; ++d) sh[d] = ((shift[d] % L->dev.g.L[d]) + L->dev.g.L[d]) % L->dev.g.L[d];
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(ensure_flow_space(L));
  const LatDev tmp = with_links(L->dev, L->fw[0]);
  CU(launch_translate(tmp, L->dev, sh, c->stream, 0), "translate");
  c->launches++;
  CU(cudaMemcpyAsync(L->dev.links, L->fw[0], L->bytes, cudaMemcpyDeviceToDevice, c->stream), "translate copy");
  return QCB_OK;
}

// ---- observables ---------------------------------------------------------------------------
int qcb_plaquette(qcb_lattice* L, double* out) {
  CHECK_LAT(L);
  if (!out) return fail(QCB_ERR_INVALID, "null output");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  CU(launch_plaquette(L->dev, c->d_scratch, c->d_out, c->stream, c->block), "plaquette");
  c->launches += 2;
  CU(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
  TRY(check_status(c));
  *out = c->h_out[0] / (6.0 * (double)L->dev.g.Vg);
  return QCB_OK;
}

int qcb_topo_qe(qcb_lattice* L, double* q, double* e) {
  CHECK_LAT(L);
  if (!q || !e) return fail(QCB_ERR_INVALID, "null output");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(qe_async(L, L->dev, c->d_out));
  CU(cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
  TRY(check_status(c));
  *q = c->h_out[0];
  *e = c->h_out[1];
  return QCB_OK;
}

// ---- Wilson flow --------------------------------------------------------------------------
int qcb_flow_measure(qcb_lattice* L, double eps, int n_steps_gf, int n_rk_steps, double* tQE) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (n_steps_gf < 0 || n_rk_steps < 0) return fail(QCB_ERR_INVALID, "negative step count");
  if (n_steps_gf > 0 && !tQE) return fail(QCB_ERR_INVALID, "null output");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(ensure_flow_space(L));
  // gf.copy(field): the flow runs on a copy (observables_mpi.cpp:320).
  CU(cudaMemcpyAsync(L->fw[0], L->dev.links, L->bytes, cudaMemcpyDeviceToDevice, c->stream), "D2D copy");
  LatDev a = with_links(L->dev, L->fw[0]);
  LatDev b = with_links(L->dev, L->fw[1]);
  double t = 0.0;
  const int chunk = 32;  // (t, Q, E) records staged in d_out (64 doubles) between host reads
  for (int s0 = 0; s0 < n_steps_gf; s0 += chunk) {
    const int n = (s0 + chunk <= n_steps_gf) ? chunk : n_steps_gf - s0;
    std::vector<double> ts(n);
    for (int k = 0; k < n; ++k) {
      ts[k] = t;
      // FP32: the record is summed inside stage 1 of the group's first RK3 step, which reads
      // the same links; otherwise (FP64, or no step follows) by the clover kernel.
      const bool fused = a.prec == QCB_FP32 && n_rk_steps > 0;
      if (!fused) TRY(qe_async(L, a, c->d_out + 2 * k));
      for (int r = 0; r < n_rk_steps; ++r) {
        if (fused && r == 0)
          TRY(rk3_qe(L, a, b, eps, c->d_out + 2 * k));
        else
          TRY(rk3(L, a, b, eps));
        LatDev tmp = a;
        a = b;
        b = tmp;
        t += eps;
      }
    }
    CU(cudaMemcpyAsync(c->h_out, c->d_out, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
    TRY(check_status(c));
    for (int k = 0; k < n; ++k) {
      tQE[3 * (s0 + k)] = ts[k];
      tQE[3 * (s0 + k) + 1] = c->h_out[2 * k];
      tQE[3 * (s0 + k) + 2] = c->h_out[2 * k + 1];
    }
  }
  return QCB_OK;
}

int qcb_flow_steps(qcb_lattice* L, double eps, int n) {
  CHECK_LAT(L);
  if (L->slab_tl) return fail(QCB_ERR_STATE, "not available on a slab (needs halo exchanges between its passes)");
  if (n < 0) return fail(QCB_ERR_INVALID, "negative step count");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(ensure_flow_space(L));
  // Each RK3 step ping-pongs between the primary buffer and fw[0]; the result is copied
  // back to the primary buffer when it ends up in fw[0].
  LatDev a = L->dev;
  LatDev b = with_links(L->dev, L->fw[0]);
  for (int r = 0; r < n; ++r) {
    TRY(rk3(L, a, b, eps));
    LatDev tmp = a;
    a = b;
    b = tmp;
  }
  if (a.links != L->dev.links)
    CU(cudaMemcpyAsync(L->dev.links, a.links, L->bytes, cudaMemcpyDeviceToDevice, c->stream), "D2D copy");
  return QCB_OK;
}

// ---- slabs: one pass / one stage at a time, halo exchange --------------------------------------
int qcb_heatbath_pass(qcb_lattice* L, int mu, int parity, double beta, int n_hits, uint64_t seed, uint64_t sweep) {
  CHECK_LAT(L);
  if (mu < 0 || mu > 3 || (parity != 0 && parity != 1)) return fail(QCB_ERR_INVALID, "bad direction or parity");
  if (n_hits < 0 || n_hits > (1 << 20)) return fail(QCB_ERR_INVALID, "bad hit count");
  if (!(beta > 0.0)) return fail(QCB_ERR_INVALID, "beta must be positive");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  // local time = global time - t0 + 1, so local parity = global parity + (1 - t0) (mod 2)
  const int local_par = L->slab_tl ? (parity ^ ((L->slab_t0 + 1) & 1)) : parity;
  CU(launch_hb_pass(L->dev, mu, local_par, beta, seed, (uint32_t)sweep, n_hits, c->d_status, c->stream, c->block),
     "heatbath pass");
  c->launches++;
  return QCB_OK;
}

int qcb_flow_stage(qcb_lattice* L, int stage, double eps, int step) {
  CHECK_LAT(L);
  if (stage < 1 || stage > 3 || step < 0) return fail(QCB_ERR_INVALID, "bad stage or step");
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  TRY(ensure_flow_space(L));
  // step s ping-pongs between the links (a) and the work buffer fw[0] (b) as qcb_flow_steps:
  // stage 1 a -> b, stage 2 b -> a, stage 3 a -> b, with a and b swapped for odd s
  const LatDev x = L->dev, y = with_links(L->dev, L->fw[0]);
  const LatDev& a = (step & 1) ? y : x;
  const LatDev& b = (step & 1) ? x : y;
  AlgDev z;
  z.p = L->fz;
  const LatDev& src = (stage == 2) ? b : a;
  const LatDev& dst = (stage == 2) ? a : b;
  CU(launch_flow_stage(stage, src, dst, z, eps, c->stream, c->block), "flow stage");
  c->launches++;
  return QCB_OK;
}

int qcb_flow_finish(qcb_lattice* L, int n_steps) {
  CHECK_LAT(L);
  if (n_steps < 0) return fail(QCB_ERR_INVALID, "negative step count");
  if (!(n_steps & 1)) return QCB_OK;  // the result is already in the links
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  if (!L->fw[0]) return fail(QCB_ERR_STATE, "no flow stage has run on this lattice");
  CU(cudaMemcpyAsync(L->dev.links, L->fw[0], L->bytes, cudaMemcpyDeviceToDevice, c->stream), "D2D copy");
  return QCB_OK;
}

namespace {
// Device pointers of one face of a slab: the NC chunk segments of time slice `slice` for
// links (mu, local parity par) of buffer `which` (0 links, 1 flow work buffer).
int face_segments(qcb_lattice* L, int which, int slice, int mu, int par, char** seg, size_t* bytes, int* nseg) {
  const Geom& g = L->dev.g;
  const int prec_bytes = (L->dev.prec == QCB_FP64) ? 8 : 4;
  const int nc = (L->dev.prec == QCB_FP32 && L->dev.nr == 12) ? 3 : (L->dev.nr == 12 ? 6 : 9);
  const size_t vbytes = (size_t)prec_bytes * (size_t)L->dev.nr / (size_t)nc;  // bytes of one chunk element
  char* base = (char*)(which == 0 ? L->dev.links : L->fw[0]);
  if (!base) return fail(QCB_ERR_STATE, "the flow work buffer does not exist yet");
  const size_t half = (size_t)g.str[3] / 2;  // checkerboard sites of one parity in one time slice
  for (int c = 0; c < nc; ++c)
    seg[c] = base + (((size_t)((mu * 2 + par) * nc + c)) * g.stride + (size_t)slice * half) * vbytes;
  *bytes = half * vbytes;
  *nseg = nc;
  return QCB_OK;
}
}  // namespace

int qcb_slab_info(const qcb_lattice* L, int global_dims[4], int* t0, int* t_local) {
  CHECK_LAT(L);
  if (global_dims)
    for (int d = 0; d < 4; ++d) global_dims[d] = L->slab_tl ? L->gdims[d] : L->dev.g.L[d];
  if (t0) *t0 = L->slab_t0;
  if (t_local) *t_local = L->slab_tl;
  return QCB_OK;
}

int qcb_slab_face(qcb_lattice* L, int which, int side, int mu, int parity, void** segments, size_t* bytes,
                  int* n_segments) {
  CHECK_LAT(L);
  if (!L->slab_tl) return fail(QCB_ERR_STATE, "not a slab");
  if (which < 0 || which > 1 || side < 0 || side > 3 || mu < 0 || mu > 3 || (parity != 0 && parity != 1) ||
      !segments || !bytes || !n_segments)
    return fail(QCB_ERR_INVALID, "bad face arguments");
  const int slice = (side == 0) ? 0 : (side == 1) ? 1 : (side == 2) ? L->slab_tl : L->slab_tl + 1;
  const int par = parity ^ ((L->slab_t0 + 1) & 1);
  char* seg[9];
  TRY(face_segments(L, which, slice, mu, par, seg, bytes, n_segments));
  for (int c = 0; c < *n_segments; ++c) segments[c] = seg[c];
  return QCB_OK;
}

int qcb_slab_face_copy(qcb_lattice* L, int which, int side, int mu, int parity, void* buf, int to_face) {
  CHECK_LAT(L);
  if (!buf) return fail(QCB_ERR_INVALID, "null buffer");
  void* seg[9];
  size_t nb = 0;
  int ns = 0;
  TRY(qcb_slab_face(L, which, side, mu, parity, seg, &nb, &ns));
  qcb_ctx* c = L->ctx;
  LOCK(c);
  TRY(set_device(c));
  char* b = (char*)buf;
  for (int k = 0; k < ns; ++k) {
    if (to_face)
      CU(cudaMemcpyAsync(seg[k], b + (size_t)k * nb, nb, cudaMemcpyDefault, c->stream), "face copy");
    else
      CU(cudaMemcpyAsync(b + (size_t)k * nb, seg[k], nb, cudaMemcpyDefault, c->stream), "face copy");
  }
  CU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  return QCB_OK;
}

int qcb_slab_faces_copy_async(qcb_lattice* L, int which, int side, int mu, int parity, void* buf, int to_face) {
  CHECK_LAT(L);
  if (!buf) return fail(QCB_ERR_INVALID, "null buffer");
  if (!L->slab_tl) return fail(QCB_ERR_STATE, "not a slab");
  if (mu < -1 || mu > 3 || parity < -1 || parity > 1) return fail(QCB_ERR_INVALID, "bad face arguments");
  const int m0 = mu < 0 ? 0 : mu, m1 = mu < 0 ? 3 : mu;
  const int p0 = parity < 0 ? 0 : parity, p1 = parity < 0 ? 1 : parity;
  qcb_ctx* c = L->ctx;
  char* b = (char*)buf;
  for (int m = m0; m <= m1; ++m)
    for (int p = p0; p <= p1; ++p) {
      void* seg[9];
      size_t nb = 0;
      int ns = 0;
      TRY(qcb_slab_face(L, which, side, m, p, seg, &nb, &ns));
      LOCK(c);
      TRY(set_device(c));
      for (int k = 0; k < ns; ++k) {
        if (to_face)
          CU(cudaMemcpyAsync(seg[k], b, nb, cudaMemcpyDefault, c->stream), "face copy");
        else
          CU(cudaMemcpyAsync(b, seg[k], nb, cudaMemcpyDefault, c->stream), "face copy");
        b += nb;
      }
    }
  return QCB_OK;
}

int qcb_slab_exchange(qcb_lattice* lower, qcb_lattice* upper, int which, int mu, int parity) {
  if (!lower || !upper) return fail(QCB_ERR_INVALID, "null lattice");
  if (!lower->slab_tl || !upper->slab_tl) return fail(QCB_ERR_STATE, "not a slab");
  for (int d = 0; d < 4; ++d)
    if (lower->gdims[d] != upper->gdims[d]) return fail(QCB_ERR_INVALID, "slabs of different lattices");
  if (lower->dev.prec != upper->dev.prec || lower->dev.nr != upper->dev.nr)
    return fail(QCB_ERR_INVALID, "slabs of different storage");
  if ((lower->slab_t0 + lower->slab_tl) % lower->gdims[3] != upper->slab_t0)
    return fail(QCB_ERR_INVALID, "upper slab does not follow lower slab in time");
  if (which < 0 || which > 1 || mu < -1 || mu > 3 || parity < -1 || parity > 1)
    return fail(QCB_ERR_INVALID, "bad exchange arguments");
  qcb_ctx* cl = lower->ctx;
  qcb_ctx* cu = upper->ctx;
  // both slabs' work must be done before their faces move; copies run on the lower stream
  {
    LOCK(cu);
    CU(cudaSetDevice(cu->device), "cudaSetDevice");
    CU(cudaStreamSynchronize(cu->stream), "cudaStreamSynchronize");
  }
  LOCK(cl);
  TRY(set_device(cl));
  CU(cudaStreamSynchronize(cl->stream), "cudaStreamSynchronize");
  for (int m = 0; m < 4; ++m) {
    if (mu >= 0 && m != mu) continue;
    for (int p = 0; p < 2; ++p) {
      if (parity >= 0 && p != parity) continue;
      char *lo_last[9], *lo_halo[9], *up_first[9], *up_halo[9];
      size_t nb = 0;
      int ns = 0;
      const int lp = p ^ ((lower->slab_t0 + 1) & 1), up = p ^ ((upper->slab_t0 + 1) & 1);
      TRY(face_segments(lower, which, lower->slab_tl, m, lp, lo_last, &nb, &ns));
      TRY(face_segments(lower, which, lower->slab_tl + 1, m, lp, lo_halo, &nb, &ns));
      TRY(face_segments(upper, which, 1, m, up, up_first, &nb, &ns));
      TRY(face_segments(upper, which, 0, m, up, up_halo, &nb, &ns));
      for (int k = 0; k < ns; ++k) {
        CU(cudaMemcpyPeerAsync(up_halo[k], cu->device, lo_last[k], cl->device, nb, cl->stream), "face copy");
        CU(cudaMemcpyPeerAsync(lo_halo[k], cl->device, up_first[k], cu->device, nb, cl->stream), "face copy");
      }
    }
  }
  CU(cudaStreamSynchronize(cl->stream), "cudaStreamSynchronize");
  return QCB_OK;
}

// ---- input file -----------------------------------------------------------------------------
int qcb_params_default(qcb_hb_params* p) {
  if (!p) return fail(QCB_ERR_INVALID, "null params");
  memset(p, 0, sizeof *p);
  // src/io/params.h:46-63 (RunParamsHbCB) and :19-25 (HbParams)
  p->L_core = 6;
  p->n_core_dims = 2;
  p->cold_start = 1;
  p->N_switch_eo = 3;
  p->N_shift = 2;
  p->seed = 123;
  p->beta = 6.0;
  p->N_samples = 10;
  p->N_hits = 1;
  p->N_sweeps = 1;
  p->N_therm = 100;
  p->topo = 1;
  p->N_shift_plaquette = 2;
  p->N_shift_topo = 10;
  p->N_steps_gf = 10;
  p->N_rk_steps = 40;
  strcpy(p->run_name, "c");
  strcpy(p->run_dir, "data");
  p->save_each_shifts = 2;
  return QCB_OK;
}

int qcb_params_load(const char* path, qcb_hb_params* p) {
  if (!path || !p) return fail(QCB_ERR_INVALID, "null argument");
  std::string err;
  int r = params_load(path, p, &err);
  if (r != QCB_OK) return fail(r, err);
  return QCB_OK;
}

int qcb_ecmc_run_params_default(qcb_ecmc_run_params* p) {
  if (!p) return fail(QCB_ERR_INVALID, "null params");
  memset(p, 0, sizeof *p);
  // src/io/params.h:27-44 (RunParamsECB) and :9-17 (ECMCParams)
  p->L_core = 6;
  p->n_core_dims = 2;
  p->cold_start = 1;
  p->seed = 123;
  p->N_shift = 2;
  p->ecmc.beta = 6.0;
  p->ecmc.theta_sample = 100.0;
  p->ecmc.theta_refresh_site = 50.0;
  p->ecmc.theta_refresh_R = 15.0;
  p->ecmc.poisson = 0;
  p->ecmc.epsilon_set = 0.15;
  p->ecmc.l_core = 6;
  p->N_therm = 100;
  p->topo = 1;
  p->N_shift_plaquette = 2;
  p->N_shift_topo = 10;
  p->N_steps_gf = 10;
  p->N_rk_steps = 40;
  strcpy(p->run_name, "c");
  strcpy(p->run_dir, "data");
  p->save_each_shifts = 2;
  return QCB_OK;
}

int qcb_ecmc_run_params_load(const char* path, qcb_ecmc_run_params* p) {
  if (!path || !p) return fail(QCB_ERR_INVALID, "null argument");
  std::string err;
  int r = ecmc_params_load(path, p, &err);
  if (r != QCB_OK) return fail(r, err);
  return QCB_OK;
}

}  // extern "C"
