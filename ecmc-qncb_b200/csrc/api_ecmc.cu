// api_ecmc.cu — C ABI of the event-chain Monte Carlo (include/qcb.h, "event-chain Monte
// Carlo"): chain records on the device, one launch per sample call of every chain.
#include <string.h>

#include <new>
#include <string>

#include "api_internal.h"
#include "ecmc.h"

using namespace qcb;

struct qcb_ecmc {
  qcb_ctx* ctx = nullptr;
  qcb_lattice* lat = nullptr;
  qcb_ecmc_params p{};
  uint64_t seed = 0;
  uint64_t calls = 0;  // sample calls made (keys the chains' sets in the next call)
  int nb[4] = {0, 0, 0, 0};
  uint32_t n_chains = 0;
  int lanes = 0;               // lanes per chain asked for (0: chosen by the library)
  double2* d_links = nullptr;  // FP64 array-of-structures copy of the lattice
  qcb_ecmc_chain* d_chains = nullptr;
  double2* d_sx = nullptr;     // per chain: the set element of the current lift (9 double2)
  uint32_t* d_status = nullptr;
  unsigned long long* d_count = nullptr;  // events, lifts, revs
  unsigned long long* h_count = nullptr;  // pinned: 3 counters + status word
};

namespace {

int efail(int code, const std::string& msg) { return qcb::set_error(code, msg.c_str()); }
int ecuda(cudaError_t e, const char* what) {
  return qcb::set_error(QCB_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}
#define ECU(call, what)                             \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return ecuda(e_, what);  \
  } while (0)

void ecmc_free(qcb_ecmc* e) {
  cudaFree(e->d_links);
  cudaFree(e->d_chains);
  cudaFree(e->d_sx);
  cudaFree(e->d_status);
  cudaFree(e->d_count);
  cudaFreeHost(e->h_count);
  cudaGetLastError();
  delete e;
}

size_t link_aos_bytes(const qcb_lattice* L) { return (size_t)L->dev.g.V * 72 * sizeof(double); }

}  // namespace

extern "C" {

int qcb_ecmc_create(qcb_lattice* L, const qcb_ecmc_params* p, uint64_t seed, qcb_ecmc** out) {
  if (!L || !p || !out) return efail(QCB_ERR_INVALID, "null argument");
  *out = nullptr;
  if (L->slab_tl) return efail(QCB_ERR_STATE, "not available on a slab");
  if (!(p->beta > 0.0)) return efail(QCB_ERR_INVALID, "beta must be positive");
  if (!(p->theta_sample > 0.0) || !(p->theta_refresh_site > 0.0) || !(p->theta_refresh_R > 0.0))
    return efail(QCB_ERR_INVALID, "the angle budgets must be positive");
  if (!(p->epsilon_set >= 0.0 && p->epsilon_set <= 1.0)) return efail(QCB_ERR_INVALID, "epsilon_set must lie in [0, 1]");
  if (p->l_core < 3) return efail(QCB_ERR_INVALID, "l_core must be at least 3 (random sites lie in 1 .. l_core-2)");
  qcb_ecmc* e = new (std::nothrow) qcb_ecmc();
  if (!e) return efail(QCB_ERR_NOMEM, "host allocation failed");
  e->lat = L;
  e->p = *p;
  e->seed = seed;
  uint64_t n = 1;
  for (int d = 0; d < 4; ++d) {
    if (L->dev.g.L[d] % p->l_core) {
      delete e;
      return efail(QCB_ERR_INVALID, "l_core must divide every extent");
    }
    e->nb[d] = L->dev.g.L[d] / p->l_core;
    n *= (uint64_t)e->nb[d];
  }
  e->n_chains = (uint32_t)n;
  qcb_ctx* c = L->ctx;
  std::lock_guard<std::mutex> lk(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) {
    delete e;
    return efail(QCB_ERR_CUDA, "cudaSetDevice failed");
  }
  if (cudaMalloc(&e->d_links, link_aos_bytes(L)) != cudaSuccess ||
      cudaMalloc(&e->d_chains, (size_t)e->n_chains * sizeof(qcb_ecmc_chain)) != cudaSuccess ||
      cudaMalloc(&e->d_sx, (size_t)e->n_chains * 9 * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&e->d_status, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&e->d_count, 3 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&e->h_count, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    ecmc_free(e);
    return efail(QCB_ERR_NOMEM, "cannot allocate the chain work space");
  }
  if (cudaMemsetAsync(e->d_chains, 0, (size_t)e->n_chains * sizeof(qcb_ecmc_chain), c->stream) != cudaSuccess ||
      cudaMemsetAsync(e->d_status, 0, sizeof(uint32_t), c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    cudaGetLastError();
    ecmc_free(e);
    return efail(QCB_ERR_CUDA, "cannot initialise the chain records");
  }
  e->ctx = c;
  c->refs++;  // under the context lock
  *out = e;
  return QCB_OK;
}

int qcb_ecmc_destroy(qcb_ecmc* e) {
  if (!e) return QCB_OK;
  qcb_ctx* c = e->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  ecmc_free(e);
  ctx_unref(c);
  return QCB_OK;
}

int qcb_ecmc_num_chains(const qcb_ecmc* e, int* n) {
  if (!e || !n) return efail(QCB_ERR_INVALID, "null argument");
  *n = (int)e->n_chains;
  return QCB_OK;
}

int qcb_ecmc_set_lanes(qcb_ecmc* e, int lanes) {
  if (!e) return efail(QCB_ERR_INVALID, "null argument");
  if (lanes != 0 && lanes != 1 && lanes != 3 && lanes != 6)
    return efail(QCB_ERR_INVALID, "lanes per chain must be 0 (automatic), 1, 3 or 6");
  e->lanes = lanes;
  return QCB_OK;
}

int qcb_ecmc_lanes(const qcb_ecmc* e, int* lanes) {
  if (!e || !lanes) return efail(QCB_ERR_INVALID, "null argument");
  qcb_ctx* c = e->ctx;
  std::lock_guard<std::mutex> lk(c->mu);
  ECU(cudaSetDevice(c->device), "cudaSetDevice");
  const int layout = ecmc_layout(e->n_chains, e->lanes);
  *lanes = layout == ECMC_LAYOUT_1 ? 1 : (layout == ECMC_LAYOUT_6 || layout == ECMC_LAYOUT_6C ? 6 : 3);
  return QCB_OK;
}

int qcb_ecmc_sample_n(qcb_ecmc* e, const int* shifts, int n) {
  if (!e || (!shifts && n > 0)) return efail(QCB_ERR_INVALID, "null argument");
  if (n < 0) return efail(QCB_ERR_INVALID, "negative call count");
  if (n == 0) return QCB_OK;
  qcb_lattice* L = e->lat;
  qcb_ctx* c = e->ctx;
  EcmcLaunch a;
  a.links = e->d_links;
  a.epsilon_set = e->p.epsilon_set;
  a.sx = e->d_sx;
  a.chains = e->d_chains;
  a.n_chains = e->n_chains;
  for (int d = 0; d < 4; ++d) {
    a.L[d] = L->dev.g.L[d];
    a.nb[d] = e->nb[d];
  }
  a.l = e->p.l_core;
  a.beta = e->p.beta;
  a.theta_sample = e->p.theta_sample;
  a.theta_refresh_site = e->p.theta_refresh_site;
  a.theta_refresh_R = e->p.theta_refresh_R;
  a.poisson = e->p.poisson ? 1 : 0;
  a.k0 = (uint32_t)e->seed;
  a.k1 = (uint32_t)(e->seed >> 32);
  a.status = e->d_status;
  std::lock_guard<std::mutex> lk(c->mu);
  ECU(cudaSetDevice(c->device), "cudaSetDevice");
  ECU(launch_soa_to_aos(L->dev, reinterpret_cast<double*>(e->d_links), 0, L->dev.g.V, 0, c->stream, 0),
      "links to FP64 array-of-structures");
  c->launches++;
  // A launch that fails part-way leaves the calls before it complete: their link updates are
  // still unpacked into the lattice below, so the lattice and the chain records (and the call
  // count) stay consistent, and the failure is returned after the unpack.
  cudaError_t err = cudaSuccess;
  const char* what = nullptr;
  const int layout = ecmc_layout(e->n_chains, e->lanes);
  for (int k = 0; k < n && err == cudaSuccess; ++k) {
    for (int d = 0; d < 4; ++d) a.cum[d] = ((shifts[4 * k + d] % a.L[d]) + a.L[d]) % a.L[d];
    a.call = (uint32_t)e->calls;
    err = launch_ecmc_sample(a, layout, c->stream);
    if (err != cudaSuccess) {
      what = "ECMC sample";
      break;
    }
    c->launches++;
    e->calls++;
  }
  ECU(launch_aos_to_soa(L->dev, reinterpret_cast<const double*>(e->d_links), 0, L->dev.g.V, 0, c->stream, 0),
      "links from FP64 array-of-structures");
  c->launches++;
  if (err != cudaSuccess) return efail(QCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
  return QCB_OK;
}

int qcb_ecmc_sample(qcb_ecmc* e, const int shift[4]) {
  if (!e || !shift) return efail(QCB_ERR_INVALID, "null argument");
  return qcb_ecmc_sample_n(e, shift, 1);
}

int qcb_ecmc_counters(qcb_ecmc* e, uint64_t out[3], int reset) {
  if (!e || !out) return efail(QCB_ERR_INVALID, "null argument");
  qcb_ctx* c = e->ctx;
  std::lock_guard<std::mutex> lk(c->mu);
  ECU(cudaSetDevice(c->device), "cudaSetDevice");
  ECU(cudaMemsetAsync(e->d_count, 0, 3 * sizeof(unsigned long long), c->stream), "counter reset");
  ECU(launch_ecmc_counters(e->d_chains, e->n_chains, e->d_count, reset, c->stream), "ECMC counters");
  c->launches++;
  ECU(cudaMemcpyAsync(e->h_count, e->d_count, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
      "counter copy");
  uint32_t* st = reinterpret_cast<uint32_t*>(&e->h_count[3]);
  ECU(cudaMemcpyAsync(st, e->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream), "status copy");
  ECU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  for (int k = 0; k < 3; ++k) out[k] = (uint64_t)e->h_count[k];
  if (*st) {
    const uint32_t bits = *st;
    ECU(cudaMemsetAsync(e->d_status, 0, sizeof(uint32_t), c->stream), "status reset");
    ECU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return efail(QCB_ERR_STATE, std::string("a chain stopped early:") + ((bits & 1) ? " non-finite event angle" : "") +
                                    ((bits & 2) ? " 2^26 events in one sample call" : ""));
  }
  return QCB_OK;
}

int qcb_ecmc_get_chains(qcb_ecmc* e, qcb_ecmc_chain* chains, uint64_t* calls) {
  if (!e || !chains) return efail(QCB_ERR_INVALID, "null argument");
  qcb_ctx* c = e->ctx;
  std::lock_guard<std::mutex> lk(c->mu);
  ECU(cudaSetDevice(c->device), "cudaSetDevice");
  ECU(cudaMemcpyAsync(chains, e->d_chains, (size_t)e->n_chains * sizeof(qcb_ecmc_chain), cudaMemcpyDeviceToHost,
                      c->stream),
      "chain copy");
  ECU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  if (calls) *calls = e->calls;
  return QCB_OK;
}

int qcb_ecmc_set_chains(qcb_ecmc* e, const qcb_ecmc_chain* chains, uint64_t calls) {
  if (!e || !chains) return efail(QCB_ERR_INVALID, "null argument");
  for (uint32_t i = 0; i < e->n_chains; ++i) {
    const qcb_ecmc_chain& r = chains[i];
    if (!r.initialized) continue;
    bool ok = r.mu >= 0 && r.mu < 4 && (r.epsilon == -1 || r.epsilon == 1) && r.set_counter >= 0 &&
              r.set_counter <= 10000;
    for (int d = 0; d < 4; ++d) ok = ok && r.site[d] >= -(1 << 20) && r.site[d] <= (1 << 20);
    if (!ok) return efail(QCB_ERR_INVALID, "chain " + std::to_string(i) + " has a direction, sense, site or set counter out of range");
  }
  qcb_ctx* c = e->ctx;
  std::lock_guard<std::mutex> lk(c->mu);
  ECU(cudaSetDevice(c->device), "cudaSetDevice");
  ECU(cudaMemcpyAsync(e->d_chains, chains, (size_t)e->n_chains * sizeof(qcb_ecmc_chain), cudaMemcpyHostToDevice,
                      c->stream),
      "chain copy");
  ECU(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
  e->calls = calls;
  return QCB_OK;
}

}  // extern "C"
