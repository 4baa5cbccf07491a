// api_batch.cu — C ABI of lattice batches (include/qcb.h, "batches of lattices"):
// persistent multi-lattice launches, batched observables, the graph-captured workload
// and the tile autotuner.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "api_internal.h"
#include "batch.h"

using namespace qcb;

namespace {

// Descriptor sets (n entries each) held on the device:
enum { SET_LINKS = 0,    // links = primary (heatbath, plaquette, in-place flow with work = fw0)
       SET_COPY_EVEN,    // links = fw0, work = fw1 (flow on a copy, even cumulative steps)
       SET_COPY_ODD,     // links = fw1, work = fw0 (odd cumulative steps)
       NSETS };

constexpr int DEFAULT_TILE = 256;

}  // namespace

struct qcb_batch {
  qcb_ctx* ctx = nullptr;
  int n = 0, prec = 0, nr = 0;
  std::vector<qcb_lattice*> lats;
  std::vector<uint32_t> hb_tile, flow_tile;
  BatchLat* d_desc = nullptr;  // NSETS * n
  BatchLat* h_desc = nullptr;  // pinned mirror
  uint32_t* d_prefix = nullptr;  // hb (n+1) | flow (n+1) | reduction (n+1)
  std::vector<uint32_t> h_prefix;
  uint32_t per_hb = 0, per_flow = 0, nred = 0;
  uint32_t* d_done = nullptr;
  uint32_t* d_status = nullptr;  // [0] KP cap hits, [1] wait timeouts, [2] abort
  uint32_t* h_status = nullptr;
  double* d_scratch = nullptr;  // 2 * nred
  double* d_out = nullptr;
  double* h_out = nullptr;
  size_t out_cap = 0;
  cudaGraphExec_t exec = nullptr;
  qcb_batch_plan plan{};
  bool have_plan = false;
  bool graph_ok = true;
};

namespace {

int bfail(int code, const std::string& msg) { return qcb::set_error(code, msg.c_str()); }
int bcuda(cudaError_t e, const char* what) {
  return qcb::set_error(QCB_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}
#define BCU(call, what)                                 \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return bcuda(e_, what);      \
  } while (0)
#define BTRY(x)                  \
  do {                           \
    int r_ = (x);                \
    if (r_ != QCB_OK) return r_; \
  } while (0)

uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// Rebuild descriptors and prefix sums from the lattices and tiles; upload them.
int upload_layout(qcb_batch* b) {
  const int n = b->n;
  b->h_prefix.assign(3 * (n + 1), 0);
  uint32_t* ph = &b->h_prefix[0];
  uint32_t* pf = &b->h_prefix[n + 1];
  uint32_t* pr = &b->h_prefix[2 * (n + 1)];
  for (int l = 0; l < n; ++l) {
    const qcb_lattice* L = b->lats[l];
    const uint32_t nth = ceil_div(L->dev.g.Vh, b->hb_tile[l]);
    const uint32_t ntf = flow_items_per_tile(L->dev.prec) * ceil_div(L->dev.g.Vh, b->flow_tile[l]);
    ph[l + 1] = ph[l] + nth;
    pf[l + 1] = pf[l] + ntf;
    pr[l + 1] = pr[l] + ceil_div(L->dev.g.V, (uint32_t)batch_red_sites());
    for (int s = 0; s < NSETS; ++s) {
      BatchLat& d = b->h_desc[s * n + l];
      memset(&d, 0, sizeof d);
      d.g = L->dev.g;
      d.acc = L->fz;
      d.tile = b->hb_tile[l];
      d.ntiles = nth;
      if (s == SET_LINKS) {
        d.links = L->dev.links;
        d.work = L->fw[0];
      } else if (s == SET_COPY_EVEN) {
        d.links = L->fw[0];
        d.work = L->fw[1];
      } else {
        d.links = L->fw[1];
        d.work = L->fw[0];
      }
    }
  }
  b->per_hb = ph[n];
  b->per_flow = pf[n];
  b->nred = pr[n];
  cudaFree(b->d_scratch);
  b->d_scratch = nullptr;
  BCU(cudaMalloc(&b->d_scratch, 2 * (size_t)b->nred * sizeof(double)), "batch scratch");
  BCU(cudaMemcpyAsync(b->d_prefix, b->h_prefix.data(), b->h_prefix.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                      b->ctx->stream),
      "prefix upload");
  BCU(cudaMemcpyAsync(b->d_desc, b->h_desc, (size_t)NSETS * n * sizeof(BatchLat), cudaMemcpyHostToDevice,
                      b->ctx->stream),
      "descriptor upload");
  BCU(cudaStreamSynchronize(b->ctx->stream), "sync");
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  b->have_plan = false;
  return QCB_OK;
}

// Heatbath parameters go into the SET_LINKS descriptors (host mirror + async upload).
int set_hb_params(qcb_batch* b, const double* betas, const uint64_t* seeds, const uint64_t* sweep_offsets) {
  for (int l = 0; l < b->n; ++l) {
    if (!(betas[l] > 0.0)) return bfail(QCB_ERR_INVALID, "beta must be positive");
    BatchLat& d = b->h_desc[SET_LINKS * b->n + l];
    d.beta = betas[l];
    d.k0 = (uint32_t)seeds[l];
    d.k1 = (uint32_t)(seeds[l] >> 32);
    d.sweep0 = (uint32_t)sweep_offsets[l];
  }
  BCU(cudaMemcpyAsync(b->d_desc, b->h_desc, (size_t)b->n * sizeof(BatchLat), cudaMemcpyHostToDevice, b->ctx->stream),
      "descriptor upload");
  return QCB_OK;
}

// Flow descriptors use the flow tile.
void flow_tiles_into(qcb_batch* b, int set, std::vector<BatchLat>& out) {
  out.assign(b->h_desc + set * b->n, b->h_desc + (set + 1) * b->n);
  for (int l = 0; l < b->n; ++l) {
    out[l].tile = b->flow_tile[l];
    out[l].ntiles = flow_items_per_tile(b->prec) * ceil_div(out[l].g.Vh, b->flow_tile[l]);
  }
}

BatchRun make_run(qcb_batch* b, int set, int kind, uint32_t nlevels, int n_hits, double eps) {
  BatchRun r;
  r.lats = b->d_desc + set * b->n;
  r.prefix = b->d_prefix + (kind == BATCH_HB ? 0 : (b->n + 1));
  r.nlat = b->n;
  r.nlevels = nlevels;
  r.per_level = (kind == BATCH_HB) ? b->per_hb : b->per_flow;
  r.done = b->d_done;
  r.status = b->d_status;
  r.n_hits = n_hits;
  r.eps = eps;
  return r;
}

// The flow descriptors (flow tile) live in a second device region after the NSETS sets.
BatchLat* flow_desc(qcb_batch* b, int set) { return b->d_desc + (NSETS + set) * b->n; }

int upload_flow_desc(qcb_batch* b) {
  for (int s = 0; s < NSETS; ++s) {
    std::vector<BatchLat> v;
    flow_tiles_into(b, s, v);
    BCU(cudaMemcpyAsync(flow_desc(b, s), v.data(), v.size() * sizeof(BatchLat), cudaMemcpyHostToDevice, b->ctx->stream),
        "flow descriptor upload");
    BCU(cudaStreamSynchronize(b->ctx->stream), "sync");
  }
  return QCB_OK;
}

int launch_hb(qcb_batch* b, int n_sweeps, int n_hits) {
  if (n_sweeps <= 0) return QCB_OK;
  BCU(cudaMemsetAsync(b->d_done, 0, b->n * sizeof(uint32_t), b->ctx->stream), "memset");
  BatchRun r = make_run(b, SET_LINKS, BATCH_HB, 8u * (uint32_t)n_sweeps, n_hits, 0.0);
  BCU(launch_batch(BATCH_HB, r, b->prec, b->nr, 128, 0, b->ctx->stream), "batched heatbath");
  b->ctx->launches++;
  return QCB_OK;
}

// n RK3 steps over descriptor set `set` (flow tiles).
int launch_flow(qcb_batch* b, int set, int n_steps, double eps) {
  if (n_steps <= 0) return QCB_OK;
  BCU(cudaMemsetAsync(b->d_done, 0, b->n * sizeof(uint32_t), b->ctx->stream), "memset");
  BatchRun r = make_run(b, set, BATCH_FLOW, 3u * (uint32_t)n_steps, 0, eps);
  r.lats = flow_desc(b, set);
  BCU(launch_batch(BATCH_FLOW, r, b->prec, b->nr, 128, 0, b->ctx->stream), "batched flow");
  b->ctx->launches++;
  return QCB_OK;
}

int launch_plaq(qcb_batch* b, int set, double* out) {
  BCU(launch_batch_plaquette(b->d_desc + set * b->n, b->d_prefix + 2 * (b->n + 1), b->n, b->nred, b->prec, b->nr,
                             b->d_scratch, out, b->ctx->stream),
      "batched plaquette");
  b->ctx->launches += 2;
  return QCB_OK;
}
int launch_qe(qcb_batch* b, int set, double* out2) {
  BCU(launch_batch_qe(b->d_desc + set * b->n, b->d_prefix + 2 * (b->n + 1), b->n, b->nred, b->prec, b->nr,
                      b->d_scratch, out2, b->ctx->stream),
      "batched clover Q/E");
  b->ctx->launches += 2;
  return QCB_OK;
}

int ensure_out(qcb_batch* b, size_t count) {
  if (b->out_cap >= count) return QCB_OK;
  cudaFree(b->d_out);
  cudaFreeHost(b->h_out);
  b->d_out = nullptr;
  b->h_out = nullptr;
  b->out_cap = 0;
  if (cudaMalloc(&b->d_out, count * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&b->h_out, count * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return bfail(QCB_ERR_NOMEM, "cannot allocate batch result buffers");
  }
  b->out_cap = count;
  return QCB_OK;
}

// Read back status words of the batch (KP cap hits, wait timeouts) after a sync.
int batch_status(qcb_batch* b) {
  BCU(cudaMemcpyAsync(b->h_status, b->d_status, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->ctx->stream),
      "status copy");
  BCU(cudaStreamSynchronize(b->ctx->stream), "sync");
  const uint32_t kp = b->h_status[0], to = b->h_status[1];
  if (kp || to || b->h_status[2]) {
    BCU(cudaMemsetAsync(b->d_status, 0, 4 * sizeof(uint32_t), b->ctx->stream), "status reset");
    BCU(cudaStreamSynchronize(b->ctx->stream), "sync");
    if (to || b->h_status[2])
      return bfail(QCB_ERR_STATE, "batched kernel: a dependency wait timed out (" + std::to_string(to) +
                                      "); the launch was abandoned");
    return bfail(QCB_ERR_KP_CAP, "Kennedy-Pendleton draw hit its attempt cap " + std::to_string(kp) + " time(s)");
  }
  return QCB_OK;
}

// The whole plan (heatbath, plaquette, flow on copies with records) as stream work.
int enqueue_plan(qcb_batch* b, const qcb_batch_plan& p) {
  const int n = b->n;
  const int per = 1 + 3 * (p.n_groups + 1);
  BTRY(launch_hb(b, p.n_sweeps, p.n_hits));
  // plaquette -> d_out[0 .. n)
  BTRY(launch_plaq(b, SET_LINKS, b->d_out));
  for (int l = 0; l < n; ++l) {
    qcb_lattice* L = b->lats[l];
    BCU(cudaMemcpyAsync(L->fw[0], L->dev.links, L->bytes, cudaMemcpyDeviceToDevice, b->ctx->stream), "copy");
  }
  // records: (Q, E) of group g -> d_out[n + 2 (g n + l)]
  int cum = 0;
  for (int g = 0; g <= p.n_groups; ++g) {
    BTRY(launch_qe(b, (cum & 1) ? SET_COPY_ODD : SET_COPY_EVEN, b->d_out + n + 2 * (size_t)g * n));
    if (g < p.n_groups) {
      BTRY(launch_flow(b, (cum & 1) ? SET_COPY_ODD : SET_COPY_EVEN, p.rk_per_group, p.eps));
      cum += p.rk_per_group;
    }
  }
  (void)per;
  BCU(cudaMemcpyAsync(b->h_out, b->d_out, (n + 2 * (size_t)(p.n_groups + 1) * n) * sizeof(double),
                      cudaMemcpyDeviceToHost, b->ctx->stream),
      "result copy");
  return QCB_OK;
}

void batch_free(qcb_batch* b);

bool same_plan(const qcb_batch_plan& a, const qcb_batch_plan& c) {
  return a.n_sweeps == c.n_sweeps && a.n_hits == c.n_hits && a.eps == c.eps && a.n_groups == c.n_groups &&
         a.rk_per_group == c.rk_per_group;
}

}  // namespace

extern "C" {

int qcb_batch_create(qcb_ctx* ctx, int n, qcb_lattice* const* lats, qcb_batch** out) {
  if (!ctx || !lats || !out || n <= 0) return bfail(QCB_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  for (int l = 0; l < n; ++l) {
    if (!lats[l]) return bfail(QCB_ERR_INVALID, "null lattice in batch");
    if (lats[l]->slab_tl) return bfail(QCB_ERR_INVALID, "a slab cannot join a batch (it needs halo exchanges)");
    if (lats[l]->ctx != ctx) return bfail(QCB_ERR_INVALID, "batch lattices must share the context");
    if (lats[l]->dev.prec != lats[0]->dev.prec || lats[l]->dev.nr != lats[0]->dev.nr)
      return bfail(QCB_ERR_INVALID, "batch lattices must share precision and storage");
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  BCU(cudaSetDevice(ctx->device), "cudaSetDevice");
  qcb_batch* b = new (std::nothrow) qcb_batch();
  if (!b) return bfail(QCB_ERR_NOMEM, "host allocation failed");
  b->ctx = ctx;
  b->n = n;
  b->prec = lats[0]->dev.prec;
  b->nr = lats[0]->dev.nr;
  b->lats.assign(lats, lats + n);
  b->hb_tile.assign(n, DEFAULT_TILE);
  b->flow_tile.assign(n, DEFAULT_TILE);
  auto fail_all = [&](int code) {
    b->ctx = nullptr;  // not counted yet
    batch_free(b);
    return code;
  };
  for (int l = 0; l < n; ++l) {
    int r = ensure_flow_space(b->lats[l]);
    if (r != QCB_OK) return fail_all(r);
  }
  if (cudaMalloc(&b->d_desc, 2 * (size_t)NSETS * n * sizeof(BatchLat)) != cudaSuccess ||
      cudaMallocHost(&b->h_desc, (size_t)NSETS * n * sizeof(BatchLat)) != cudaSuccess ||
      cudaMalloc(&b->d_prefix, 3 * (size_t)(n + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_done, (size_t)n * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_status, 4 * sizeof(uint32_t)) != cudaSuccess ||
      cudaMallocHost(&b->h_status, 4 * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    bfail(QCB_ERR_NOMEM, "cannot allocate batch descriptors");
    return fail_all(QCB_ERR_NOMEM);
  }
  if (cudaMemset(b->d_status, 0, 4 * sizeof(uint32_t)) != cudaSuccess) return fail_all(QCB_ERR_CUDA);
  int r = upload_layout(b);
  if (r == QCB_OK) r = upload_flow_desc(b);
  if (r != QCB_OK) return fail_all(r);
  ctx->refs++;  // under the context lock
  *out = b;
  return QCB_OK;
}

int qcb_batch_destroy(qcb_batch* b) {
  if (!b) return QCB_OK;
  qcb_ctx* c = b->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  batch_free(b);
  ctx_unref(c);
  return QCB_OK;
}

}  // extern "C"

namespace {
void batch_free(qcb_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  cudaFree(b->d_desc);
  cudaFreeHost(b->h_desc);
  cudaFree(b->d_prefix);
  cudaFree(b->d_done);
  cudaFree(b->d_status);
  cudaFreeHost(b->h_status);
  cudaFree(b->d_scratch);
  cudaFree(b->d_out);
  cudaFreeHost(b->h_out);
  cudaGetLastError();
  delete b;
}
}  // namespace

extern "C" {

int qcb_batch_set_tiles(qcb_batch* b, const int* hb_tile, const int* flow_tile) {
  if (!b) return bfail(QCB_ERR_INVALID, "null batch");
  for (int l = 0; l < b->n; ++l) {
    for (const int* t : {hb_tile, flow_tile})
      if (t && (t[l] < 32 || t[l] > 65536 || (t[l] & 31)))
        return bfail(QCB_ERR_INVALID, "tiles must be multiples of 32 in [32, 65536]");
  }
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  for (int l = 0; l < b->n; ++l) {
    if (hb_tile) b->hb_tile[l] = (uint32_t)hb_tile[l];
    if (flow_tile) b->flow_tile[l] = (uint32_t)flow_tile[l];
  }
  BTRY(upload_layout(b));
  return upload_flow_desc(b);
}

int qcb_batch_get_tiles(qcb_batch* b, int* hb_tile, int* flow_tile) {
  if (!b) return bfail(QCB_ERR_INVALID, "null batch");
  for (int l = 0; l < b->n; ++l) {
    if (hb_tile) hb_tile[l] = (int)b->hb_tile[l];
    if (flow_tile) flow_tile[l] = (int)b->flow_tile[l];
  }
  return QCB_OK;
}

int qcb_batch_heatbath(qcb_batch* b, const double* betas, int n_sweeps, int n_hits, const uint64_t* seeds,
                       const uint64_t* sweep_offsets) {
  if (!b || !betas || !seeds || !sweep_offsets) return bfail(QCB_ERR_INVALID, "null argument");
  if (n_sweeps < 0 || n_hits < 0 || n_hits > (1 << 20)) return bfail(QCB_ERR_INVALID, "bad sweep or hit count");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  BTRY(set_hb_params(b, betas, seeds, sweep_offsets));
  return launch_hb(b, n_sweeps, n_hits);
}

int qcb_batch_flow_steps(qcb_batch* b, double eps, int n_steps) {
  if (!b) return bfail(QCB_ERR_INVALID, "null batch");
  if (n_steps < 0) return bfail(QCB_ERR_INVALID, "negative step count");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  BTRY(launch_flow(b, SET_LINKS, n_steps, eps));
  if (n_steps & 1)  // the result is in fw0
    for (int l = 0; l < b->n; ++l) {
      qcb_lattice* L = b->lats[l];
      BCU(cudaMemcpyAsync(L->dev.links, L->fw[0], L->bytes, cudaMemcpyDeviceToDevice, b->ctx->stream), "copy back");
    }
  return QCB_OK;
}

int qcb_batch_plaquette(qcb_batch* b, double* out) {
  if (!b || !out) return bfail(QCB_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  BTRY(ensure_out(b, (size_t)b->n * 2));
  BTRY(launch_plaq(b, SET_LINKS, b->d_out));
  BCU(cudaMemcpyAsync(b->h_out, b->d_out, b->n * sizeof(double), cudaMemcpyDeviceToHost, b->ctx->stream), "D2H");
  BTRY(batch_status(b));
  memcpy(out, b->h_out, b->n * sizeof(double));
  return QCB_OK;
}

int qcb_batch_topo_qe(qcb_batch* b, double* q, double* e) {
  if (!b || !q || !e) return bfail(QCB_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  BTRY(ensure_out(b, (size_t)b->n * 2));
  BTRY(launch_qe(b, SET_LINKS, b->d_out));
  BCU(cudaMemcpyAsync(b->h_out, b->d_out, 2 * b->n * sizeof(double), cudaMemcpyDeviceToHost, b->ctx->stream), "D2H");
  BTRY(batch_status(b));
  for (int l = 0; l < b->n; ++l) {
    q[l] = b->h_out[2 * l];
    e[l] = b->h_out[2 * l + 1];
  }
  return QCB_OK;
}

int qcb_batch_run(qcb_batch* b, const qcb_batch_plan* plan, const double* betas, const uint64_t* seeds,
                  const uint64_t* sweep_offsets, double* results, int* used_graph) {
  if (!b || !plan || !betas || !seeds || !sweep_offsets || !results) return bfail(QCB_ERR_INVALID, "null argument");
  const qcb_batch_plan& p = *plan;
  if (p.n_sweeps < 0 || p.n_hits < 0 || p.n_groups < 0 || p.rk_per_group < 0 || p.n_hits > (1 << 20))
    return bfail(QCB_ERR_INVALID, "bad plan");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  const int n = b->n;
  BTRY(ensure_out(b, (size_t)n + 2 * (size_t)(p.n_groups + 1) * n));
  BTRY(set_hb_params(b, betas, seeds, sweep_offsets));
  bool graph = false;
  if (b->graph_ok) {
    if (!b->have_plan || !same_plan(b->plan, p) || !b->exec) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
      }
      // Capture the plan; on any capture failure fall back to direct launches.
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(b->ctx->stream, cudaStreamCaptureModeThreadLocal);
      int r = QCB_OK;
      if (e == cudaSuccess) {
        r = enqueue_plan(b, p);
        e = cudaStreamEndCapture(b->ctx->stream, &g);
      }
      if (e == cudaSuccess && r == QCB_OK && g) e = cudaGraphInstantiate(&b->exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess || r != QCB_OK || !b->exec) {
        cudaGetLastError();
        b->exec = nullptr;
        b->graph_ok = false;
      } else {
        b->plan = p;
        b->have_plan = true;
      }
    }
    if (b->exec) {
      BCU(cudaGraphLaunch(b->exec, b->ctx->stream), "graph launch");
      graph = true;
    }
  }
  if (!graph) BTRY(enqueue_plan(b, p));
  BTRY(batch_status(b));
  const int per = 1 + 3 * (p.n_groups + 1);
  for (int l = 0; l < n; ++l) {
    results[(size_t)l * per] = b->h_out[l];
    for (int g = 0; g <= p.n_groups; ++g) {
      double* rec = results + (size_t)l * per + 1 + 3 * g;
      rec[0] = (double)g * (double)p.rk_per_group * p.eps;
      rec[1] = b->h_out[n + 2 * ((size_t)g * n + l)];
      rec[2] = b->h_out[n + 2 * ((size_t)g * n + l) + 1];
    }
  }
  if (used_graph) *used_graph = graph ? 1 : 0;
  return QCB_OK;
}

int qcb_wait_selftest(qcb_ctx* ctx, double limit_s, uint32_t* timeouts, uint32_t* aborted) {
  if (!ctx || !timeouts || !aborted) return bfail(QCB_ERR_INVALID, "null argument");
  if (!(limit_s > 0.0 && limit_s <= 5.0)) return bfail(QCB_ERR_INVALID, "limit_s must be in (0, 5]");
  std::lock_guard<std::mutex> lk(ctx->mu);
  BCU(cudaSetDevice(ctx->device), "cudaSetDevice");
  uint32_t* d = nullptr;  // [0] the flag nothing sets, [1..4] status words
  BCU(cudaMalloc(&d, 8 * sizeof(uint32_t)), "self-test buffer");
  uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaError_t e = cudaMemsetAsync(d, 0, 8 * sizeof(uint32_t), ctx->stream);
  if (e == cudaSuccess) e = launch_wait_probe(d, d + 1, (uint64_t)(limit_s * 1e9), 4, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return bcuda(e, "wait self-test");
  ctx->launches++;
  *timeouts = h[2];
  *aborted = h[3];
  if (h[4] != 0) return bfail(QCB_ERR_STATE, "a wait on a flag that nothing sets succeeded");
  return QCB_OK;
}

}  // extern "C"

// ---- autotuner --------------------------------------------------------------------------
namespace {

std::map<std::string, int> read_cache(const char* path) {
  std::map<std::string, int> m;
  if (!path) return m;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    // lines of the form   "key": value,
    size_t a = line.find('"'), b2 = (a == std::string::npos) ? a : line.find('"', a + 1);
    if (a == std::string::npos || b2 == std::string::npos) continue;
    size_t c = line.find(':', b2);
    if (c == std::string::npos) continue;
    m[line.substr(a + 1, b2 - a - 1)] = atoi(line.c_str() + c + 1);
  }
  return m;
}

void write_cache(const char* path, const std::map<std::string, int>& m) {
  if (!path) return;
  std::ofstream f(path);
  f << "{\n";
  size_t k = 0;
  for (auto& kv : m) f << "  \"" << kv.first << "\": " << kv.second << (++k < m.size() ? ",\n" : "\n");
  f << "}\n";
}

}  // namespace

extern "C" int qcb_batch_autotune(qcb_batch* b, const char* cache_path) {
  if (!b) return bfail(QCB_ERR_INVALID, "null batch");
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  BCU(cudaSetDevice(b->ctx->device), "cudaSetDevice");
  cudaDeviceProp prop;
  BCU(cudaGetDeviceProperties(&prop, b->ctx->device), "device properties");
  const std::string pfx = std::string(prop.name) + "|" + (b->prec == QCB_FP64 ? "fp64" : "fp32") + "-" +
                          std::to_string(b->nr) + "|";
  auto cache = read_cache(cache_path);
  // distinct sizes
  std::map<std::string, std::vector<int>> by_size;
  for (int l = 0; l < b->n; ++l) {
    const Geom& g = b->lats[l]->dev.g;
    by_size[std::to_string(g.L[0]) + "x" + std::to_string(g.L[1]) + "x" + std::to_string(g.L[2]) + "x" +
            std::to_string(g.L[3])]
        .push_back(l);
  }
  const int cands[] = {128, 256, 512, 1024, 2048};
  std::vector<uint32_t> hb(b->hb_tile), fl(b->flow_tile);
  cudaEvent_t e0, e1;
  BCU(cudaEventCreate(&e0), "event");
  BCU(cudaEventCreate(&e1), "event");
  for (auto& kv : by_size) {
    const std::string khb = pfx + "hb|" + kv.first, kfl = pfx + "flow|" + kv.first;
    if (cache.count(khb) && cache.count(kfl)) {
      for (int l : kv.second) {
        hb[l] = (uint32_t)cache[khb];
        fl[l] = (uint32_t)cache[kfl];
      }
      continue;
    }
    // A sub-batch of this size's lattices, timed on scratch copies: the heatbath runs on
    // fw1 (copied from the links) and the flow on fw1/fw0, so the lattices are untouched.
    const int m = (int)kv.second.size();
    std::vector<BatchLat> dsc(m);
    std::vector<uint32_t> pre(m + 1, 0);
    for (int j = 0; j < m; ++j) {
      qcb_lattice* L = b->lats[kv.second[j]];
      BCU(cudaMemcpyAsync(L->fw[1], L->dev.links, L->bytes, cudaMemcpyDeviceToDevice, b->ctx->stream), "copy");
    }
    BatchLat* d_dsc = nullptr;
    uint32_t* d_pre = nullptr;
    BCU(cudaMalloc(&d_dsc, m * sizeof(BatchLat)), "tune alloc");
    BCU(cudaMalloc(&d_pre, (m + 1) * sizeof(uint32_t)), "tune alloc");
    float best_hb = 1e30f, best_fl = 1e30f;
    int arg_hb = DEFAULT_TILE, arg_fl = DEFAULT_TILE;
    for (int kind = 0; kind < 2; ++kind)
      for (int cand : cands) {
        for (int j = 0; j < m; ++j) {
          qcb_lattice* L = b->lats[kv.second[j]];
          BatchLat& d = dsc[j];
          memset(&d, 0, sizeof d);
          d.g = L->dev.g;
          d.links = L->fw[1];
          d.work = L->fw[0];
          d.acc = L->fz;
          d.beta = 6.0;
          d.k0 = 12345u;
          d.tile = (uint32_t)cand;
          d.ntiles = (kind == 0 ? 1u : flow_items_per_tile(L->dev.prec)) * ceil_div(d.g.Vh, (uint32_t)cand);
          pre[j + 1] = pre[j] + d.ntiles;
        }
        if (cand > 2 * (int)dsc[0].g.Vh && cand != cands[0]) continue;  // larger than the lattice
        BCU(cudaMemcpyAsync(d_dsc, dsc.data(), m * sizeof(BatchLat), cudaMemcpyHostToDevice, b->ctx->stream), "H2D");
        BCU(cudaMemcpyAsync(d_pre, pre.data(), (m + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, b->ctx->stream),
            "H2D");
        BatchRun r;
        r.lats = d_dsc;
        r.prefix = d_pre;
        r.nlat = m;
        r.per_level = pre[m];
        r.done = b->d_done;
        r.status = b->d_status;
        r.n_hits = 1;
        r.eps = 0.02;
        r.nlevels = kind == 0 ? 16 : 6;  // 2 sweeps / 2 RK3 steps
        float best = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
          BCU(cudaMemsetAsync(b->d_done, 0, m * sizeof(uint32_t), b->ctx->stream), "memset");
          BCU(cudaEventRecord(e0, b->ctx->stream), "event");
          BCU(launch_batch(kind == 0 ? BATCH_HB : BATCH_FLOW, r, b->prec, b->nr, 128, 0, b->ctx->stream), "tune launch");
          BCU(cudaEventRecord(e1, b->ctx->stream), "event");
          BCU(cudaEventSynchronize(e1), "event sync");
          float ms = 0;
          BCU(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
          if (rep > 0) best = std::min(best, ms);
          b->ctx->launches++;
        }
        if (kind == 0 && best < best_hb) {
          best_hb = best;
          arg_hb = cand;
        }
        if (kind == 1 && best < best_fl) {
          best_fl = best;
          arg_fl = cand;
        }
      }
    cudaFree(d_dsc);
    cudaFree(d_pre);
    cache[khb] = arg_hb;
    cache[kfl] = arg_fl;
    for (int l : kv.second) {
      hb[l] = (uint32_t)arg_hb;
      fl[l] = (uint32_t)arg_fl;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BTRY(batch_status(b));
  write_cache(cache_path, cache);
  b->hb_tile = hb;
  b->flow_tile = fl;
  BTRY(upload_layout(b));
  return upload_flow_desc(b);
}
