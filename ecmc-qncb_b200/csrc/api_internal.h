// api_internal.h — the C ABI's opaque objects and shared host helpers (library-internal).
#pragma once
#include <mutex>
#include <string>

#include "../../include/qcb.h"
#include "kernels.h"

struct qcb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int block = 0;
  uint32_t* d_status = nullptr;  // [0] KP cap hits
  uint32_t* h_status = nullptr;  // pinned mirror
  double* d_scratch = nullptr;   // reduction partials
  double* d_out = nullptr;       // small results
  double* h_out = nullptr;       // pinned mirror
  double* d_stage[2] = {nullptr, nullptr};
  size_t stage_bytes = 0;
  double* h_stage = nullptr;  // pinned, for file I/O
  uint64_t launches = 0;
  std::mutex mu;
  // Objects created on this context (lattices, batches, servers).  qcb_ctx_destroy with
  // live objects only marks the context; the last object's destroy frees it, so no child
  // ever uses a freed context.
  int refs = 0;
  bool doomed = false;
};

struct qcb_lattice {
  qcb_ctx* ctx = nullptr;
  qcb::LatDev dev;
  size_t bytes = 0;
  // Wilson-flow work space, allocated on first use: two link buffers + accumulator.
  void* fw[2] = {nullptr, nullptr};
  void* fz = nullptr;
  // Partial sums of the measuring heatbath passes, allocated on first use.
  double* meas = nullptr;
  size_t meas_n = 0;
  // Slab of a larger lattice (qcb_lattice_create_slab): global extents and the global time
  // of local time 1; slab_tl == 0 for a whole lattice.
  int gdims[4] = {0, 0, 0, 0};
  int slab_t0 = 0, slab_tl = 0;
};

namespace qcb {
// Reference counting of a context's child objects (see qcb_ctx::refs).
void ctx_ref(qcb_ctx* c);
void ctx_unref(qcb_ctx* c);
// Allocates a lattice's Wilson-flow work space (two link buffers + accumulator) once.
int ensure_flow_space(qcb_lattice* L);
// Reads and clears the context's device status words (after synchronising its stream).
int check_status(qcb_ctx* c);
}  // namespace qcb
