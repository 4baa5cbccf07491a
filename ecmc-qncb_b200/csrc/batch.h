// batch.h — device descriptors and launchers of the persistent multi-lattice kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace qcb {

// One lattice of a batched launch (device array).
struct BatchLat {
  Geom g;
  void* links;      // heatbath: the links; flow: buffer a of even steps
  void* work;       // flow: buffer b of even steps
  void* acc;        // flow: force accumulator
  double beta;      // heatbath coupling
  uint32_t k0, k1;  // Philox key (seed)
  uint32_t sweep0;  // sweep counter of the launch's first sweep
  uint32_t tile;    // sites per work item (any multiple of the block size)
  uint32_t ntiles;  // work items of this lattice per level (flow: flow_items_per_tile x site tiles)
  uint32_t nlev;    // levels this lattice takes part in (0 = all levels of the launch)
  int kind;         // BATCH_HB or BATCH_FLOW (mixed launches); BATCH_NONE: no work
  int n_hits;       // heatbath hits (0 = the launch's value)
  double eps;       // flow step (0 = the launch's value)
};

// One persistent launch: nlevels levels of per_level items each.
struct BatchRun {
  const BatchLat* lats;    // nlat descriptors
  const uint32_t* prefix;  // nlat+1 prefix sums of ntiles; prefix[nlat] = per_level
  int nlat;
  uint32_t nlevels;
  uint32_t per_level;
  uint32_t* done;    // nlat finished-tile counters, zero at launch
  uint32_t* status;  // [0] KP cap hits, [1] wait timeouts, [2] abort flag
  int n_hits;
  double eps;
};

enum : int { BATCH_NONE = -1, BATCH_HB = 0, BATCH_FLOW = 1, BATCH_MIXED = 2 };

// Work items of one flow level per tile of sites: FP32 lattices run one thread per site (both
// parities, 2 items), FP64 lattices one thread per link (4 directions x 2 parities, 8 items),
// as the single-lattice flow does, so that batched and single results stay bit-identical.
inline uint32_t flow_items_per_tile(int prec) { return prec == 1 ? 2u : 8u; }

// Cooperative persistent launch (kind BATCH_HB, BATCH_FLOW or BATCH_MIXED): the grid is the
// co-resident maximum (capped by max_blocks when > 0) for the given block size.
cudaError_t launch_batch(int kind, const BatchRun& run, int prec, int nr, int block, int max_blocks,
                         cudaStream_t s);

// Bounded-wait self-test: `blocks` co-resident blocks wait on flag[0] (never set); block 0
// gives up after limit_ns.  status[1] = timeouts, status[2] = abort flag, status[3] = waits
// that succeeded.
cudaError_t launch_wait_probe(const uint32_t* flag, uint32_t* status, uint64_t limit_ns, int blocks,
                              cudaStream_t s);

// Batched reductions: one item per (lattice, tile of RED sites), item r of lattice l in
// [rprefix[l], rprefix[l+1]).  out[l] = mean plaquette; out2[2l], out2[2l+1] = (Q, E).
// scratch holds 2 * rprefix[nlat] doubles.
int batch_red_sites();
cudaError_t launch_batch_plaquette(const BatchLat* lats, const uint32_t* rprefix, int nlat, uint32_t nitems,
                                   int prec, int nr, double* scratch, double* out, cudaStream_t s);
cudaError_t launch_batch_qe(const BatchLat* lats, const uint32_t* rprefix, int nlat, uint32_t nitems, int prec,
                            int nr, double* scratch, double* out2, cudaStream_t s);

}  // namespace qcb
