// ecmc.h — launchers of the event-chain Monte Carlo kernels (k_ecmc.cu), library-internal.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/qcb.h"

namespace qcb {

// Size of the set of SU(3) elements near the identity (sample_persistant's set,
// src/ecmc/ecmc_mpi_cb.cpp:560): the identity and 5000 pairs (M, M^dagger).
constexpr int ECMC_SET_SIZE = 10001;

// One sample call of every chain.
struct EcmcLaunch {
  double2* links;        // FP64 array-of-structures copy: link (s, mu) = 9 double2 at (4 s + mu) * 9
  qcb_ecmc_chain* chains;
  uint32_t n_chains;
  int L[4];              // lattice extents
  int nb[4];             // blocks per direction (L[d] / l)
  int cum[4];            // cumulative shift of the field's frame, in [0, L[d])
  int l;                 // block edge (l_core)
  double beta, theta_sample, theta_refresh_site, theta_refresh_R;
  int poisson;
  uint32_t k0, k1;       // Philox key (seed)
  uint32_t call;         // sample calls made so far (keys the chains' sets)
  double epsilon_set;    // size of the near-identity set's rotations
  double2* sx;           // per chain: 9 double2 holding the set element of the current lift
  uint32_t* status;      // OR of the chains' status bits
};
// Launch shapes of the sample kernel: lanes per chain (1, 3 or 6, each lane computing an
// equal share of the six staples; lanes 0-2 of a group also share the lift's three products)
// and the register budget (C: capped for more resident chains).  All give the same results,
// bit for bit.
enum { ECMC_LAYOUT_1 = 1, ECMC_LAYOUT_3 = 3, ECMC_LAYOUT_3C = 4, ECMC_LAYOUT_6 = 6, ECMC_LAYOUT_6C = 7 };
// The layout for n_chains chains: `lanes` 1, 3 or 6 fixes the lanes per chain, 0 lets the
// number of chains choose them too; the register budget follows the waves of resident chains.
int ecmc_layout(uint32_t n_chains, int lanes);
cudaError_t launch_ecmc_sample(const EcmcLaunch& a, int layout, cudaStream_t s);
// out[0..2] += the chains' events, lifts, same-site lifts; zeroes them with reset.
cudaError_t launch_ecmc_counters(qcb_ecmc_chain* chains, uint32_t n, unsigned long long* out, int reset,
                                 cudaStream_t s);

}  // namespace qcb
