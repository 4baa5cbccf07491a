// kernels.h — host-side launchers of the sm_100a kernels (one .cu file per family).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.cuh"

namespace qcb {

// Device description of one lattice's link storage.
struct LatDev {
  Geom g;
  int prec;   // QCB_FP64 / QCB_FP32
  int nr;     // 18 / 12
  void* links;
};

// Device description of one su(3) algebra field (flow accumulator), same precision.
struct AlgDev {
  void* p;
};

size_t link_bytes(const Geom& g, int prec, int nr);
size_t alg_bytes(const Geom& g, int prec);
Geom make_geom(const int dims[4]);
// Slab of global lattice global_dims: global times t0 .. t0 + tl - 1 as local times 1 .. tl,
// plus one halo time slice on each side (local extents Lx, Ly, Lz, tl + 2).
Geom make_slab_geom(const int global_dims[4], int t0, int tl);

// ---- util (k_util.cu) --------------------------------------------------------------
cudaError_t launch_cold(const LatDev& L, cudaStream_t s, int block);
cudaError_t launch_hot(const LatDev& L, uint64_t seed, cudaStream_t s, int block);
cudaError_t launch_gauge_transform(const LatDev& L, uint64_t seed, cudaStream_t s, int block);
cudaError_t launch_reunitarize(const LatDev& L, cudaStream_t s, int block);
// AoS FP64 (72 doubles per site, ILDG order) for the sites [site0, site0+nsites) <-> lattice.
cudaError_t launch_aos_to_soa(const LatDev& L, const double* aos, uint32_t site0, uint32_t nsites, int bswap,
                              cudaStream_t s, int block);
cudaError_t launch_soa_to_aos(const LatDev& L, double* aos, uint32_t site0, uint32_t nsites, int bswap,
                              cudaStream_t s, int block);
cudaError_t launch_convert(const LatDev& dst, const LatDev& src, cudaStream_t s, int block);
// dst(x) = src(x - shift), periodic (same geometry and storage; dst != src).
cudaError_t launch_translate(const LatDev& dst, const LatDev& src, const int shift[4], cudaStream_t s, int block);

// ---- heatbath (k_hb.cu) ------------------------------------------------------------
// One checkerboard pass: every link (mu, parity) gets n_hits Cabibbo-Marinari hits.
// status[0] counts KP draws that hit the attempt cap.  frozen (optional) = {lcore, s0, s1,
// s2, s3}: links with (x_d + s_d) % lcore == 0 for some d != mu are left unchanged.
cudaError_t launch_hb_pass(const LatDev& L, int mu, int parity, double beta, uint64_t seed, uint32_t sweep,
                           int n_hits, uint32_t* status, cudaStream_t s, int block, const int* frozen = nullptr);

// Pass (mu = 3, parity) of the last sweep of a measurement: the same updates as
// launch_hb_pass, and one FP64 partial per block of 128 threads written to parts[0 ..
// hb_meas_blocks(L)): the sum over the block's sites x of Re tr of the spatial plaquettes
// P_ij(x), i < j < 3, plus for parity 1 Re tr(U_3(x) A_3(x)) with the updated link.  After
// both parities, the partials of the two passes sum to the sum of Re tr P over all 6V
// plaquettes of the final links.
int hb_meas_blocks(const LatDev& L);
cudaError_t launch_hb_pass_meas(const LatDev& L, int parity, double beta, uint64_t seed, uint32_t sweep,
                                int n_hits, uint32_t* status, double* parts, cudaStream_t s);

// ---- observables (k_obs.cu) --------------------------------------------------------
// Reductions write per-block partial sums into scratch (nparts doubles per quantity,
// nparts = reduce_blocks()) and a final single-block kernel writes the FP64 total(s)
// into out (device).
int reduce_blocks();
cudaError_t launch_plaquette(const LatDev& L, double* scratch, double* out, cudaStream_t s, int block);
cudaError_t launch_clover_qe(const LatDev& L, double* scratch, double* out2, cudaStream_t s, int block);
// Plaquette sum with nblocks reduction blocks (scratch holds nblocks doubles); out[0] = sum.
cudaError_t launch_plaquette_partials(const LatDev& L, int nblocks, double* scratch, double* out, cudaStream_t s);
int reduce_threads();
// out[0] = sum of parts[0 .. n) in a fixed order (two launches); tmp holds 256 doubles.
cudaError_t launch_sum_parts(const double* parts, int n, double* tmp, double* out, cudaStream_t s);
// (Q, E) from per-block clover partials: parts[0 .. n) unscaled q sums, parts[n .. 2n) unscaled
// e sums; out2[0] = Q = sum q / (4 pi^2), out2[1] = E = sum e / 2 * inv_vol.  tmp holds 512
// doubles.
cudaError_t launch_qe_from_parts(const double* parts, int n, double* tmp, double* out2, double inv_vol,
                                 cudaStream_t s);

// ---- flow (k_flow.cu) --------------------------------------------------------------
// RK3 stage k (1, 2, 3) of Luescher's integrator: reads links from src, the force
// accumulator z, writes links to dst.
cudaError_t launch_flow_stage(int stage, const LatDev& src, const LatDev& dst, const AlgDev& z, double eps,
                              cudaStream_t s, int block);
// The same stage with one thread per site (k_flow_site.cu; FP32 storages).
cudaError_t launch_flow_site(int stage, const LatDev& src, const LatDev& dst, const AlgDev& z, double eps,
                             cudaStream_t s);
// Stage 1 with one thread per site that also sums the clover (q, e) of every site of src:
// parts[0 .. n) and parts[n .. 2n) receive the per-block unscaled sums, n = flow_site_blocks(src)
// (feed them to launch_qe_from_parts).  FP32 whole lattices; the links are those of
// launch_flow_site, bit for bit, and each site's (q, e) that of launch_clover_qe.
int flow_site_blocks(const LatDev& L);
cudaError_t launch_flow_site_qe(const LatDev& src, const LatDev& dst, const AlgDev& z, double eps, double* parts,
                                cudaStream_t s);

// Sets the calling thread's qcb_last_error() message; returns code.
int set_error(int code, const char* msg);

}  // namespace qcb
