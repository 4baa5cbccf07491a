/*
 * qcb.h — C ABI of the B200 (sm_100a) implementation of the ECMC-QNCB heatbath /
 * plaquette / Wilson-flow hot path.
 *
 * Conventions
 *   - Every function returns int: QCB_OK (0) or an error code; qcb_last_error()
 *     returns the message of the last failure on the calling thread.
 *   - No C++ exception crosses this boundary.
 *   - An opaque qcb_ctx binds one CUDA device and one stream; a qcb_lattice owns its
 *     device memory.  Calls on one context are serialised in stream order; different
 *     contexts may be driven from different threads.
 *   - Host buffers are owned by the caller and only borrowed for the duration of a call.
 *   - Host link buffers ("AoS") use the ILDG site order of the reference
 *     (src/io/ildg.cpp:87-106): t slowest, then z, y, x; per site mu = 0..3; per link a
 *     row-major 3x3 of (re, im) doubles, i.e. 72 doubles per site, native endian.
 *
 * The reference exposes no FFI; each entry point names the reference function whose
 * role it takes over (file:line within the reference project).
 */
#ifndef QCB_H
#define QCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QCB_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------- */
enum {
  QCB_OK = 0,
  QCB_ERR_INVALID = 1,   /* bad argument (null pointer, odd extent, bad enum, ...)      */
  QCB_ERR_CUDA = 2,      /* a CUDA runtime call failed (no device, launch error, ...)   */
  QCB_ERR_IO = 3,        /* file could not be opened / read / written                   */
  QCB_ERR_FORMAT = 4,    /* malformed LIME/ILDG file or input file value                */
  QCB_ERR_NOMEM = 5,     /* device or host allocation failed / admission refused        */
  QCB_ERR_KP_CAP = 6,    /* Kennedy-Pendleton rejection loop hit its attempt cap        */
  QCB_ERR_STATE = 7,     /* call not valid in the current object state                  */
  QCB_ERR_CANCELLED = 8  /* serving job cancelled before completion                     */
};

/* ---- enums ------------------------------------------------------------------------ */
enum { QCB_FP64 = 0, QCB_FP32 = 1 };           /* arithmetic / storage precision        */
enum { QCB_R18 = 18, QCB_R12 = 12 };           /* reals stored per link                 */

typedef struct qcb_ctx qcb_ctx;
typedef struct qcb_lattice qcb_lattice;

/* ---- library ---------------------------------------------------------------------- */
int qcb_abi_version(void);
const char* qcb_last_error(void);
/* Number of CUDA devices visible (0 on a host without GPU; never fails). */
int qcb_device_count(int* count);

/* ---- context ------------------------------------------------------------------------
 * Replaces the per-rank process state of the reference driver
 * (src/bin/gauge_hb_ncb.cpp:18-28: MpiTopology + GeometryCB + RNG). */
int qcb_ctx_create(int device, unsigned flags, qcb_ctx** out);
int qcb_ctx_destroy(qcb_ctx* ctx);
/* Waits for all work queued on the context's stream, then reports device-side
 * status words (KP cap hits) accumulated since the last call. */
int qcb_ctx_sync(qcb_ctx* ctx);
/* Number of kernels this context launched so far (all kinds). */
int qcb_ctx_launch_count(qcb_ctx* ctx, uint64_t* count);
/* Thread-block size used by subsequent launches of the per-link/per-site kernels
 * (0 = built-in default).  Results do not depend on it. */
int qcb_ctx_set_block(qcb_ctx* ctx, int threads);
/* The cudaStream_t the context launches on (as void*). */
int qcb_ctx_stream(qcb_ctx* ctx, void** stream);

/* ---- lattice ------------------------------------------------------------------------
 * Replaces GaugeField + GeometryCB (src/gauge/GaugeField.h:18-62,
 * src/geometry/GeometryCB.h:8-58): periodic lattice of extents dims = {Lx,Ly,Lz,Lt}
 * (all even, >= 2), stored on the device in a parity-split structure-of-arrays layout.
 * A new lattice is cold (every link the identity, GaugeField.h:37-42). */
int qcb_lattice_create(qcb_ctx* ctx, const int dims[4], int precision, int storage,
                       qcb_lattice** out);
int qcb_lattice_destroy(qcb_lattice* lat);
int qcb_lattice_info(const qcb_lattice* lat, int dims[4], int* precision, int* storage,
                     size_t* device_bytes);
/* Device address of the link storage and its layout parameters (for zero-copy users):
 * chunk c of link (mu, parity, i) sits at element ((mu*2+parity)*nchunk + c)*stride + i
 * of an array of chunk-sized vectors (double2, float4 or float2). */
int qcb_lattice_device_links(const qcb_lattice* lat, void** dev_ptr, size_t* stride,
                             int* nchunk, int* chunk_bytes);

/* GaugeField::cold_start (src/gauge/GaugeField.cpp:23-34). */
int qcb_cold_start(qcb_lattice* lat);
/* GaugeField::hot_start (src/gauge/GaugeField.cpp:10-20), redesigned: every link drawn
 * Haar-uniformly in SU(3) from a Philox4x32-10 stream keyed by seed. */
int qcb_hot_start(qcb_lattice* lat, uint64_t seed);
/* Copy links from / to a host AoS FP64 buffer (72*V doubles, ILDG order, native endian);
 * replaces the pack/unpack loops of src/io/ildg.cpp:87-106,212-232. */
int qcb_set_links(qcb_lattice* lat, const double* aos);
int qcb_get_links(qcb_lattice* lat, double* aos);
/* Copy src into dst (same dims; precision/storage may differ: converts on the device). */
int qcb_copy_links(qcb_lattice* dst, const qcb_lattice* src);
/* Reunitarise every link (Gram-Schmidt on rows 0,1; row 2 = conj(row0 x row1)).
 * Reference counterpart: GaugeField::project_field_su3 (GaugeField.cpp:36-58), which uses
 * columns; both map a near-SU(3) matrix to SU(3). */
int qcb_reunitarize(qcb_lattice* lat);
/* Random gauge transformation U_mu(x) -> G(x) U_mu(x) G(x+mu)^dagger with Haar G from
 * seed (GaugeField::gauge_transform, GaugeField.cpp:100-114). */
int qcb_gauge_transform(qcb_lattice* lat, uint64_t seed);

/* ---- ILDG / LIME -------------------------------------------------------------------
 * save_ildg_clime / read_ildg_clime (src/io/ildg.cpp:34-136, 138-237): a LIME file with an
 * "ildg-format" XML record and an "ildg-binary-data" record of big-endian FP64 links.
 * The lattice must be hypercubic (the reference's XML carries one extent). */
int qcb_save_ildg(qcb_lattice* lat, const char* path);
int qcb_load_ildg(qcb_lattice* lat, const char* path);
/* Host-only: locate the binary record; returns its byte offset and length. */
int qcb_ildg_probe(const char* path, uint64_t* data_offset, uint64_t* data_bytes);

/* ---- heatbath ----------------------------------------------------------------------
 * mpi::heatbathcb::samples / sweep / hit (src/heatbath/heatbath_mpi.cpp:11-69) with
 * heatbath::su2_step / generate_su2_kp (src/heatbath/heatbath.cpp:8-44): n_sweeps sweeps of
 * Cabibbo-Marinari updates over subgroups (0,1),(1,2),(0,2), n_hits hits per link, each
 * sweep = 8 checkerboard passes (mu = 0..3, parity 0 then 1).  Random numbers come from
 * Philox4x32-10 keyed by seed with counters (link, sweep_offset + s, hit/subgroup, draw),
 * so the result does not depend on the launch shape.  Asynchronous: the KP status is
 * reported by the next qcb_ctx_sync / result-returning call. */
int qcb_heatbath(qcb_lattice* lat, double beta, int n_sweeps, int n_hits, uint64_t seed,
                 uint64_t sweep_offset);
/* mpi::heatbathcb::samples followed by mean_plaquette_global (heatbath_mpi.cpp:37-69,
 * observables_mpi.cpp:8-43), as the driver runs them when N_shift_plaquette = 1
 * (src/bin/gauge_hb_ncb.cpp:122-143): n_sweeps sweeps exactly as qcb_heatbath (the same
 * links, bit for bit), then *plaq = the mean plaquette of the final links.  The plaquette is
 * summed inside the last sweep's two mu = 3 passes, with no separate plaquette launch; it
 * agrees with qcb_plaquette to rounding.  n_sweeps = 0 only measures.  Whole lattices only
 * (QCB_ERR_STATE on a slab).  Synchronous. */
int qcb_heatbath_plaquette(qcb_lattice* lat, double beta, int n_sweeps, int n_hits, uint64_t seed,
                           uint64_t sweep_offset, double* plaq);
/* The same sweeps with the reference's frozen links (src/geometry/GeometryCB.cpp:33-56):
 * the lattice is cut into blocks of edge l_core (one block per MPI rank in the reference)
 * and, after the field has been translated by the cumulative shift `shift` of its random
 * shifts (src/mpi/Shift.cpp:163-186), link (x, mu) is not updated when
 * (x_d + shift_d) % l_core == 0 for some d != mu.  The lattice is not moved: the links keep
 * the frame of the untranslated field, and qcb_translate by the cumulative shift gives the
 * reference's frame.  l_core must divide every extent; shift is taken mod l_core. */
int qcb_heatbath_frozen(qcb_lattice* lat, double beta, int n_sweeps, int n_hits, uint64_t seed,
                        uint64_t sweep_offset, int l_core, const int shift[4]);
/* Periodic translation of the whole field, U'(x) = U(x - shift) (mpi::shift::shift_field,
 * src/mpi/Shift.cpp:109-160, on one device).  shift is taken mod the extents.  Uses the
 * lattice's flow work space (allocated on first use). */
int qcb_translate(qcb_lattice* lat, const int shift[4]);

/* ---- observables -------------------------------------------------------------------
 * mpi::observables::mean_plaquette_global (src/observables/observables_mpi.cpp:8-43):
 * sum_{x, mu<nu} Re tr P_{mu nu}(x) / 3, divided by 6V.  FP64 accumulation. */
int qcb_plaquette(qcb_lattice* lat, double* out);
/* topo_q_e_clover_global (observables_mpi.cpp:61-150): clover charge Q (total) and energy
 * density E = (1/V) sum_x 1/2 sum_{mu<nu} |F_{mu nu}|^2 with F = (C - C^dagger)/8. */
int qcb_topo_qe(qcb_lattice* lat, double* q, double* e);

/* ---- allocation-free plaquette ---------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory (a
 * host whose pool allocator owns the device memory, or a loop where cudaMalloc's implicit
 * device synchronisation is not acceptable): the mean plaquette of links already on the
 * device, in this library's layout (dims, precision, storage and stride as reported by
 * qcb_lattice_device_links), written to out[0] (caller-owned device memory) on `stream`
 * (a cudaStream_t; NULL = legacy default stream), asynchronously.  It calls no cudaMalloc,
 * cudaFree or other allocating routine: its reduction scratch is a static device array of
 * QCB_NOALLOC_MAX_PARTIALS doubles (16 KiB per GPU, held until the process exits).  Every
 * call looks up that array's device address for the current device; the first call on a
 * device also loads the library's device code there (make it before any stream capture).
 * Calls share the array, so calls that overlap on the GPU race; requests that would need
 * more partial sums than the array holds are rejected with QCB_ERR_INVALID, and so are
 * links not aligned to the storage's chunk size (16 bytes; 8 for FP32 18-real) and an out
 * pointer not aligned to 8 bytes. */
#define QCB_NOALLOC_MAX_PARTIALS 2048
int qcb_plaquette_noalloc(const void* links, const int dims[4], int precision, int storage, size_t stride,
                          double* out, void* stream);

/* ---- Wilson flow -------------------------------------------------------------------
 * mpi::observables::topo_charge_flowed (observables_mpi.cpp:153-178) with
 * GradientFlow::rk3_step (src/flow/gradient_flow.cpp:15-128): on a copy of the links,
 * for s < n_steps_gf: record (t, Q, E) into tQE[3s..3s+2], then n_rk_steps RK3 steps of
 * size eps.  The lattice itself is left unchanged.  tQE holds 3*n_steps_gf doubles. */
int qcb_flow_measure(qcb_lattice* lat, double eps, int n_steps_gf, int n_rk_steps,
                     double* tQE);
/* n RK3 steps of size eps applied to the lattice in place (no measurement). */
int qcb_flow_steps(qcb_lattice* lat, double eps, int n);

/* ---- batches of lattices ------------------------------------------------------------
 * No single counterpart in the reference (it runs one lattice per process,
 * src/bin/gauge_hb_ncb.cpp:18-201).  A batch advances many independent lattices of any
 * sizes (same context, precision and storage) in one persistent cooperative launch per
 * phase: work items (lattice, level, tile of sites) run level-major, each lattice's levels
 * in order, different lattices overlapping.  Every result is bit-identical to running the
 * lattice alone through qcb_heatbath / qcb_flow_steps with the same seed and sweep counter.
 * The batch borrows the lattices: they must outlive it. */
typedef struct qcb_batch qcb_batch;
int qcb_batch_create(qcb_ctx* ctx, int n, qcb_lattice* const* lats, qcb_batch** out);
int qcb_batch_destroy(qcb_batch* b);
/* Sites per work item for the heatbath / flow of each lattice (multiples of 32 in
 * [32, 65536]); NULL keeps the current value (default 256). */
int qcb_batch_set_tiles(qcb_batch* b, const int* hb_tile, const int* flow_tile);
int qcb_batch_get_tiles(qcb_batch* b, int* hb_tile, int* flow_tile);
/* n_sweeps checkerboard sweeps of every lattice l at betas[l], seeds[l], sweeps
 * sweep_offsets[l] .. sweep_offsets[l] + n_sweeps - 1 (one launch).  Asynchronous. */
int qcb_batch_heatbath(qcb_batch* b, const double* betas, int n_sweeps, int n_hits, const uint64_t* seeds,
                       const uint64_t* sweep_offsets);
/* n RK3 steps of size eps on every lattice, in place (one launch). */
int qcb_batch_flow_steps(qcb_batch* b, double eps, int n_steps);
/* Per-lattice mean plaquette / clover (Q, E) of every lattice (one launch each). */
int qcb_batch_plaquette(qcb_batch* b, double* out);
int qcb_batch_topo_qe(qcb_batch* b, double* q, double* e);
/* A whole batched workload as one CUDA graph: n_sweeps heatbath sweeps in place, the mean
 * plaquette, then the Wilson flow on copies of the links with (t, Q, E) recorded before
 * each of n_groups groups of rk_per_group RK3 steps and once after the last group.
 * results holds n * (1 + 3 * (n_groups + 1)) doubles: per lattice the plaquette, then the
 * records.  The graph is captured on the first call with a given plan and replayed after;
 * *used_graph (if not NULL) tells whether the graph path ran. */
typedef struct qcb_batch_plan {
  int n_sweeps, n_hits;
  double eps;
  int n_groups, rk_per_group;
} qcb_batch_plan;
int qcb_batch_run(qcb_batch* b, const qcb_batch_plan* plan, const double* betas, const uint64_t* seeds,
                  const uint64_t* sweep_offsets, double* results, int* used_graph);
/* Project-written autotuner: for each distinct lattice size of the batch, times the
 * heatbath and the flow of that size's lattices on scratch copies for candidate tiles and
 * keeps the fastest; results are cached in the JSON file cache_path (created if absent,
 * NULL = no cache) under keys "<device name>|<precision>-<storage>|<hb|flow>|LxLyLzLt". */
int qcb_batch_autotune(qcb_batch* b, const char* cache_path);

/* ---- slabs: one lattice split along t over several devices or processes ------------------
 * A slab holds global times t0 .. t0 + t_local - 1 of a lattice of extents global_dims as
 * local times 1 .. t_local, plus one halo time slice on each side (local extents Lx, Ly, Lz,
 * t_local + 2).  t0 and t_local must be even.  It replaces the reference's MPI block
 * decomposition with halo exchange (src/mpi/HalosExchange.cpp, src/geometry/GeometryCB.cpp)
 * by a decomposition along t with one face exchange per heatbath pass or flow stage.
 * Random numbers are keyed by the global link, so N slabs reproduce the whole-lattice run
 * bit for bit.  qcb_set_links / qcb_get_links use the local sites (halos included);
 * qcb_plaquette and qcb_topo_qe return the slab's contribution to the global mean plaquette,
 * Q and E (sum them over the slabs).  qcb_heatbath, qcb_heatbath_frozen, qcb_translate,
 * qcb_flow_steps, qcb_flow_measure and the ILDG calls return QCB_ERR_STATE on a slab. */
int qcb_lattice_create_slab(qcb_ctx* ctx, const int global_dims[4], int t0, int t_local, int precision,
                            int storage, qcb_lattice** out);
int qcb_slab_info(const qcb_lattice* lat, int global_dims[4], int* t0, int* t_local);
/* One checkerboard heatbath pass (direction mu, global parity) of sweep `sweep`; on a
 * whole lattice the same as one pass of qcb_heatbath. */
int qcb_heatbath_pass(qcb_lattice* lat, int mu, int parity, double beta, int n_hits, uint64_t seed,
                      uint64_t sweep);
/* Stage 1, 2 or 3 of RK3 step `step` of the Wilson flow, in place as qcb_flow_steps: step s
 * uses the links (a) and the lattice's work buffer (b), swapped for odd s; stage 1 writes b,
 * stage 2 writes a, stage 3 writes b.  qcb_flow_finish(lat, n) after n steps moves the
 * result into the links when n is odd. */
int qcb_flow_stage(qcb_lattice* lat, int stage, double eps, int step);
int qcb_flow_finish(qcb_lattice* lat, int n_steps);
/* Face exchange between slab `lower` and the slab `upper` that follows it in time
 * (periodically): lower's last own slice -> upper's low halo, upper's first own slice ->
 * lower's high halo, for the links (which = 0) or the flow work buffer (which = 1), of
 * direction mu (-1: all) and global parity (-1: both).  Waits for both slabs' streams;
 * peer copies when the slabs are on different devices. */
int qcb_slab_exchange(qcb_lattice* lower, qcb_lattice* upper, int which, int mu, int parity);
/* Device pointers of one face, for an exchange by another transport (NCCL send / recv):
 * side 0 low halo, 1 first own slice, 2 last own slice, 3 high halo; *n_segments contiguous
 * segments of *bytes bytes each. */
int qcb_slab_face(qcb_lattice* lat, int which, int side, int mu, int parity, void** segments, size_t* bytes,
                  int* n_segments);
/* Copies one face to (to_face = 0) or from (to_face = 1) a contiguous buffer of
 * n_segments * bytes bytes, host or device memory; synchronous. */
int qcb_slab_face_copy(qcb_lattice* lat, int which, int side, int mu, int parity, void* buf, int to_face);
/* The faces of every direction mu (-1: all, ascending) and every global parity (-1: both,
 * ascending) of one side, packed back to back in buf (each face n_segments * bytes bytes, in
 * the order of qcb_slab_face) or unpacked from it, enqueued on the context's stream without
 * waiting: one call per side per exchange, ordered with the slab's kernels.  buf is device
 * memory or pinned host memory that stays valid until the stream has run the copies. */
int qcb_slab_faces_copy_async(qcb_lattice* lat, int which, int side, int mu, int parity, void* buf,
                              int to_face);

/* ---- failure detection --------------------------------------------------------------
 * The persistent batch and server kernels wait on per-lattice counters that other blocks
 * advance; every wait is bounded (2 s of wall-clock time or 2^28 polls), after which the
 * block counts a timeout, raises an abort flag that makes every block return, and the host
 * reports QCB_ERR_CUDA with the count.  qcb_wait_selftest runs that path on purpose: four
 * co-resident blocks wait on a device flag that nothing sets; the first gives up after
 * limit_s (at most 5 s) and aborts the others.  On return *timeouts = 1 and *aborted = 1 and
 * the context stays usable.  No GPU fault is involved. */
int qcb_wait_selftest(qcb_ctx* ctx, double limit_s, uint32_t* timeouts, uint32_t* aborted);

/* ---- serving ---------------------------------------------------------------------------
 * No counterpart in the reference.  A request server with continuous batching: jobs
 * (Wilson-flow measurements and generate-N-sweeps runs on resident lattices of any sizes)
 * are admitted in arrival order while the server's device work-space arena (its HBM budget)
 * and job slots allow; every tick advances every admitted job by a quantum of sweeps or RK3
 * steps in ONE persistent launch (heatbath and flow items mixed), measures the jobs that
 * finish, and admits new arrivals at the tick boundary.  A job's result does not depend on
 * what else runs with it (counter-based random numbers, per-lattice arithmetic).  The
 * server runs its own scheduler thread and CUDA stream on the context's device; a job's
 * lattice is lent to the server from submission until its result is returned (a sweeps job
 * updates it in place; a flow job flows a copy held in the server's arena). */
typedef struct qcb_server qcb_server;
enum { QCB_JOB_FLOW = 1, QCB_JOB_SWEEPS = 2 };
typedef struct qcb_job {
  int kind;               /* QCB_JOB_FLOW or QCB_JOB_SWEEPS */
  qcb_lattice* lat;       /* resident input; precision and storage of the server */
  double beta;            /* sweeps: coupling */
  uint64_t seed;          /* sweeps: Philox key */
  uint64_t sweep_offset;  /* sweeps: counter of the first sweep */
  int n_sweeps, n_hits;   /* sweeps */
  double eps;             /* flow: step size */
  int n_steps;            /* flow: RK3 steps; Q and E are measured at t = n_steps * eps */
} qcb_job;
typedef struct qcb_job_result {
  uint64_t id;
  int status;            /* QCB_OK, QCB_ERR_CANCELLED, QCB_ERR_KP_CAP, ... */
  int kind;
  double plaquette;      /* sweeps: mean plaquette after the last sweep */
  double t, q, e;        /* flow: flow time, clover charge, energy density */
  double submit_s, admit_s, finish_s; /* server clock (s since creation) */
} qcb_job_result;
typedef struct qcb_server_config {
  int precision, storage; /* of every job's lattice */
  size_t hbm_budget;      /* bytes of device work space (0: 80% of the free memory) */
  int max_jobs;           /* concurrent jobs (0: 256) */
  int quantum_sweeps;     /* sweeps per sweeps-job per tick (0: 2) */
  int quantum_steps;      /* RK3 steps per flow-job per tick (0: 4) */
  int tile;               /* sites per work item (0: 256) */
} qcb_server_config;
typedef struct qcb_server_stats {
  uint64_t submitted, admitted, completed, ticks;
  int max_active;
  size_t arena_bytes, arena_peak;
} qcb_server_stats;
int qcb_server_create(qcb_ctx* ctx, const qcb_server_config* cfg, qcb_server** out);
/* Non-blocking; the job's lattice must not be touched until its result is polled. */
int qcb_server_submit(qcb_server* s, const qcb_job* job, uint64_t* id);
/* Non-blocking: copies up to max finished results (in completion order) into out. */
int qcb_server_poll(qcb_server* s, qcb_job_result* out, int max, int* n);
/* Blocks until every submitted job has finished or timeout_s elapses (QCB_ERR_STATE). */
int qcb_server_drain(qcb_server* s, double timeout_s);
/* A pending job is dropped, an admitted one stops at the next tick; its result carries
 * QCB_ERR_CANCELLED. */
int qcb_server_cancel(qcb_server* s, uint64_t id);
int qcb_server_stats_get(qcb_server* s, qcb_server_stats* st);
double qcb_server_clock(qcb_server* s);
int qcb_server_destroy(qcb_server* s);

/* ---- event-chain Monte Carlo ------------------------------------------------------------
 * mpi::ecmccb::sample_persistant (src/ecmc/ecmc_mpi_cb.cpp:496-637) driven by
 * generate_ecmc_cb (src/bin/gauge_ecmc_ncb.cpp:20-269).  The lattice is cut into blocks of
 * edge l_core (one per MPI rank in the reference) and every block runs its own persistent
 * event chain, all chains at once: one sample call moves every chain until it has travelled
 * theta_sample (lifts, site refreshes and R refreshes as in the reference).  The blocks are
 * placed as in qcb_heatbath_frozen: after the cumulative shift `shift` of the field's random
 * translations, links with (x_d + shift_d) % l_core == 0 for some d != mu are frozen and
 * block (bx, by, bz, bt) starts at x_d = b_d l_core - shift_d; its chain keeps its
 * block-local position across calls.  Chain c = ((bx nby + by) nbz + bz) nbt + bt (the MPI
 * Cartesian rank order) draws from Philox4x32-10 keyed by seed with counter (draw, c); the
 * set of 10001 SU(3) elements near the identity (ecmc_set, src/su3/utils.cpp:119-127) is
 * drawn once per call and shared by the chains.  The links are updated in FP64 whatever the
 * lattice's storage.  The lattice is borrowed and must outlive the object. */
typedef struct qcb_ecmc qcb_ecmc;
typedef struct qcb_ecmc_params {
  double beta;
  double theta_sample;        /* param_theta_sample: angle travelled per sample call */
  double theta_refresh_site;  /* param_theta_refresh_site */
  double theta_refresh_R;     /* param_theta_refresh_R */
  double epsilon_set;         /* epsilon_set: spread of the set around the identity, in [0, 1] */
  int poisson;                /* budgets drawn from exponentials of these means */
  int l_core;                 /* block edge, >= 3, dividing every extent */
} qcb_ecmc_params;
/* One chain (LocalChainState, src/ecmc/ecmc_mpi_cb.h:15-35), 256 bytes. */
typedef struct qcb_ecmc_chain {
  double R[18];               /* row-major 3x3 of (re, im) */
  double theta_refresh_site, theta_refresh_R;   /* current budgets */
  double travelled_site, travelled_R;           /* angle travelled since the last refreshes */
  uint64_t draws;             /* position in the chain's Philox stream */
  uint64_t events, lifts, revs;                 /* event, lift and same-site-lift counters */
  int32_t site[4];            /* block-local x, y, z, t of the active link, in [0, l_core) */
  int32_t mu, epsilon;        /* direction of the active link, sense of rotation (+1 / -1) */
  int32_t initialized;        /* 0: drawn at the next call (site, mu, epsilon, R, budgets) */
  int32_t status;             /* latest call: bit 0 non-finite event angle; bit 1 2^26 events */
  int32_t set_counter;        /* lifts since the chain's near-identity set was renewed */
  int32_t pad[3];
} qcb_ecmc_chain;
int qcb_ecmc_create(qcb_lattice* lat, const qcb_ecmc_params* params, uint64_t seed, qcb_ecmc** out);
int qcb_ecmc_destroy(qcb_ecmc* e);
int qcb_ecmc_num_chains(const qcb_ecmc* e, int* n);
/* Lanes of a warp that run one chain: 1, 3 or 6 (each lane computes an equal share of an
 * event's six staples, lanes 0-2 also one product each of a lift), or 0 to let the library
 * choose from the number of chains (the default).  Results do not depend on it, bit for
 * bit.  qcb_ecmc_lanes returns the lanes the next call will use. */
int qcb_ecmc_set_lanes(qcb_ecmc* e, int lanes);
int qcb_ecmc_lanes(const qcb_ecmc* e, int* lanes);
/* One sample call of every chain (asynchronous).  shift = cumulative shift of the field. */
int qcb_ecmc_sample(qcb_ecmc* e, const int shift[4]);
/* n sample calls in a row, call k with the cumulative shift shifts[4k .. 4k+3], with the
 * lattice packed into the chains' FP64 copy once before and unpacked once after: the same
 * result as n qcb_ecmc_sample calls, bit for bit (asynchronous).  If a launch fails after
 * k calls, those k calls stay complete: their link updates are unpacked into the lattice,
 * the chain records and the call count cover exactly them, and QCB_ERR_CUDA is returned. */
int qcb_ecmc_sample_n(qcb_ecmc* e, const int* shifts, int n);
/* Waits, then sums the chains' events, lifts and same-site lifts into out[0..2]; with reset,
 * zeroes the three counters afterwards (the reference resets them after each plaquette
 * measurement).  If a chain stopped early (non-finite event angle, or 2^26 events in one
 * call) since the previous check, returns QCB_ERR_STATE once; the chain records keep the
 * status bits of their latest call. */
int qcb_ecmc_counters(qcb_ecmc* e, uint64_t out[3], int reset);
/* Copies the chain records (qcb_ecmc_num_chains of them) and the number of sample calls
 * made so far (which keys the chains' near-identity sets in the next call) to / from host
 * memory; synchronous. */
int qcb_ecmc_get_chains(qcb_ecmc* e, qcb_ecmc_chain* chains, uint64_t* calls);
int qcb_ecmc_set_chains(qcb_ecmc* e, const qcb_ecmc_chain* chains, uint64_t calls);

/* ---- input file ----------------------------------------------------------------------
 * io::load_params(..., RunParamsHbCB&) (src/io/io.cpp:353-399) with the defaults of
 * src/io/params.h:46-63.  Host-only.  Strings are NUL-terminated and truncated to fit. */
typedef struct qcb_hb_params {
  int L_core, n_core_dims, cold_start, N_switch_eo, N_shift, seed;
  double beta;
  int N_samples, N_hits, N_sweeps, N_therm;
  int topo, N_shift_plaquette, N_shift_topo, N_steps_gf, N_rk_steps;
  int save_each_shifts;
  char run_name[256];
  char run_dir[1024];
} qcb_hb_params;
int qcb_params_default(qcb_hb_params* p);
int qcb_params_load(const char* path, qcb_hb_params* p);

/* io::load_params(..., RunParamsECB&) (src/io/io.cpp:298-341) with the defaults of
 * src/io/params.h:9-44, for the event-chain driver.  Same line rules as qcb_params_load;
 * keys L_core, n_core_dims, cold_start, seed, N_shift, beta, param_theta_sample,
 * param_theta_refresh_site, param_theta_refresh_R, poisson, epsilon_set, N_shift_plaquette,
 * N_shift_therm, topo, N_shift_topo, N_steps_gf, N_rk_steps, run_name, run_dir,
 * save_each_shifts.  ecmc.l_core is set to L_core.  Host-only. */
typedef struct qcb_ecmc_run_params {
  int L_core, n_core_dims, cold_start, seed, N_shift;
  qcb_ecmc_params ecmc;
  int N_therm, topo, N_shift_plaquette, N_shift_topo, N_steps_gf, N_rk_steps, save_each_shifts;
  char run_name[256];
  char run_dir[1024];
} qcb_ecmc_run_params;
int qcb_ecmc_run_params_default(qcb_ecmc_run_params* p);
int qcb_ecmc_run_params_load(const char* path, qcb_ecmc_run_params* p);

#ifdef __cplusplus
}
#endif
#endif /* QCB_H */
