// gauge_ecmc_ncb — drop-in replacement of the reference's event-chain driver
// (src/bin/gauge_ecmc_ncb.cpp:20-317) on one B200 through the C ABI (include/qcb.h).
//
//   gauge_ecmc_ncb <input_file.txt>
//
// Same input keys (src/io/io.cpp:298-341), same outputs under run_dir/run_name/:
//   run_name                       ILDG/LIME configuration (src/io/ildg.cpp:34-136)
//   run_name_plaquette.txt         one mean plaquette per line, fixed, 10 decimals
//   run_name_topo.txt              "t Q E" per line, fixed, 10 decimals
//   run_name_nbevent.txt           "events lifts same-site-lifts lambda" per plaquette sample
//                                  (io::save_event_nb, io.cpp:49-75)
//   run_name_params.txt            parameter log + "Saved shift N" / "Saved final state !"
//   run_name_state/run_name_state<r>.txt   chain r's state (io::save_state, io.cpp:140-192)
//   run_name_seed/run_name_seed<r>.txt     chain r's generator position
//
// One process runs every chain: the global lattice (L_core * n_core_dims)^4 is cut into
// n_core_dims^4 blocks of edge L_core, chain r = MPI rank r of the reference, and all chains
// advance in one launch per shift.  Each shift draws the random translation (x, y, z, t),
// each uniform in [0, L_core), from std::mt19937_64 (src/mpi/Shift.cpp:163-186); the field
// is not moved, the cumulative shift places the blocks, and the field is translated into the
// reference's frame before a configuration is written.  Differences, by design: chain r
// draws from Philox4x32-10 keyed by `seed` (its seed file stores the key, its draw count and
// the number of sample calls; seed file 0 also holds the translations' std::mt19937_64
// state), each chain's near-identity set is drawn from counters keyed by the chain, the call
// and the set's renewal count (renewed, as the reference renews its rank's set, at every call
// and every 10000 lifts), and the state file separates set_counter from event_counter by a
// space (the reference writes them with no separator, io.cpp:174-175).
// Optional extra keys: precision = fp64 | fp32, storage = 18 | 12, device = N.
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "driver_common.h"
#include "qcb.h"

namespace fs = std::filesystem;
using drv::append_params_line;
using drv::ensure_dir;
using drv::fmt;

namespace {

void save_params(const qcb_ecmc_run_params& rp, const drv::RunDir& rd) {
  // io::save_params(const RunParamsECB&, ...) (io.cpp:577-627)
  std::ostringstream f;
  f << std::boolalpha;
  f << "\n#########################################################\n\n";
  f << "# Lattice params\n";
  f << "L_core = " << rp.L_core << "\n";
  f << "n_core_dims = " << rp.n_core_dims << "\n";
  f << "cold_start = " << (rp.cold_start != 0) << "\n\n";
  f << "# Run params\n";
  f << "seed = " << rp.seed << "\n";
  f << "N_shift_therm = " << rp.N_therm << "\n";
  f << "N_shift = " << rp.N_shift << "\n";
  f << "# ECMC params\n";
  f << "beta = " << rp.ecmc.beta << "\n";
  f << "theta_sample = " << rp.ecmc.theta_sample << "\n";
  f << "theta_refresh_site = " << rp.ecmc.theta_refresh_site << "\n";
  f << "theta_refresh_R = " << rp.ecmc.theta_refresh_R << "\n";
  f << "epsilon_set = " << rp.ecmc.epsilon_set << "\n";
  f << "poisson = " << (rp.ecmc.poisson != 0) << "\n\n";
  f << "# Plaquette params\n";
  f << "N_shift_plaquette = " << rp.N_shift_plaquette << "\n\n";
  f << "# Topo params\n";
  f << "topo = " << (rp.topo != 0) << "\n";
  f << "N_shift_topo = " << rp.N_shift_topo << "\n";
  f << "N_steps_gf = " << rp.N_steps_gf << "\n";
  f << "N_rk_steps = " << rp.N_rk_steps << "\n\n";
  f << "#Save params\n";
  f << "save_each_shifts = " << rp.save_each_shifts << "\n\n";
  append_params_line(rd, f.str());
  std::cout << "Parameters saved in " << rd.file("_params.txt") << "\n";
}

void print_parameters(const qcb_ecmc_run_params& rp) {
  // print_parameters(const RunParamsECB&, ...) (io.cpp:538-575)
  std::cout << "==========================================" << std::endl;
  std::cout << "ECMC - one chain per block, one GPU" << std::endl;
  std::cout << "==========================================" << std::endl;
  std::cout << "Run name : " << rp.run_name << "\n";
  std::cout << "---Lattice params---\n";
  std::cout << "Total lattice size : " << rp.L_core * rp.n_core_dims << "^4\n";
  std::cout << "Local lattice size : " << rp.L_core << "^4\n\n";
  std::cout << "---Run params---\n";
  std::cout << "Initial seed : " << rp.seed << "\n";
  std::cout << "Thermalization shifts : " << rp.N_therm << "\n";
  std::cout << "Number of shifts : " << rp.N_shift << "\n";
  std::cout << "Save each : " << rp.save_each_shifts << " shifts\n\n";
  std::cout << "---ECMC params---\n";
  std::cout << "Beta : " << rp.ecmc.beta << "\n";
  std::cout << "Theta sample : " << rp.ecmc.theta_sample << "\n";
  std::cout << "Theta refresh site : " << rp.ecmc.theta_refresh_site << "\n";
  std::cout << "Theta refresh R : " << rp.ecmc.theta_refresh_R << "\n";
  std::cout << "Epsilon set : " << rp.ecmc.epsilon_set << "\n";
  std::cout << "Poisson law : " << (rp.ecmc.poisson ? "Yes" : "No") << "\n\n";
  std::cout << "---Measures params---\n";
  std::cout << "Number of <P> samples : " << rp.N_shift / rp.N_shift_plaquette << "\n";
  std::cout << "Measure <P> each : " << rp.N_shift_plaquette << " shifts\n";
  std::cout << "Measure topo : " << (rp.topo ? "Yes" : "No") << "\n";
  if (rp.topo) {
    std::cout << "Number of Q samples : " << rp.N_shift / rp.N_shift_topo << "\n";
    std::cout << "Measure Q each : " << rp.N_shift_topo << " shifts\n\n";
    std::cout << "---Gradient Flow---\n";
    std::cout << "Number of RK3 steps per GF step : " << rp.N_rk_steps << "\n";
    std::cout << "Number of GF steps : " << rp.N_steps_gf << "\n";
  }
  std::cout << "==========================================" << std::endl;
}

struct Run {
  qcb_ecmc_run_params rp;
  drv::RunDir rd;
  qcb_ctx* ctx = nullptr;
  qcb_lattice* lat = nullptr;
  qcb_ecmc* ecmc = nullptr;
  int n_chains = 0;
  uint64_t key = 0;
  int cum[4] = {0, 0, 0, 0};  // cumulative shift not yet applied to the stored links
  std::vector<int> pending;   // cumulative shifts of sample calls not yet launched
  std::mt19937_64 shift_rng;
  std::vector<size_t> event_nb, lift_nb, rev_nb;
  std::vector<double> lambda;

  int Lext() const { return rp.L_core + 2; }
  fs::path state_path(int r) const {
    return rd.path() / (rd.name + "_state") / (rd.name + "_state" + std::to_string(r) + ".txt");
  }
  fs::path seed_path(int r) const {
    return rd.path() / (rd.name + "_seed") / (rd.name + "_seed" + std::to_string(r) + ".txt");
  }

  // mpi::shift::random_shift + mpi::ecmccb::sample_persistant on every rank.  The sample
  // calls between two measurements are launched together (one pack and one unpack of the
  // lattice): flush() runs them before anything reads the links or the chains.
  void shift_and_sample() {
    std::uniform_int_distribution<int> rand_l_shift(0, rp.L_core - 1);
    int s[4];
    for (int d = 0; d < 4; ++d) s[d] = rand_l_shift(shift_rng);
    std::cout << "Shift (" << s[0] << ", " << s[1] << ", " << s[2] << ", " << s[3] << ")\n";
    const int Lg = rp.L_core * rp.n_core_dims;
    for (int d = 0; d < 4; ++d) {
      cum[d] = (cum[d] + s[d]) % Lg;
      pending.push_back(cum[d]);
    }
  }
  void flush() {
    if (pending.empty()) return;
    CHECK(qcb_ecmc_sample_n(ecmc, pending.data(), (int)(pending.size() / 4)), "ECMC sample");
    pending.clear();
  }
  double plaquette() {
    flush();
    double p = 0;
    CHECK(qcb_plaquette(lat, &p), "plaquette");
    return p;
  }
  // Event counting after a plaquette sample (gauge_ecmc_ncb.cpp:176-210): lambda is the
  // angle travelled by all chains since the last sample over their lifts.
  void count_events() {
    flush();
    uint64_t c[3];
    CHECK(qcb_ecmc_counters(ecmc, c, 1), "ECMC counters");
    const double total = (double)rp.N_shift_plaquette * rp.ecmc.theta_sample * (double)n_chains;
    const double lam = total / (double)c[1];
    const size_t avg_lift = c[1] / n_chains, avg_rev = c[2] / n_chains, avg_event = c[0] / n_chains;
    lambda.push_back(lam);
    lift_nb.push_back(avg_lift);
    event_nb.push_back(avg_event);
    rev_nb.push_back(avg_rev);
    std::cout << ">>> Average λ = " << lam << ", Events : " << avg_event
              << " (Reversibility : " << (double)avg_rev / (double)avg_lift * 100 << "%)\n";
  }
  std::vector<double> topo() {
    flush();
    std::vector<double> tqe(3 * (size_t)rp.N_steps_gf);
    const double eps = 0.02;  // hard-coded in the reference driver (gauge_ecmc_ncb.cpp:62)
    CHECK(qcb_flow_measure(lat, eps, rp.N_steps_gf, rp.N_rk_steps, tqe.data()), "flow");
    for (int s = 0; s < rp.N_steps_gf; ++s) {
      const double t = tqe[3 * s], q = tqe[3 * s + 1], e = tqe[3 * s + 2];
      std::cout << "n = " << s << ", t = " << fmt(t, 2) << ", Q = " << fmt(q, 6) << ", t²E = " << fmt(t * t * e, 6)
                << "\n";
    }
    return tqe;
  }
  void save_event_nb() {
    ensure_dir(rd.path());
    fs::path p = rd.file("_nbevent.txt");
    std::ofstream f(p, std::ios::out | std::ios::app);
    if (!f.is_open()) {
      std::cout << "Could not open file " << p << "\n";
      return;
    }
    for (size_t i = 0; i < event_nb.size(); i++)
      f << event_nb[i] << " " << lift_nb[i] << " " << rev_nb[i] << " " << lambda[i] << "\n";
    std::cout << "Number of events written in " << p << "\n";
    event_nb.clear();
    lift_nb.clear();
    rev_nb.clear();
    lambda.clear();
  }
  void save_conf() {
    flush();
    if (cum[0] | cum[1] | cum[2] | cum[3]) {
      // the blocks keep their place: after U'(x) = U(x - cum) they start at b * L_core
      CHECK(qcb_translate(lat, cum), "translate");
      cum[0] = cum[1] = cum[2] = cum[3] = 0;
    }
    ensure_dir(rd.path());
    fs::path p = rd.path() / rd.name;
    CHECK(qcb_save_ildg(lat, p.string().c_str()), "save ILDG");
    std::cout << "Configuration saved in " << p << "\n";
  }
  // io::save_state (io.cpp:140-192) per chain, site as the index of the reference's padded
  // block ((t Lext + z) Lext + y) Lext + x with coordinates local + 1; plus the seed files.
  void save_state() {
    flush();
    std::vector<qcb_ecmc_chain> ch(n_chains);
    uint64_t calls = 0;
    CHECK(qcb_ecmc_get_chains(ecmc, ch.data(), &calls), "ECMC chains");
    ensure_dir(state_path(0).parent_path());
    ensure_dir(seed_path(0).parent_path());
    const int E = Lext();
    for (int r = 0; r < n_chains; ++r) {
      const qcb_ecmc_chain& c = ch[r];
      const long site = (((long)(c.site[3] + 1) * E + (c.site[2] + 1)) * E + (c.site[1] + 1)) * E + (c.site[0] + 1);
      std::ofstream f(state_path(r));
      if (!f.is_open()) {
        std::cerr << "[Rank " << r << "] Error: Could not open state file for writing: " << state_path(r) << std::endl;
        return;
      }
      f << std::setprecision(17);
      f << site << " " << c.mu << " " << c.epsilon << " " << c.travelled_site << " " << c.travelled_R << " "
        << c.theta_refresh_site << " " << c.theta_refresh_R << " " << c.set_counter << " " << c.events << " " << c.lifts << " "
        << c.revs << " " << " " << (c.initialized != 0) << "\n";
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) f << c.R[2 * (3 * i + j)] << " " << c.R[2 * (3 * i + j) + 1] << " ";
        f << "\n";
      }
      std::ofstream s(seed_path(r));
      s << "qcb-philox4x32-10-ecmc " << key << " " << c.draws << " " << calls << "\n";
      if (r == 0) s << shift_rng << "\n";  // the translations' generator (io::save_seed, io.cpp:108-138)
    }
    std::cout << "ECMC Chain saved in : " << state_path(0).parent_path() << std::endl;
  }
  // io::load_state (io.cpp:194-231) and the seed files; a missing state file leaves that
  // chain uninitialised (drawn at the next call), as in the reference.
  void load_state() {
    std::vector<qcb_ecmc_chain> ch(n_chains);
    memset(ch.data(), 0, ch.size() * sizeof(qcb_ecmc_chain));
    uint64_t calls = 0;
    const int E = Lext();
    for (int r = 0; r < n_chains; ++r) {
      std::ifstream s(seed_path(r));
      std::string tag;
      uint64_t k = 0, draws = 0, cl = 0;
      if (s.is_open() && (s >> tag >> k >> draws >> cl) && tag == "qcb-philox4x32-10-ecmc") {
        key = k;
        ch[r].draws = draws;
        calls = cl;
        if (r == 0 && !(s >> shift_rng)) shift_rng.seed(key);
      }
      std::ifstream f(state_path(r));
      if (!f.is_open()) continue;
      long site = 0;
      uint64_t set_counter = 0;
      bool init = false;
      qcb_ecmc_chain& c = ch[r];
      f >> site >> c.mu >> c.epsilon >> c.travelled_site >> c.travelled_R >> c.theta_refresh_site >>
          c.theta_refresh_R >> set_counter >> c.events >> c.lifts >> c.revs >> init;
      for (int k2 = 0; k2 < 18; ++k2) f >> c.R[k2];
      if (!f) {
        std::cerr << "Could not read " << state_path(r) << "\n";
        c.initialized = 0;
        continue;
      }
      c.site[0] = (int)(site % E) - 1;
      c.site[1] = (int)((site / E) % E) - 1;
      c.site[2] = (int)((site / E / E) % E) - 1;
      c.site[3] = (int)(site / E / E / E) - 1;
      c.initialized = init ? 1 : 0;
      c.set_counter = (int32_t)(set_counter % 10000);
    }
    CHECK(qcb_ecmc_set_chains(ecmc, ch.data(), calls), "ECMC chains");
    std::cout << "Successfully loaded ECMC chain state from: " << state_path(0).parent_path() << std::endl;
  }
};

void generate_ecmc_cb(Run& R, bool existing, int precision, int storage, int device) {
  qcb_ecmc_run_params& rp = R.rp;
  const int L = rp.L_core * rp.n_core_dims;
  const int dims[4] = {L, L, L, L};
  CHECK(qcb_ctx_create(device, 0, &R.ctx), "context");
  CHECK(qcb_lattice_create(R.ctx, dims, precision, storage, &R.lat), "lattice");
  R.key = (uint64_t)(int64_t)rp.seed;
  if (!rp.cold_start) CHECK(qcb_hot_start(R.lat, R.key), "hot start");
  R.shift_rng.seed(R.key);
  qcb_ecmc_params ep = rp.ecmc;
  ep.l_core = rp.L_core;
  if (existing) {
    fs::path p = R.rd.path() / R.rd.name;
    CHECK(qcb_load_ildg(R.lat, p.string().c_str()), "read ILDG");
  }
  // the seed files carry the key of a resumed run; read it before the chains are created
  if (existing) {
    std::ifstream s(R.seed_path(0));
    std::string tag;
    uint64_t k = 0;
    if (s.is_open() && (s >> tag >> k) && tag == "qcb-philox4x32-10-ecmc") R.key = k;
  }
  CHECK(qcb_ecmc_create(R.lat, &ep, R.key, &R.ecmc), "ECMC chains");
  CHECK(qcb_ecmc_num_chains(R.ecmc, &R.n_chains), "ECMC chains");
  if (existing) R.load_state();
  save_params(rp, R.rd);
  print_parameters(rp);

  std::vector<double> plaquette, tQE_tot;
  std::cout << "\n\n===========================================\n";
  std::cout << "Thermalisation : " << rp.N_therm << " shifts\n";
  std::cout << "===========================================\n";
  for (int i = 0; i < rp.N_therm; i++) {
    std::cout << "\n\n==========" << "(Therm) Shift " << i << "==========\n";
    R.shift_and_sample();
    if (i % rp.N_shift_plaquette == 0) {
      double p = R.plaquette();
      std::cout << "====== Plaquette ======\n";
      std::cout << "(Therm) Sample " << i / rp.N_shift_plaquette << ", <P> = " << p << "\n";
    }
  }
  std::cout << "\n\n===========================================\n";
  std::cout << "Sampling : " << rp.N_shift / rp.N_shift_plaquette << " <P> samples, " << rp.N_shift / rp.N_shift_topo
            << " Q samples\n";
  std::cout << "===========================================\n";
  {  // the thermalisation's events are not counted (gauge_ecmc_ncb.cpp:122-130)
    R.flush();
    uint64_t c[3];
    CHECK(qcb_ecmc_counters(R.ecmc, c, 1), "ECMC counters");
  }
  for (int i = 0; i < rp.N_shift; i++) {
    std::cout << "\n\n=============" << "Shift " << i << "=============\n";
    R.shift_and_sample();
    if (i % rp.N_shift_plaquette == 0) {
      double p = R.plaquette();
      std::cout << "====== Plaquette ======\n";
      std::cout << "Sample " << i / rp.N_shift_plaquette << ", <P> = " << p << "\n";
      plaquette.push_back(p);
      R.count_events();
    }
    if (rp.topo && (i % rp.N_shift_topo == 0)) {
      std::cout << "====== Topology ======\n";
      std::vector<double> cur = R.topo();
      if (!cur.empty())
        std::cout << "Sample " << i / rp.N_shift_topo << ", final Q = " << cur[cur.size() - 2] << "\n";
      tQE_tot.insert(tQE_tot.end(), cur.begin(), cur.end());
    }
    if (i > 0 && i % rp.save_each_shifts == 0) {
      std::cout << "\n\n==========================================\n";
      drv::save_plaquette(plaquette, R.rd);
      if (rp.topo) drv::save_topo(tQE_tot, R.rd);
      append_params_line(R.rd, "Saved shift " + std::to_string(i) + "\n");
      R.save_event_nb();
      R.save_conf();
      R.save_state();
      std::cout << "==========================================\n";
      plaquette.clear();
      tQE_tot.clear();
    }
  }
  std::cout << "\n\n==========================================\n";
  drv::save_plaquette(plaquette, R.rd);
  if (rp.topo) drv::save_topo(tQE_tot, R.rd);
  append_params_line(R.rd, "Saved shift " + std::to_string(rp.N_shift) + "\n");
  append_params_line(R.rd, "Saved final state !\n");
  R.save_event_nb();
  R.save_conf();
  R.save_state();
  std::cout << "==========================================\n";
  R.flush();
  CHECK(qcb_ctx_sync(R.ctx), "sync");
  qcb_ecmc_destroy(R.ecmc);
  qcb_lattice_destroy(R.lat);
  qcb_ctx_destroy(R.ctx);
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc < 2) {
    std::cerr << "Usage: " << argv[0] << " <input_file.txt>" << std::endl;
    return 1;
  }
  Run R;
  qcb_ecmc_run_params_default(&R.rp);
  if (qcb_ecmc_run_params_load(argv[1], &R.rp) != QCB_OK) {
    std::cerr << "Error reading input : " << qcb_last_error() << std::endl;
    return 1;
  }
  if (R.rp.N_shift_plaquette <= 0 || R.rp.N_shift_topo <= 0 || R.rp.save_each_shifts <= 0) {
    std::cerr << "Error reading input : N_shift_plaquette, N_shift_topo and save_each_shifts must be positive"
              << std::endl;
    return 1;
  }
  if (R.rp.L_core < 3) {
    std::cerr << "Error reading input : L_core must be at least 3 for the event chains" << std::endl;
    return 1;
  }
  R.rd = drv::RunDir{R.rp.run_dir, R.rp.run_name};
  auto ex = drv::extra_keys(argv[1]);
  int precision = QCB_FP64, storage = QCB_R18, device = 0;
  if (ex.count("precision")) precision = (ex["precision"] == "fp32") ? QCB_FP32 : QCB_FP64;
  if (ex.count("storage")) storage = (ex["storage"] == "12") ? QCB_R12 : QCB_R18;
  if (ex.count("device")) device = atoi(ex["device"].c_str());

  fs::path config_file = R.rd.path() / R.rd.name;
  bool existing = fs::exists(config_file) && fs::exists(R.seed_path(0));
  if (existing) std::cout << "All ranks found existing configuration. Resuming...\n";

  auto t0 = std::chrono::steady_clock::now();
  generate_ecmc_cb(R, existing, precision, storage, device);
  double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "==========================================" << std::endl;
  std::cout << "Elapsed time : " << (long)total << "s\n";
  std::cout << "==========================================" << std::endl;
  std::cout << "Elapsed time (exact) : " << std::fixed << std::setprecision(4) << total << "s\n";
  return 0;
}
