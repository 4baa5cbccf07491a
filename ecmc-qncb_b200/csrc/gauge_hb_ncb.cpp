// gauge_hb_ncb — drop-in replacement of the reference's heatbath driver
// (src/bin/gauge_hb_ncb.cpp:18-238) on one B200 through the C ABI (include/qcb.h).
//
//   gauge_hb_ncb <input_file.txt>
//
// Same input keys (src/io/io.cpp:353-399), same outputs under run_dir/run_name/:
//   run_name                       ILDG/LIME configuration (src/io/ildg.cpp:34-136)
//   run_name_plaquette.txt         one mean plaquette per line, fixed, 10 decimals (io.cpp:20-47)
//   run_name_topo.txt              "t Q E" per line, fixed, 10 decimals (io.cpp:78-105)
//   run_name_params.txt            parameter log + "Saved shift N" / "Saved final state !"
//                                  (io.cpp:233-287, 725-772)
//   run_name_seed/run_name_seed0.txt  generator state for resumption (io.cpp:108-138)
//
// Differences, by design: the global lattice is (L_core * n_core_dims)^4 on one GPU with
// periodic indexing, updated by checkerboard sweeps (every link of a sweep is updated; no
// frozen links, so no random translation is needed); the generator is Philox keyed by
// `seed` with a sweep counter, and the seed file stores that pair.  Optional extra keys:
// precision = fp64 | fp32 (default fp64), storage = 18 | 12 (default 18), device = N,
// schedule = checkerboard | reference (default checkerboard).
//
// schedule = reference keeps the reference's update schedule on the one device: before each
// shift's sweeps it draws the random shift (x, y, z, t), each uniform in [0, L_core), from
// std::mt19937_64 (src/mpi/Shift.cpp:163-186) and prints it, and the sweeps leave the links
// frozen by the L_core block faces of the shifted field unchanged
// (src/geometry/GeometryCB.cpp:33-56).  The field is not moved each shift: the cumulative
// shift is tracked and applied once (qcb_translate) before a configuration is written, so
// the saved file is in the reference's frame.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "driver_common.h"
#include "qcb.h"

namespace fs = std::filesystem;
using drv::ensure_dir;
using drv::fmt;

namespace {

drv::RunDir run_dir(const qcb_hb_params& rp) { return drv::RunDir{rp.run_dir, rp.run_name}; }
fs::path run_path(const qcb_hb_params& rp) { return run_dir(rp).path(); }
void save_plaquette(const std::vector<double>& data, const qcb_hb_params& rp) { drv::save_plaquette(data, run_dir(rp)); }
void save_topo(const std::vector<double>& tQE, const qcb_hb_params& rp) { drv::save_topo(tQE, run_dir(rp)); }
void append_params_line(const qcb_hb_params& rp, const std::string& line) { drv::append_params_line(run_dir(rp), line); }

void save_params(const qcb_hb_params& rp) {
  std::ostringstream f;
  f << std::boolalpha;
  f << "\n#########################################################\n\n";
  f << "# Lattice params\n";
  f << "L_core=" << rp.L_core << "\n";
  f << "n_core_dims=" << rp.n_core_dims << "\n";
  f << "cold_start=" << (rp.cold_start != 0) << "\n\n";
  f << "# Run params\n";
  f << "seed=" << rp.seed << "\n";
  f << "N_shift_therm = " << rp.N_therm << "\n";
  f << "N_shift =" << rp.N_shift << "\n";
  f << "# Heatbath params\n";
  f << "beta = " << rp.beta << "\n";
  f << "N_sweeps = " << rp.N_sweeps << "\n";
  f << "N_hits = " << rp.N_hits << "\n\n";
  f << "# Plaquette params\n";
  f << "N_shift_plaquette = " << rp.N_shift_plaquette << "\n\n";
  f << "# Topo params\n";
  f << "topo = " << (rp.topo != 0) << "\n";
  f << "N_shift_topo = " << rp.N_shift_topo << "\n";
  f << "N_steps_gf = " << rp.N_steps_gf << "\n";
  f << "N_rk_steps = " << rp.N_rk_steps << "\n\n";
  f << "#Save params\n";
  f << "save_each_shifts = " << rp.save_each_shifts << "\n\n";
  append_params_line(rp, f.str());
  std::cout << "Parameters saved in " << (run_path(rp) / (std::string(rp.run_name) + "_params.txt")) << "\n";
}

fs::path seed_path(const qcb_hb_params& rp) {
  return run_path(rp) / (std::string(rp.run_name) + "_seed") / (std::string(rp.run_name) + "_seed0.txt");
}

void save_seed(uint64_t key, uint64_t sweep, const qcb_hb_params& rp) {
  fs::path p = seed_path(rp);
  ensure_dir(p.parent_path());
  std::ofstream f(p);
  if (!f.is_open()) {
    std::cout << "Could not open file " << p << "\n";
    return;
  }
  f << "qcb-philox4x32-10 " << key << " " << sweep << "\n";
  std::cout << "Seed saved in " << p << "\n";
}

// Reads our own state file; a file in another format (for example a std::mt19937_64 state
// written by the reference) is hashed (FNV-1a) into a fresh key so the run can continue.
void load_seed(const qcb_hb_params& rp, uint64_t* key, uint64_t* sweep) {
  std::ifstream f(seed_path(rp));
  if (!f.is_open()) {
    std::cerr << "Could not open " << seed_path(rp) << "\n";
    return;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string text = ss.str(), tag;
  std::istringstream is(text);
  uint64_t k = 0, s = 0;
  if ((is >> tag >> k >> s) && tag == "qcb-philox4x32-10") {
    *key = k;
    *sweep = s;
    return;
  }
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : text) h = (h ^ ch) * 1099511628211ull;
  *key = h;
  *sweep = 0;
}

void print_parameters(const qcb_hb_params& rp) {
  std::cout << "==========================================" << std::endl;
  std::cout << "Heatbath - checkerboard, one GPU" << std::endl;
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
  std::cout << "---Heatbath params---\n";
  std::cout << "Beta : " << rp.beta << "\n";
  std::cout << "Number of sweeps : " << rp.N_sweeps << "\n";
  std::cout << "Number of hits : " << rp.N_hits << "\n\n";
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
  qcb_hb_params rp;
  qcb_ctx* ctx = nullptr;
  qcb_lattice* lat = nullptr;
  uint64_t key = 0, sweep = 0;
  bool ref_schedule = false;
  int cum[4] = {0, 0, 0, 0};  // cumulative shift not yet applied to the stored links
  std::mt19937_64 shift_rng;

  // One shift of the run: N_samples * N_sweeps sweeps (heatbathcb::samples); with plaq, also
  // the mean plaquette after them (on the periodic schedule summed inside the last sweep).
  void heatbath(double* plaq = nullptr) {
    const int n = rp.N_samples * rp.N_sweeps;
    if (ref_schedule) {
      std::uniform_int_distribution<int> rand_l_shift(0, rp.L_core - 1);
      int s[4];
      for (int d = 0; d < 4; ++d) s[d] = rand_l_shift(shift_rng);
      std::cout << "Shift (" << s[0] << ", " << s[1] << ", " << s[2] << ", " << s[3] << ")\n";
      const int Lg = rp.L_core * rp.n_core_dims;
      for (int d = 0; d < 4; ++d) cum[d] = (cum[d] + s[d]) % Lg;
      CHECK(qcb_heatbath_frozen(lat, rp.beta, n, rp.N_hits, key, sweep, rp.L_core, cum), "heatbath");
      if (plaq) CHECK(qcb_plaquette(lat, plaq), "plaquette");
    } else if (plaq) {
      CHECK(qcb_heatbath_plaquette(lat, rp.beta, n, rp.N_hits, key, sweep, plaq), "heatbath");
    } else {
      CHECK(qcb_heatbath(lat, rp.beta, n, rp.N_hits, key, sweep), "heatbath");
    }
    sweep += (uint64_t)n;
  }
  std::vector<double> topo() {
    std::vector<double> tqe(3 * (size_t)rp.N_steps_gf);
    const double eps = 0.02;  // hard-coded in the reference driver (gauge_hb_ncb.cpp:57)
    CHECK(qcb_flow_measure(lat, eps, rp.N_steps_gf, rp.N_rk_steps, tqe.data()), "flow");
    for (int s = 0; s < rp.N_steps_gf; ++s) {
      const double t = tqe[3 * s], q = tqe[3 * s + 1], e = tqe[3 * s + 2];
      std::cout << "n = " << s << ", t = " << fmt(t, 2) << ", Q = " << fmt(q, 6) << ", t²E = " << fmt(t * t * e, 6)
                << "\n";
    }
    return tqe;
  }
  void save_conf() {
    if (cum[0] | cum[1] | cum[2] | cum[3]) {
      CHECK(qcb_translate(lat, cum), "translate");
      cum[0] = cum[1] = cum[2] = cum[3] = 0;
    }
    fs::path dir = run_path(rp);
    ensure_dir(dir);
    fs::path p = dir / rp.run_name;
    CHECK(qcb_save_ildg(lat, p.string().c_str()), "save ILDG");
    std::cout << "Configuration saved in " << p << "\n";
  }
};

void generate_hb_cb(Run& R, bool existing, int precision, int storage, int device, bool ref_schedule) {
  qcb_hb_params& rp = R.rp;
  const int L = rp.L_core * rp.n_core_dims;
  const int dims[4] = {L, L, L, L};
  CHECK(qcb_ctx_create(device, 0, &R.ctx), "context");
  CHECK(qcb_lattice_create(R.ctx, dims, precision, storage, &R.lat), "lattice");
  R.key = (uint64_t)(int64_t)rp.seed;  // rp.seed + rank, rank 0
  R.sweep = 0;
  if (!rp.cold_start) CHECK(qcb_hot_start(R.lat, R.key), "hot start");
  if (existing) {
    fs::path p = run_path(rp) / rp.run_name;
    CHECK(qcb_load_ildg(R.lat, p.string().c_str()), "read ILDG");
    load_seed(rp, &R.key, &R.sweep);
  }
  R.ref_schedule = ref_schedule;
  R.shift_rng.seed(R.key ^ R.sweep);
  save_params(rp);
  print_parameters(rp);

  std::vector<double> plaquette, tQE_tot;
  std::cout << "\n\n===========================================\n";
  std::cout << "Thermalisation : " << rp.N_therm << " shifts\n";
  std::cout << "===========================================\n";
  for (int i = 0; i < rp.N_therm; i++) {
    double p = 0;
    const bool meas = i % rp.N_shift_plaquette == 0;
    R.heatbath(meas ? &p : nullptr);
    if (meas) {
      std::cout << "====== Plaquette ======\n";
      std::cout << "(Therm) Sample " << i / rp.N_shift_plaquette << ", <P> = " << p << "\n";
    }
  }
  std::cout << "\n\n===========================================\n";
  std::cout << "Sampling : " << rp.N_shift / rp.N_shift_plaquette << " <P> samples, " << rp.N_shift / rp.N_shift_topo
            << " Q samples\n";
  std::cout << "===========================================\n";
  for (int i = 0; i < rp.N_shift; i++) {
    std::cout << "\n\n=============" << "Shift " << i << "=============\n";
    double p = 0;
    const bool meas = i % rp.N_shift_plaquette == 0;
    R.heatbath(meas ? &p : nullptr);
    if (meas) {
      std::cout << "====== Plaquette ======\n";
      std::cout << "Sample " << i / rp.N_shift_plaquette << ", <P> = " << p << "\n";
      plaquette.push_back(p);
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
      save_plaquette(plaquette, rp);
      if (rp.topo) save_topo(tQE_tot, rp);
      append_params_line(rp, "Saved shift " + std::to_string(i) + "\n");
      save_seed(R.key, R.sweep, rp);
      R.save_conf();
      std::cout << "==========================================\n";
      plaquette.clear();
      tQE_tot.clear();
    }
  }
  std::cout << "\n\n==========================================\n";
  save_plaquette(plaquette, rp);
  if (rp.topo) save_topo(tQE_tot, rp);
  append_params_line(rp, "Saved shift " + std::to_string(rp.N_shift) + "\n");
  append_params_line(rp, "Saved final state !\n");
  save_seed(R.key, R.sweep, rp);
  R.save_conf();
  std::cout << "==========================================\n";
  CHECK(qcb_ctx_sync(R.ctx), "sync");
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
  qcb_params_default(&R.rp);
  if (qcb_params_load(argv[1], &R.rp) != QCB_OK) {
    std::cerr << "Error reading input : " << qcb_last_error() << std::endl;
    return 1;
  }
  if (R.rp.N_shift_plaquette <= 0 || R.rp.N_shift_topo <= 0 || R.rp.save_each_shifts <= 0) {
    std::cerr << "Error reading input : N_shift_plaquette, N_shift_topo and save_each_shifts must be positive"
              << std::endl;
    return 1;
  }
  auto ex = drv::extra_keys(argv[1]);
  int precision = QCB_FP64, storage = QCB_R18, device = 0;
  if (ex.count("precision")) precision = (ex["precision"] == "fp32") ? QCB_FP32 : QCB_FP64;
  if (ex.count("storage")) storage = (ex["storage"] == "12") ? QCB_R12 : QCB_R18;
  if (ex.count("device")) device = atoi(ex["device"].c_str());
  bool ref_schedule = false;
  if (ex.count("schedule")) {
    if (ex["schedule"] == "reference")
      ref_schedule = true;
    else if (ex["schedule"] != "checkerboard") {
      std::cerr << "Error reading input : schedule must be checkerboard or reference" << std::endl;
      return 1;
    }
  }

  fs::path config_file = run_path(R.rp) / R.rp.run_name;
  bool existing = fs::exists(config_file) && fs::exists(seed_path(R.rp));
  if (existing) std::cout << "All ranks found existing configuration. Resuming...\n";

  auto t0 = std::chrono::steady_clock::now();
  generate_hb_cb(R, existing, precision, storage, device, ref_schedule);
  double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "==========================================" << std::endl;
  std::cout << "Elapsed time : " << (long)total << "s\n";
  std::cout << "==========================================" << std::endl;
  std::cout << "Elapsed time (exact) : " << std::fixed << std::setprecision(4) << total << "s\n";
  return 0;
}
