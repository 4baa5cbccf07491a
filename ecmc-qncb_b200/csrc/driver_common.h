// driver_common.h — host helpers shared by the drop-in drivers (gauge_hb_ncb, gauge_ecmc_ncb):
// error exit, the extra-key reader, and the reference's plaquette / topology / parameter-log
// outputs under run_dir/run_name/ (src/io/io.cpp:20-105, 233-287).
#pragma once
#include <stdlib.h>

#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "qcb.h"

namespace drv {

namespace fs = std::filesystem;

[[noreturn]] inline void die(const std::string& what) {
  std::cerr << "Error: " << what << ": " << qcb_last_error() << std::endl;
  exit(1);
}
#define CHECK(call, what)              \
  do {                                 \
    if ((call) != QCB_OK) drv::die(what); \
  } while (0)

inline std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t");
  return s.substr(a, b - a + 1);
}

// Extra keys that the reference does not know; parsed with the same line rules.
inline std::map<std::string, std::string> extra_keys(const char* path) {
  std::map<std::string, std::string> m;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string k, v;
    if (std::getline(is, k, '=') && std::getline(is, v)) m[trim(k)] = trim(v);
  }
  return m;
}

inline std::string fmt(double v, int p) {
  std::ostringstream ss;
  ss << std::fixed << std::setprecision(p) << v;
  return ss.str();
}

inline void ensure_dir(const fs::path& d) {
  std::error_code ec;
  if (!fs::exists(d)) fs::create_directories(d, ec);
  if (ec) std::cerr << "Couldn't create folder data : " << ec.message() << std::endl;
}

// run_dir/run_name, the folder of every output of a run.
struct RunDir {
  std::string dir, name;
  fs::path path() const { return fs::path(dir) / name; }
  fs::path file(const std::string& suffix) const { return path() / (name + suffix); }
};

// io::save_plaquette (io.cpp:20-47): appended, fixed, 10 decimals.
inline void save_plaquette(const std::vector<double>& data, const RunDir& rd) {
  ensure_dir(rd.path());
  fs::path p = rd.file("_plaquette.txt");
  std::ofstream f(p, std::ios::out | std::ios::app);
  if (!f.is_open()) {
    std::cout << "Could not open file " << p << "\n";
    return;
  }
  f << std::fixed << std::setprecision(10);
  for (double x : data) f << x << "\n";
  std::cout << "Plaquette written in " << p << "\n";
}

// io::save_topo (io.cpp:78-105): "t Q E" per line, appended, fixed, 10 decimals.
inline void save_topo(const std::vector<double>& tQE, const RunDir& rd) {
  ensure_dir(rd.path());
  fs::path p = rd.file("_topo.txt");
  std::ofstream f(p, std::ios::out | std::ios::app);
  if (!f.is_open()) {
    std::cout << "Could not open file " << p << "\n";
    return;
  }
  f << std::fixed << std::setprecision(10);
  for (size_t i = 0; i + 2 < tQE.size(); i += 3) f << tQE[i] << " " << tQE[i + 1] << " " << tQE[i + 2] << "\n";
  std::cout << "Topology written in " << p << "\n";
}

inline void append_params_line(const RunDir& rd, const std::string& line) {
  ensure_dir(rd.path());
  std::ofstream f(rd.file("_params.txt"), std::ios::out | std::ios::app);
  if (f.is_open()) f << line;
}

}  // namespace drv
