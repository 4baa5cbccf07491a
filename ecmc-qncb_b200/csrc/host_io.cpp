// host_io.cpp — LIME container codec, ILDG XML, and the input-file parser.
//
// The reference links c-lime (fetched unpinned from GitHub, CMakeLists.txt:16-21) for the
// container and writes the data with MPI-IO (src/io/ildg.cpp:34-136).  This file writes the
// LIME record headers itself, from the published LIME layout, so the library has no
// external dependency.
#include "host_io.h"

#include <string.h>

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

#include "../../include/qcb.h"

namespace qcb {

static void put_be(unsigned char* p, uint64_t v, int n) {
  for (int k = n - 1; k >= 0; --k) {
    p[k] = (unsigned char)(v & 0xff);
    v >>= 8;
  }
}
static uint64_t get_be(const unsigned char* p, int n) {
  uint64_t v = 0;
  for (int k = 0; k < n; ++k) v = (v << 8) | p[k];
  return v;
}

bool lime_write_header(FILE* fp, bool mb, bool me, const char* type, uint64_t nbytes) {
  unsigned char h[LIME_HDR];
  memset(h, 0, sizeof h);
  put_be(h + 0, LIME_MAGIC, 4);
  put_be(h + 4, 1, 2);
  uint16_t flags = (uint16_t)((mb ? 0x8000u : 0u) | (me ? 0x4000u : 0u));
  put_be(h + 6, flags, 2);
  put_be(h + 8, nbytes, 8);
  strncpy(reinterpret_cast<char*>(h + 16), type, 127);
  return fwrite(h, 1, LIME_HDR, fp) == LIME_HDR;
}

bool lime_write_padding(FILE* fp, uint64_t nbytes) {
  static const unsigned char zeros[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const size_t pad = (size_t)((8 - (nbytes % 8)) % 8);
  return pad == 0 || fwrite(zeros, 1, pad, fp) == pad;
}

int lime_find(FILE* fp, const char* type, uint64_t* offset, uint64_t* nbytes, std::string* err) {
  if (fseeko(fp, 0, SEEK_SET) != 0) {
    *err = "seek failed";
    return QCB_ERR_IO;
  }
  for (;;) {
    unsigned char h[LIME_HDR];
    const size_t got = fread(h, 1, LIME_HDR, fp);
    if (got == 0) {
      *err = std::string("record '") + type + "' not found";
      return QCB_ERR_FORMAT;
    }
    if (got != LIME_HDR) {
      *err = "truncated LIME record header";
      return QCB_ERR_FORMAT;
    }
    if (get_be(h, 4) != LIME_MAGIC) {
      *err = "bad LIME magic number";
      return QCB_ERR_FORMAT;
    }
    const uint64_t len = get_be(h + 8, 8);
    char t[129];
    memcpy(t, h + 16, 128);
    t[128] = 0;
    const off_t here = ftello(fp);
    if (strcmp(t, type) == 0) {
      *offset = (uint64_t)here;
      *nbytes = len;
      return QCB_OK;
    }
    const uint64_t skip = len + (8 - len % 8) % 8;
    if (fseeko(fp, (off_t)skip, SEEK_CUR) != 0) {
      *err = "truncated LIME record";
      return QCB_ERR_FORMAT;
    }
  }
}

std::string ildg_xml(const int dims[4]) {
  char buf[512];
  snprintf(buf, sizeof buf,
           "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n"
           "<ildgFormat><version>1.0</version><field>su3gauge</field>"
           "<precision>64</precision><lx>%d</lx><ly>%d</ly><lz>%d</lz><lt>%d</lt>"
           "</ildgFormat>",
           dims[0], dims[1], dims[2], dims[3]);
  return std::string(buf);
}

}  // namespace qcb

// ---- input file ----------------------------------------------------------------------
// Semantics of io::load_params(const std::string&, RunParamsHbCB&) (src/io/io.cpp:353-399):
// lines that are empty or start with '#' are skipped; a line is split at its first '=';
// key and value are trimmed of spaces and tabs only (io::trim, io.cpp:290-295); a line with
// no '=' or an empty value is ignored; later keys override earlier ones.  Integers and
// doubles are parsed with std::stoi / std::stod (leading whitespace skipped, trailing text
// ignored, failure is an error).  cold_start and topo are true only for the exact string
// "true".  N_samples is forced to 1 (io.cpp:381).  N_switch_eo is accepted and ignored,
// as in the reference, which never parses it for the heatbath.

namespace qcb {

static std::string trim_st(const std::string& s) {
  size_t first = s.find_first_not_of(" \t");
  if (first == std::string::npos) return "";
  size_t last = s.find_last_not_of(" \t");
  return s.substr(first, last - first + 1);
}

// key -> value of an input file, with the line rules above.
static int read_config(const char* path, std::map<std::string, std::string>* cfg, std::string* err) {
  std::ifstream file(path);
  if (!file.is_open()) {
    *err = std::string("Can't open file ") + path;
    return QCB_ERR_IO;
  }
  std::string line;
  while (std::getline(file, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string key, value;
    if (std::getline(is, key, '=') && std::getline(is, value)) (*cfg)[trim_st(key)] = trim_st(value);
  }
  return QCB_OK;
}

int params_load(const char* path, qcb_hb_params* p, std::string* err) {
  std::map<std::string, std::string> cfg;
  int r = read_config(path, &cfg, err);
  if (r != QCB_OK) return r;
  try {
    auto geti = [&](const char* k, int& dst) {
      auto it = cfg.find(k);
      if (it != cfg.end()) dst = std::stoi(it->second);
    };
    auto getb = [&](const char* k, int& dst) {
      auto it = cfg.find(k);
      if (it != cfg.end()) dst = (it->second == "true") ? 1 : 0;
    };
    auto gets = [&](const char* k, char* dst, size_t cap) {
      auto it = cfg.find(k);
      if (it != cfg.end()) {
        strncpy(dst, it->second.c_str(), cap - 1);
        dst[cap - 1] = 0;
      }
    };
    geti("L_core", p->L_core);
    geti("n_core_dims", p->n_core_dims);
    getb("cold_start", p->cold_start);
    geti("seed", p->seed);
    geti("N_shift", p->N_shift);
    {
      auto it = cfg.find("beta");
      if (it != cfg.end()) p->beta = std::stod(it->second);
    }
    p->N_samples = 1;
    geti("N_sweeps", p->N_sweeps);
    geti("N_hits", p->N_hits);
    geti("N_shift_plaquette", p->N_shift_plaquette);
    geti("N_shift_therm", p->N_therm);
    getb("topo", p->topo);
    geti("N_shift_topo", p->N_shift_topo);
    geti("N_steps_gf", p->N_steps_gf);
    geti("N_rk_steps", p->N_rk_steps);
    gets("run_name", p->run_name, sizeof p->run_name);
    gets("run_dir", p->run_dir, sizeof p->run_dir);
    geti("save_each_shifts", p->save_each_shifts);
  } catch (const std::exception& e) {
    *err = std::string("Error reading input : ") + e.what();
    return QCB_ERR_FORMAT;
  }
  return QCB_OK;
}

// io::load_params(const std::string&, RunParamsECB&) (src/io/io.cpp:298-341): the same line
// rules; ECMC keys are param_theta_sample, param_theta_refresh_site, param_theta_refresh_R,
// poisson ("true" only), epsilon_set.
int ecmc_params_load(const char* path, qcb_ecmc_run_params* p, std::string* err) {
  std::map<std::string, std::string> cfg;
  int r = read_config(path, &cfg, err);
  if (r != QCB_OK) return r;
  try {
    auto geti = [&](const char* k, int& dst) {
      auto it = cfg.find(k);
      if (it != cfg.end()) dst = std::stoi(it->second);
    };
    auto getd = [&](const char* k, double& dst) {
      auto it = cfg.find(k);
      if (it != cfg.end()) dst = std::stod(it->second);
    };
    auto getb = [&](const char* k, int& dst) {
      auto it = cfg.find(k);
      if (it != cfg.end()) dst = (it->second == "true") ? 1 : 0;
    };
    auto gets = [&](const char* k, char* dst, size_t cap) {
      auto it = cfg.find(k);
      if (it != cfg.end()) {
        strncpy(dst, it->second.c_str(), cap - 1);
        dst[cap - 1] = 0;
      }
    };
    geti("L_core", p->L_core);
    geti("n_core_dims", p->n_core_dims);
    getb("cold_start", p->cold_start);
    geti("seed", p->seed);
    geti("N_shift", p->N_shift);
    getd("beta", p->ecmc.beta);
    getd("param_theta_sample", p->ecmc.theta_sample);
    getd("param_theta_refresh_site", p->ecmc.theta_refresh_site);
    getd("param_theta_refresh_R", p->ecmc.theta_refresh_R);
    getb("poisson", p->ecmc.poisson);
    getd("epsilon_set", p->ecmc.epsilon_set);
    geti("N_shift_plaquette", p->N_shift_plaquette);
    geti("N_shift_therm", p->N_therm);
    getb("topo", p->topo);
    geti("N_shift_topo", p->N_shift_topo);
    geti("N_steps_gf", p->N_steps_gf);
    geti("N_rk_steps", p->N_rk_steps);
    gets("run_name", p->run_name, sizeof p->run_name);
    gets("run_dir", p->run_dir, sizeof p->run_dir);
    geti("save_each_shifts", p->save_each_shifts);
    p->ecmc.l_core = p->L_core;
  } catch (const std::exception& e) {
    *err = std::string("Error reading input : ") + e.what();
    return QCB_ERR_FORMAT;
  }
  return QCB_OK;
}

}  // namespace qcb

