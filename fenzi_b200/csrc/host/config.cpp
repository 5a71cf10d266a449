// .in run-file parser: the keyword set of ReadInput (src/prmread.cu:491-913),
// case-insensitive, '#' comments, defaults from src/globals.cu:28-593.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "host.h"

namespace fz {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
fz_status fail(fz_status code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cicompare(const std::string& a, const std::string& b) {
  if (a.size() != b.size()) return 1;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return 1;
  return 0;
}

std::string join_dir(const std::string& base_file, const std::string& rel) {
  if (rel.empty() || rel[0] == '/') return rel;
  const size_t p = base_file.find_last_of('/');
  if (p == std::string::npos) return rel;
  return base_file.substr(0, p + 1) + rel;
}

static void copy_str(char* dst, const std::string& s, size_t cap = 512) {
  std::snprintf(dst, cap, "%s", s.c_str());
}

}  // namespace fz

using namespace fz;

extern "C" fz_status fz_last_error(char* buf, size_t len) {
  if (!buf || !len) return FZ_ERR_ARG;
  std::snprintf(buf, len, "%s", g_err.c_str());
  return FZ_OK;
}

extern "C" const char* fz_version(void) { return "fenzi_b200 1.0 (sm_100a)"; }

extern "C" fz_status fz_read_input(const char* in_path, fz_config* c) {
  if (!in_path || !c) return fail(FZ_ERR_ARG, "fz_read_input: null argument");
  std::ifstream f(in_path);
  if (!f) return fail(FZ_ERR_IO, std::string("input file not found: ") + in_path);
  std::memset(c, 0, sizeof(*c));
  // defaults, src/globals.cu
  c->temperature = 298.0;
  c->timestep_ps = 0.001;
  c->dyna_steps = 10000;
  c->output_every = 100;
  c->checkpoint_every = 100000;
  c->traj_every = -1;
  c->gpublocksize = 128;
  c->kappa = 0.032;
  c->inbfrq = -1;
  c->cuton = 7.0;
  c->cutoff = 8.0;
  c->pairlistdist = 9.5;
  c->shake_tol = 1e-6;
  c->hfac = 1.0;
  c->conjgradfac = 1e-10;
  c->steepdesfac = 1e-4;
  c->conjgradrate = 0.1;
  c->steepdesrate = 0.01;
  c->pmass = 1.0e-5;  // the pmass keyword sets pmass_cubic (src/prmread.cu:663-666), PMASS_CUBIC src/defs.in.h:104
  c->pref = 1.0;      // PREF (atm)
  c->printtostdout = 1;
  c->seed = 0;
  std::string line;
  const std::string base(in_path);
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::string key;
    if (!(ss >> key)) continue;
    if (key[0] == '#') continue;
    auto num = [&]() {
      std::string v;
      ss >> v;
      return std::atof(v.c_str());
    };
    auto str = [&]() {
      std::string v;
      ss >> v;
      return v;
    };
    if (!cicompare(key, "coordinates")) copy_str(c->coordinates, join_dir(base, str()));
    else if (!cicompare(key, "structure")) copy_str(c->structure, join_dir(base, str()));
    else if (!cicompare(key, "parameters")) copy_str(c->parameters, join_dir(base, str()));
    else if (!cicompare(key, "topology")) copy_str(c->topology, join_dir(base, str()));
    else if (!cicompare(key, "temperature")) c->temperature = num();
    else if (!cicompare(key, "thermostat")) c->thermostat = num();
    else if (!cicompare(key, "minimizesteps")) c->minimize_steps = (int)num();
    else if (!cicompare(key, "conjgradfac")) c->conjgradfac = num();
    else if (!cicompare(key, "steepdesfac")) c->steepdesfac = num();
    else if (!cicompare(key, "conjgradrate")) c->conjgradrate = num();
    else if (!cicompare(key, "steepdesrate")) c->steepdesrate = num();
    else if (!cicompare(key, "startstep")) c->start_step = (int)num();
    else if (!cicompare(key, "timestep")) c->timestep_ps = num();
    else if (!cicompare(key, "dynasteps")) c->dyna_steps = (int)num();
    else if (!cicompare(key, "kappa")) c->kappa = num();
    else if (!cicompare(key, "inbfrq")) c->inbfrq = (int)num();
    else if (!cicompare(key, "tempresettiming")) c->temp_reset_every = (int)num();
    else if (!cicompare(key, "outputtiming")) c->output_every = (int)num();
    else if (!cicompare(key, "checkpointtiming")) c->checkpoint_every = (int)num();
    else if (!cicompare(key, "cuton")) c->cuton = num();
    else if (!cicompare(key, "cutoff")) c->cutoff = num();
    else if (!cicompare(key, "pairlistdist")) c->pairlistdist = num();
    else if (!cicompare(key, "gpublocksize")) c->gpublocksize = (int)num();
    else if (!cicompare(key, "trajfrequencytiming")) c->traj_every = (int)num();
    else if (!cicompare(key, "cellbasisvector1")) { c->box[0] = num(); }
    else if (!cicompare(key, "cellbasisvector2")) { num(); c->box[1] = num(); }
    else if (!cicompare(key, "cellbasisvector3")) { num(); num(); c->box[2] = num(); }
    else if (!cicompare(key, "pmegridsizex")) c->pme_grid[0] = (int)num();
    else if (!cicompare(key, "pmegridsizey")) c->pme_grid[1] = (int)num();
    else if (!cicompare(key, "pmegridsizez")) c->pme_grid[2] = (int)num();
    else if (!cicompare(key, "pmass")) c->pmass = num();
    else if (!cicompare(key, "pref")) c->pref = num();
    else if (!cicompare(key, "consharm")) {
      c->consharm = 1;
      copy_str(c->consharm_seg[0], str(), sizeof c->consharm_seg[0]);
      copy_str(c->consharm_seg[1], str(), sizeof c->consharm_seg[1]);
    } else if (!cicompare(key, "consharmdist")) {
      for (int d = 0; d < 3; ++d) c->consharm_dist[d] = num();
    } else if (!cicompare(key, "consharmfc")) {
      c->consharm_fc = num();
    } else if (!cicompare(key, "consfix")) {
      const int k = (int)num();
      c->consfix_nseg = std::max(0, std::min(8, k));
      for (int j = 0; j < c->consfix_nseg; ++j) copy_str(c->consfix_seg[j], str(), sizeof c->consfix_seg[j]);
    } else if (!cicompare(key, "shake")) {
      const std::string v = str();
      if (!cicompare(v, "on")) c->shake = 1;
      else c->shake = 0;
      std::string t;
      if (ss >> t) c->shake_tol = std::atof(t.c_str());
    } else if (!cicompare(key, "hfac")) c->hfac = num();
    else if (!cicompare(key, "printlevel")) c->printlevel = (int)num();
    else if (!cicompare(key, "printtostdout")) c->printtostdout = (int)num();
    else if (!cicompare(key, "keepcheckpoints")) c->keepcheckpoints = (int)num();
    else if (!cicompare(key, "checkpointformat")) {
      const std::string v = str();
      const char ch = v.empty() ? 0 : (char)std::tolower((unsigned char)v[0]);
      c->checkpointformat = (ch == '1') ? 'a' : (ch == '2') ? 'b' : ch;
    } else if (!cicompare(key, "seed")) c->seed = (long long)num();
    else if (!cicompare(key, "outputname")) copy_str(c->outputname, str());
    else if (!cicompare(key, "outputtrajectory")) copy_str(c->outputtrajectory, str());
    else if (!cicompare(key, "restartfilename")) copy_str(c->restartfilename, str());
    else c->unknown_keywords++;
  }
  if (c->traj_every < 0) c->traj_every = c->output_every;
  if (!c->coordinates[0] || !c->structure[0] || !c->parameters[0])
    return fail(FZ_ERR_PARSE, "input file lacks coordinates/structure/parameters");
  if (c->box[0] <= 0 || c->box[1] <= 0 || c->box[2] <= 0)
    return fail(FZ_ERR_PARSE, "cellBasisVector1..3 must give a positive diagonal box");
  return FZ_OK;
}
