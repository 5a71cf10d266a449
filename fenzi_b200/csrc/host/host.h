// Host-side data model of a loaded system (readers -> topology -> device upload).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../../include/fenzi_b200.h"

namespace fz {

// AKMA unit constants, src/defs.in.h:156-158
constexpr double kCC = 332.0716;   // Coulomb constant (kcal A / mol e^2)
constexpr double kRC = 0.001987;   // Boltzmann constant (kcal/mol/K)
constexpr double kTU = 20.4548;    // AKMA time units per ps
constexpr double kPU = 1.4586e-5;  // atm per (kcal/mol/A^3) conversion used by the reference (src/defs.in.h:105)

struct Cluster {  // SHAKE cluster: <= 4 atoms, <= 3 constraints (src/globals.h:225-228)
  int na = 0, nc = 0;
  int atom[4] = {-1, -1, -1, -1};
  int ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
  double d[3] = {0, 0, 0};
};

struct Topology {
  int n = 0;
  std::vector<double> pos;  // 3n, as read
  std::vector<double> q, mass;
  std::vector<int> type;    // index into type_names
  std::vector<std::string> type_names, atom_names, seg_names, res_names;
  std::vector<int> resid;
  // LJ tables (nt x nt), 4*eps and sigma^2; 1-4 variants
  std::vector<double> eps4, sig2, eps4_14, sig2_14;
  // bonded terms (0-based atoms)
  std::vector<int> bond;  std::vector<double> bond_k, bond_r0;
  std::vector<int> angle; std::vector<double> angle_k, angle_t0;
  std::vector<int> ub;    std::vector<double> ub_k, ub_r0;
  std::vector<int> dihe;  std::vector<double> dihe_k, dihe_d; std::vector<int> dihe_n;
  std::vector<int> impr;  std::vector<double> impr_k, impr_p0;
  // raw PSF lists (before parameter expansion)
  std::vector<int> psf_bond, psf_angle, psf_dihe, psf_impr;
  // constraints and exclusions
  std::vector<int> cons;  std::vector<double> cons_d;
  std::vector<Cluster> clusters;
  std::vector<int> excl_pairs;  // 1-2 and 1-3 (Ewald correction), i<j pairs, flattened
  std::vector<int> p14_pairs;   // 1-4 pairs not also 1-2/1-3
  std::vector<int> excl_off, excl_idx;  // per-atom sorted full exclusion list (1-2,1-3,1-4)
  double self_energy = 0;  // -CC beta/sqrt(pi) sum q^2
};

// error reporting (thread local)
void set_error(const std::string& msg);
fz_status fail(fz_status code, const std::string& msg);

// readers (readers.cpp)
fz_status read_coordinates(const std::string& path, Topology& t);
fz_status read_psf(const std::string& psf, const std::string& rtf, const fz_config& cfg, Topology& t);
fz_status read_prm(const std::string& path, Topology& t);
// topology.cpp
fz_status build_constraints(const fz_config& cfg, Topology& t);
fz_status build_exclusions(Topology& t, double beta);

std::string join_dir(const std::string& base_file, const std::string& rel);
int cicompare(const std::string& a, const std::string& b);

}  // namespace fz

namespace fz {
struct Engine;
void destroy_engine(Engine* e);
}  // namespace fz

// the opaque handle of the C ABI
struct fz_system {
  fz_config cfg;
  fz::Topology top;
  fz::Engine* eng = nullptr;
};
