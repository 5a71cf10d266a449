// Constraint clusters (build_constraints, src/prmread.cu:1192-1439) and exclusion
// lists (GenExcl_minimal_new, src/prmread.cu:2928-3062).
#include <algorithm>
#include <cmath>
#include <set>

#include "host.h"

namespace fz {

// SHAKE constraints: every PSF bond with an atom of mass <= 1.5 amu
// (src/prmread.cu:1757-1761), grouped into connected clusters of <= 4 atoms and
// <= 3 constraints.  Constraint length = the bond's b0.
fz_status build_constraints(const fz_config& cfg, Topology& t) {
  t.cons.clear();
  t.cons_d.clear();
  t.clusters.clear();
  if (!cfg.shake) return FZ_OK;
  const int nb = (int)t.bond.size() / 2;
  for (int b = 0; b < nb; ++b) {
    const int i = t.bond[2 * b], j = t.bond[2 * b + 1];
    if (t.mass[i] <= 1.5 || t.mass[j] <= 1.5) {
      t.cons.push_back(i);
      t.cons.push_back(j);
      t.cons_d.push_back(t.bond_r0[b]);
    }
  }
  const int n = t.n;
  std::vector<int> parent(n);
  for (int i = 0; i < n; ++i) parent[i] = i;
  auto find = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  const int nc = (int)t.cons_d.size();
  for (int c = 0; c < nc; ++c) {
    const int a = find(t.cons[2 * c]), b = find(t.cons[2 * c + 1]);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
  std::vector<int> cid(n, -1);
  for (int c = 0; c < nc; ++c) {
    const int a = t.cons[2 * c], b = t.cons[2 * c + 1];
    const int r = find(a);
    if (cid[r] < 0) {
      cid[r] = (int)t.clusters.size();
      t.clusters.emplace_back();
    }
    Cluster& cl = t.clusters[cid[r]];
    auto local = [&](int g) {
      for (int k = 0; k < cl.na; ++k)
        if (cl.atom[k] == g) return k;
      if (cl.na >= 4) return -1;
      cl.atom[cl.na] = g;
      return cl.na++;
    };
    const int la = local(a), lb = local(b);
    if (la < 0 || lb < 0 || cl.nc >= 3)
      return fail(FZ_ERR_CAPACITY, "SHAKE cluster around atom " + std::to_string(a + 1) +
                                       " exceeds 4 atoms / 3 constraints");
    cl.ca[cl.nc] = la;
    cl.cb[cl.nc] = lb;
    cl.d[cl.nc] = t.cons_d[c];
    cl.nc++;
  }
  return FZ_OK;
}

// Exclusions: 1-2 (bonds) and 1-3 (angle ends) form the Ewald-correction list; 1-4
// (dihedral ends) are added to the full exclusion list and, unless already 1-2/1-3,
// get the special 1-4 interaction once per unique pair.  (The reference evaluates a
// 1-4 term per dihedral, so a pair shared by two dihedrals counts twice there.)
fz_status build_exclusions(Topology& t, double beta) {
  const int n = t.n;
  std::set<std::pair<int, int>> ew, ex, p14;
  auto key = [](int a, int b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); };
  for (size_t b = 0; b < t.psf_bond.size() / 2; ++b) {
    const int i = t.psf_bond[2 * b], j = t.psf_bond[2 * b + 1];
    if (i != j) ew.insert(key(i, j));
  }
  for (size_t a = 0; a < t.psf_angle.size() / 3; ++a) {
    const int i = t.psf_angle[3 * a], k = t.psf_angle[3 * a + 2];
    if (i != k) ew.insert(key(i, k));
  }
  ex = ew;
  for (size_t d = 0; d < t.psf_dihe.size() / 4; ++d) {
    const int i = t.psf_dihe[4 * d], l = t.psf_dihe[4 * d + 3];
    if (i == l) continue;
    auto k = key(i, l);
    ex.insert(k);
    if (!ew.count(k)) p14.insert(k);
  }
  t.excl_pairs.clear();
  for (auto& p : ew) {
    t.excl_pairs.push_back(p.first);
    t.excl_pairs.push_back(p.second);
  }
  t.p14_pairs.clear();
  for (auto& p : p14) {
    t.p14_pairs.push_back(p.first);
    t.p14_pairs.push_back(p.second);
  }
  std::vector<std::vector<int>> per(n);
  for (auto& p : ex) {
    per[p.first].push_back(p.second);
    per[p.second].push_back(p.first);
  }
  t.excl_off.assign(n + 1, 0);
  t.excl_idx.clear();
  for (int i = 0; i < n; ++i) {
    std::sort(per[i].begin(), per[i].end());
    t.excl_off[i + 1] = t.excl_off[i] + (int)per[i].size();
    t.excl_idx.insert(t.excl_idx.end(), per[i].begin(), per[i].end());
  }
  // Ewald self energy (src/prmread.cu:1621,1734)
  double s = 0;
  for (int i = 0; i < n; ++i) s += t.q[i] * t.q[i];
  t.self_energy = -kCC * beta / std::sqrt(M_PI) * s;
  return FZ_OK;
}

}  // namespace fz
