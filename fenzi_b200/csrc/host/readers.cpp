// CHARMM input readers: coordinates (src/prmread.cu:285-488), RTF MASS map and PSF
// (src/prmread.cu:1442-1955), PRM (src/prmread.cu:2181-2750, helpers :916-1190).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <tuple>

#include "host.h"

namespace fz {

static std::string ext_of(const std::string& p) {
  const size_t d = p.find_last_of('.');
  if (d == std::string::npos) return "";
  std::string e = p.substr(d + 1);
  for (auto& ch : e) ch = (char)std::tolower((unsigned char)ch);
  return e;
}

// ---------------------------------------------------------------- coordinates
static fz_status read_crd(const std::string& path, Topology& t) {
  std::ifstream f(path);
  if (!f) return fail(FZ_ERR_IO, "coordinate file not found: " + path);
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '*') continue;
    break;
  }
  const int n = std::atoi(line.c_str());
  if (n <= 0) return fail(FZ_ERR_PARSE, "bad atom count in " + path);
  t.n = n;
  t.pos.assign(3 * (size_t)n, 0.0);
  t.seg_names.assign(n, "");
  for (int i = 0; i < n; ++i) {
    if (!std::getline(f, line)) return fail(FZ_ERR_PARSE, "truncated coordinate file " + path);
    std::istringstream ss(line);
    int id;
    std::string resno, resname, aname, seg;
    double x, y, z;
    if (!(ss >> id >> resno >> resname >> aname >> x >> y >> z))
      return fail(FZ_ERR_PARSE, "bad CRD line " + std::to_string(i + 1) + " in " + path);
    ss >> seg;
    if (id < 1 || id > n) return fail(FZ_ERR_PARSE, "CRD atom id out of range in " + path);
    t.pos[3 * (id - 1)] = x;
    t.pos[3 * (id - 1) + 1] = y;
    t.pos[3 * (id - 1) + 2] = z;
    t.seg_names[id - 1] = seg;
  }
  return FZ_OK;
}

static fz_status read_pdb(const std::string& path, Topology& t) {
  std::ifstream f(path);
  if (!f) return fail(FZ_ERR_IO, "coordinate file not found: " + path);
  std::string line;
  t.pos.clear();
  while (std::getline(f, line)) {
    if (line.compare(0, 4, "ATOM") && line.compare(0, 6, "HETATM")) continue;
    if (line.size() < 54) return fail(FZ_ERR_PARSE, "short PDB ATOM record in " + path);
    t.pos.push_back(std::atof(line.substr(30, 8).c_str()));
    t.pos.push_back(std::atof(line.substr(38, 8).c_str()));
    t.pos.push_back(std::atof(line.substr(46, 8).c_str()));
  }
  t.n = (int)(t.pos.size() / 3);
  if (!t.n) return fail(FZ_ERR_PARSE, "no ATOM records in " + path);
  return FZ_OK;
}

static fz_status read_xyz(const std::string& path, Topology& t) {
  std::ifstream f(path);
  if (!f) return fail(FZ_ERR_IO, "coordinate file not found: " + path);
  std::string line;
  std::getline(f, line);
  const int n = std::atoi(line.c_str());
  if (n <= 0) return fail(FZ_ERR_PARSE, "bad atom count in " + path);
  std::getline(f, line);  // comment
  t.n = n;
  t.pos.assign(3 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    if (!std::getline(f, line)) return fail(FZ_ERR_PARSE, "truncated XYZ file " + path);
    std::istringstream ss(line);
    std::string name;
    if (!(ss >> name >> t.pos[3 * i] >> t.pos[3 * i + 1] >> t.pos[3 * i + 2]))
      return fail(FZ_ERR_PARSE, "bad XYZ line in " + path);
  }
  return FZ_OK;
}

fz_status read_coordinates(const std::string& path, Topology& t) {
  const std::string e = ext_of(path);
  if (e == "pdb") return read_pdb(path, t);
  if (e == "xyz") return read_xyz(path, t);
  return read_crd(path, t);  // the reference's default reader
}

// ---------------------------------------------------------------- RTF + PSF
static fz_status read_rtf_masses(const std::string& path, std::map<int, std::string>& ids) {
  std::ifstream f(path);
  if (!f) return FZ_ERR_IO;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::string k;
    if (!(ss >> k)) continue;
    if (!cicompare(k, "MASS")) {
      int id;
      std::string name;
      if (ss >> id >> name) ids[id] = name;
    }
  }
  return FZ_OK;
}

static bool is_int(const std::string& s) {
  if (s.empty()) return false;
  size_t i = (s[0] == '-' || s[0] == '+') ? 1 : 0;
  if (i >= s.size()) return false;
  for (; i < s.size(); ++i)
    if (!std::isdigit((unsigned char)s[i])) return false;
  return true;
}

static fz_status read_int_block(std::ifstream& f, int count, int per, std::vector<int>& out) {
  out.clear();
  out.reserve((size_t)count * per);
  std::string tok;
  while ((int)out.size() < count * per && (f >> tok)) {
    if (!is_int(tok)) return FZ_ERR_PARSE;
    out.push_back(std::atoi(tok.c_str()) - 1);
  }
  return (int)out.size() == count * per ? FZ_OK : FZ_ERR_PARSE;
}

fz_status read_psf(const std::string& psf, const std::string& rtf, const fz_config& cfg, Topology& t) {
  std::map<int, std::string> rtf_ids;
  const bool have_rtf = !rtf.empty() && read_rtf_masses(rtf, rtf_ids) == FZ_OK;
  std::ifstream f(psf);
  if (!f) return fail(FZ_ERR_IO, "structure file not found: " + psf);
  std::string line;
  bool got_atoms = false;
  std::map<std::string, int> tidx;
  while (std::getline(f, line)) {
    if (line.find("!NATOM") != std::string::npos) {
      const int n = std::atoi(line.c_str());
      if (n != t.n)
        return fail(FZ_ERR_PARSE, "Number of atoms in psf (" + std::to_string(n) +
                                      ") does not match number of atoms in coord file (" + std::to_string(t.n) + ")");
      t.q.assign(n, 0.0);
      t.mass.assign(n, 0.0);
      t.type.assign(n, 0);
      t.atom_names.assign(n, "");
      t.res_names.assign(n, "");
      t.resid.assign(n, 0);
      if ((int)t.seg_names.size() != n) t.seg_names.assign(n, "");
      for (int i = 0; i < n; ++i) {
        if (!std::getline(f, line)) return fail(FZ_ERR_PARSE, "truncated PSF atom section");
        std::istringstream ss(line);
        int id;
        std::string seg, resid, resname, aname, ty;
        double q, m;
        if (!(ss >> id >> seg >> resid >> resname >> aname >> ty >> q >> m))
          return fail(FZ_ERR_PARSE, "bad PSF atom line " + std::to_string(i + 1));
        std::string tname = ty;
        if (is_int(ty)) {
          if (!have_rtf) return fail(FZ_ERR_PARSE, "PSF uses numeric types but no RTF MASS table was read");
          auto it = rtf_ids.find(std::atoi(ty.c_str()));
          if (it == rtf_ids.end()) return fail(FZ_ERR_PARSE, "PSF type id " + ty + " not in RTF");
          tname = it->second;
        }
        auto tt = tidx.find(tname);
        int ti;
        if (tt == tidx.end()) {
          ti = (int)t.type_names.size();
          tidx[tname] = ti;
          t.type_names.push_back(tname);
        } else {
          ti = tt->second;
        }
        const int a = id - 1;
        if (a < 0 || a >= n) return fail(FZ_ERR_PARSE, "PSF atom id out of range");
        t.type[a] = ti;
        t.q[a] = q;
        // hydrogen mass repartitioning when SHAKE is off (src/prmread.cu:1580-1600)
        if (!cfg.shake && (aname == "H1" || aname == "H2" || aname == "HG1" || aname == "HB1" || aname == "HB2" ||
                           aname == "HB3"))
          m *= cfg.hfac;
        t.mass[a] = m;
        t.atom_names[a] = aname;
        t.res_names[a] = resname;
        t.resid[a] = std::atoi(resid.c_str());
        if (t.seg_names[a].empty()) t.seg_names[a] = seg;
      }
      got_atoms = true;
      continue;
    }
    if (!got_atoms) continue;
    struct {
      const char* tag;
      int per;
      std::vector<int>* dst;
    } secs[] = {{"!NBOND", 2, &t.psf_bond}, {"!NTHETA", 3, &t.psf_angle}, {"!NPHI", 4, &t.psf_dihe},
                {"!NIMPHI", 4, &t.psf_impr}};
    bool done = false;
    for (auto& s : secs) {
      if (line.find(s.tag) != std::string::npos) {
        const int cnt = std::atoi(line.c_str());
        if (read_int_block(f, cnt, s.per, *s.dst) != FZ_OK)
          return fail(FZ_ERR_PARSE, std::string("bad PSF section ") + s.tag);
        for (int v : *s.dst)
          if (v < 0 || v >= t.n) return fail(FZ_ERR_PARSE, std::string("atom index out of range in ") + s.tag);
        if (std::string(s.tag) == "!NIMPHI") done = true;
        break;
      }
    }
    if (done) break;
  }
  if (!got_atoms) return fail(FZ_ERR_PARSE, "no !NATOM section in " + psf);
  return FZ_OK;
}

// ---------------------------------------------------------------- PRM
namespace {
struct DihePrm {
  double k;
  int n;
  double d;
};
struct Prm {
  std::map<std::pair<int, int>, std::pair<double, double>> bond;
  std::map<std::tuple<int, int, int>, std::vector<double>> angle;  // k, t0(rad), kub, s0
  std::map<std::tuple<int, int, int, int>, std::vector<DihePrm>> dihe;
  std::map<std::pair<int, int>, std::vector<DihePrm>> dihe_wild;  // X t2 t3 X
  std::map<std::tuple<int, int, int, int>, std::pair<double, double>> impr;
  std::map<std::pair<int, int>, std::pair<double, double>> impr_wild;  // t1 X X t4
  std::vector<double> eps, rmh, eps14, rmh14;
  std::vector<char> have_nb;
  std::map<std::pair<int, int>, std::pair<double, double>> nbfix;  // eps, rmin
};

std::pair<int, int> k2(int a, int b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); }
std::tuple<int, int, int> k3(int a, int b, int c) {
  return a < c || (a == c) ? std::make_tuple(a, b, c) : std::make_tuple(c, b, a);
}
std::tuple<int, int, int, int> k4(int a, int b, int c, int d) {
  auto f = std::make_tuple(a, b, c, d), r = std::make_tuple(d, c, b, a);
  return f < r ? f : r;
}
void add_fold(std::vector<DihePrm>& v, DihePrm p) {
  for (auto& x : v)
    if (x.n == p.n) {
      x = p;  // same multiplicity overwrites (add_specific_dihedrals_set_type_to_prm)
      return;
    }
  v.push_back(p);
}
}  // namespace

fz_status read_prm(const std::string& path, Topology& t) {
  std::ifstream f(path);
  if (!f) return fail(FZ_ERR_IO, "parameter file not found: " + path);
  const int nt = (int)t.type_names.size();
  std::map<std::string, int> tid;
  for (int i = 0; i < nt; ++i) tid[t.type_names[i]] = i;
  auto T = [&](const std::string& s) {
    auto it = tid.find(s);
    return it == tid.end() ? -1 : it->second;
  };
  auto isX = [](const std::string& s) { return !cicompare(s, "X"); };
  Prm P;
  P.eps.assign(nt, 0);
  P.rmh.assign(nt, 0);
  P.eps14.assign(nt, 0);
  P.rmh14.assign(nt, 0);
  P.have_nb.assign(nt, 0);
  int sec = 0;
  std::string line;
  const double deg = M_PI / 180.0;
  while (std::getline(f, line)) {
    const size_t bang = line.find('!');
    const std::string body = bang == std::string::npos ? line : line.substr(0, bang);
    std::istringstream ss(body);
    std::vector<std::string> tok;
    std::string w;
    while (ss >> w) tok.push_back(w);
    if (tok.empty() || tok[0][0] == '*') continue;
    const std::string& h = tok[0];
    if (h == "BONDS") { sec = 1; continue; }
    if (h == "ANGLES" || h == "THETAS") { sec = 2; continue; }
    if (h == "DIHEDRALS" || h == "PHI") { sec = 3; continue; }
    if (h == "NONBONDED") { sec = 4; continue; }
    if (h == "NBFIX") { sec = 5; continue; }
    if (h == "CMAP") { sec = 6; continue; }
    if (h == "IMPROPER" || h == "IMPHI") { sec = 7; continue; }
    if (h == "HBOND") { sec = 8; continue; }
    if (h == "ATOMS") { sec = 9; continue; }
    if (h == "END") break;
    if (sec == 1 && tok.size() >= 4) {
      const int a = T(tok[0]), b = T(tok[1]);
      if (a < 0 || b < 0) continue;
      P.bond[k2(a, b)] = {std::atof(tok[2].c_str()), std::atof(tok[3].c_str())};
    } else if (sec == 2 && tok.size() >= 5) {
      const int a = T(tok[0]), b = T(tok[1]), c = T(tok[2]);
      if (a < 0 || b < 0 || c < 0) continue;
      std::vector<double> v = {std::atof(tok[3].c_str()), std::atof(tok[4].c_str()) * deg, 0.0, 0.0};
      if (tok.size() >= 7 && std::atof(tok[5].c_str()) != 0.0) {  // Urey-Bradley (src/prmread.cu:2354-2370)
        v[2] = std::atof(tok[5].c_str());
        v[3] = std::atof(tok[6].c_str());
      }
      P.angle[k3(a, b, c)] = v;
    } else if (sec == 3 && tok.size() >= 7) {
      DihePrm p{std::atof(tok[4].c_str()), std::atoi(tok[5].c_str()), std::atof(tok[6].c_str()) * deg};
      if (isX(tok[0]) && isX(tok[3])) {
        const int b = T(tok[1]), c = T(tok[2]);
        if (b < 0 || c < 0) continue;
        add_fold(P.dihe_wild[k2(b, c)], p);
        continue;
      }
      const int a = T(tok[0]), b = T(tok[1]), c = T(tok[2]), d = T(tok[3]);
      if (a < 0 || b < 0 || c < 0 || d < 0) continue;
      add_fold(P.dihe[k4(a, b, c, d)], p);
    } else if (sec == 4 && tok.size() >= 4) {
      const int a = T(tok[0]);
      if (a < 0) continue;  // header continuation lines (cutnb ...) and absent types
      const double ign = std::atof(tok[1].c_str());
      double e = std::fabs(std::atof(tok[2].c_str())), r = std::atof(tok[3].c_str());
      if (ign == 1.0) e = r = 0.0;  // "excluded" type (src/prmread.cu:2474-2477)
      P.eps[a] = e;
      P.rmh[a] = r;
      P.eps14[a] = e;
      P.rmh14[a] = r;
      if (tok.size() >= 7) {
        const double i14 = std::atof(tok[4].c_str());
        double e14 = std::fabs(std::atof(tok[5].c_str())), r14 = std::atof(tok[6].c_str());
        if (i14 == 1.0) e14 = r14 = 0.0;
        P.eps14[a] = e14;
        P.rmh14[a] = r14;
      }
      P.have_nb[a] = 1;
    } else if (sec == 5 && tok.size() >= 4) {
      const int a = T(tok[0]), b = T(tok[1]);
      if (a < 0 || b < 0) continue;
      P.nbfix[k2(a, b)] = {std::fabs(std::atof(tok[2].c_str())), std::atof(tok[3].c_str())};
    } else if (sec == 7 && tok.size() >= 7) {
      const double k = std::atof(tok[4].c_str()), p0 = std::atof(tok[6].c_str()) * deg;
      if (isX(tok[1]) && isX(tok[2])) {
        const int a = T(tok[0]), d = T(tok[3]);
        if (a < 0 || d < 0) continue;
        P.impr_wild[k2(a, d)] = {k, p0};
        continue;
      }
      const int a = T(tok[0]), b = T(tok[1]), c = T(tok[2]), d = T(tok[3]);
      if (a < 0 || b < 0 || c < 0 || d < 0) continue;
      P.impr[k4(a, b, c, d)] = {k, p0};
    }
  }
  for (int i = 0; i < nt; ++i)
    if (!P.have_nb[i]) return fail(FZ_ERR_PARSE, "no NONBONDED parameters for type " + t.type_names[i]);
  // LJ tables: 4*sqrt(eps_i eps_j), sigma = (rmin_i/2 + rmin_j/2)/2^(1/6); NBFIX overrides
  // (src/prmread.cu:2458-2570, 2724-2736)
  const double s6 = std::pow(2.0, 1.0 / 6.0);
  t.eps4.assign((size_t)nt * nt, 0);
  t.sig2.assign((size_t)nt * nt, 0);
  t.eps4_14.assign((size_t)nt * nt, 0);
  t.sig2_14.assign((size_t)nt * nt, 0);
  for (int i = 0; i < nt; ++i)
    for (int j = 0; j < nt; ++j) {
      const size_t ij = (size_t)i * nt + j;
      t.eps4[ij] = 4.0 * std::sqrt(P.eps[i] * P.eps[j]);
      const double sg = (P.rmh[i] + P.rmh[j]) / s6;
      t.sig2[ij] = sg * sg;
      t.eps4_14[ij] = 4.0 * std::sqrt(P.eps14[i] * P.eps14[j]);
      const double sg14 = (P.rmh14[i] + P.rmh14[j]) / s6;
      t.sig2_14[ij] = sg14 * sg14;
      auto it = P.nbfix.find(k2(i, j));
      if (it != P.nbfix.end()) {
        t.eps4[ij] = 4.0 * it->second.first;
        const double sf = it->second.second / s6;
        t.sig2[ij] = sf * sf;
      }
    }
  // expand PSF lists with parameters
  auto tn = [&](int a) { return t.type_names[t.type[a]]; };
  t.bond.clear(); t.bond_k.clear(); t.bond_r0.clear();
  for (size_t b = 0; b < t.psf_bond.size() / 2; ++b) {
    const int i = t.psf_bond[2 * b], j = t.psf_bond[2 * b + 1];
    auto it = P.bond.find(k2(t.type[i], t.type[j]));
    if (it == P.bond.end()) return fail(FZ_ERR_PARSE, "missing bond parameter " + tn(i) + " " + tn(j));
    t.bond.push_back(i);
    t.bond.push_back(j);
    t.bond_k.push_back(it->second.first);
    t.bond_r0.push_back(it->second.second);
  }
  t.angle.clear(); t.angle_k.clear(); t.angle_t0.clear(); t.ub.clear(); t.ub_k.clear(); t.ub_r0.clear();
  for (size_t a = 0; a < t.psf_angle.size() / 3; ++a) {
    const int i = t.psf_angle[3 * a], j = t.psf_angle[3 * a + 1], k = t.psf_angle[3 * a + 2];
    auto it = P.angle.find(k3(t.type[i], t.type[j], t.type[k]));
    if (it == P.angle.end()) return fail(FZ_ERR_PARSE, "missing angle parameter " + tn(i) + " " + tn(j) + " " + tn(k));
    t.angle.insert(t.angle.end(), {i, j, k});
    t.angle_k.push_back(it->second[0]);
    t.angle_t0.push_back(it->second[1]);
    if (it->second[2] != 0.0) {
      t.ub.insert(t.ub.end(), {i, k});
      t.ub_k.push_back(it->second[2]);
      t.ub_r0.push_back(it->second[3]);
    }
  }
  t.dihe.clear(); t.dihe_k.clear(); t.dihe_n.clear(); t.dihe_d.clear();
  for (size_t d = 0; d < t.psf_dihe.size() / 4; ++d) {
    const int* q = &t.psf_dihe[4 * d];
    const std::vector<DihePrm>* folds = nullptr;
    auto it = P.dihe.find(k4(t.type[q[0]], t.type[q[1]], t.type[q[2]], t.type[q[3]]));
    if (it != P.dihe.end()) folds = &it->second;
    else {
      auto iw = P.dihe_wild.find(k2(t.type[q[1]], t.type[q[2]]));
      if (iw != P.dihe_wild.end()) folds = &iw->second;
    }
    if (!folds)
      return fail(FZ_ERR_PARSE, "missing dihedral parameter " + tn(q[0]) + " " + tn(q[1]) + " " + tn(q[2]) + " " +
                                    tn(q[3]));
    for (const auto& p : *folds) {
      t.dihe.insert(t.dihe.end(), {q[0], q[1], q[2], q[3]});
      t.dihe_k.push_back(p.k);
      t.dihe_n.push_back(p.n);
      t.dihe_d.push_back(p.d);
    }
  }
  t.impr.clear(); t.impr_k.clear(); t.impr_p0.clear();
  for (size_t d = 0; d < t.psf_impr.size() / 4; ++d) {
    const int* q = &t.psf_impr[4 * d];
    auto it = P.impr.find(k4(t.type[q[0]], t.type[q[1]], t.type[q[2]], t.type[q[3]]));
    std::pair<double, double> pr;
    if (it != P.impr.end()) pr = it->second;
    else {
      auto iw = P.impr_wild.find(k2(t.type[q[0]], t.type[q[3]]));
      if (iw == P.impr_wild.end())
        return fail(FZ_ERR_PARSE, "missing improper parameter " + tn(q[0]) + " " + tn(q[1]) + " " + tn(q[2]) + " " +
                                      tn(q[3]));
      pr = iw->second;
    }
    t.impr.insert(t.impr.end(), {q[0], q[1], q[2], q[3]});
    t.impr_k.push_back(pr.first);
    t.impr_p0.push_back(pr.second);
  }
  return FZ_OK;
}

}  // namespace fz
