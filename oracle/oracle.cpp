// FP64 CPU oracle for the FEN ZI MD step.  TEST INFRASTRUCTURE ONLY: used by
// tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg, never by the
// product library.  See oracle.h for the reference file:line map.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <set>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

const double kPi = 3.14159265358979323846;

struct Cluster {
  int na = 0;             // atoms (<= 4)
  int atom[4] = {0, 0, 0, 0};
  int nc = 0;             // constraints (<= 3)
  int ca[3] = {0, 0, 0};  // local atom index of first atom
  int cb[3] = {0, 0, 0};  // local atom index of second atom
  double d[3] = {0, 0, 0};
};

struct Orc {
  orc_system s;
  std::vector<double> q, mass, eps4, sig2, eps4_14, sig2_14;
  std::vector<int> type;
  std::vector<int> bond, angle, ub, dihe, dihe_n, impr, cons;
  std::vector<double> bond_k, bond_r0, angle_k, angle_t0, ub_k, ub_r0, dihe_k, dihe_d, impr_k,
      impr_p0, cons_d;
  // exclusions: per atom sorted list of excluded partners (1-2, 1-3, 1-4)
  std::vector<int> excl_off, excl_idx;
  std::vector<std::pair<int, int>> ew_pairs;   // 1-2 and 1-3 (Ewald exclusion correction)
  std::vector<std::pair<int, int>> p14_pairs;  // 1-4 (not also 1-2/1-3)
  std::vector<Cluster> clusters;
  int nthreads = 0;
};

inline void minimg(double* d, const double* L) {
  for (int k = 0; k < 3; ++k) d[k] -= L[k] * std::nearbyint(d[k] / L[k]);
}

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

bool excluded(const Orc& o, int i, int j) {
  const int* b = o.excl_idx.data() + o.excl_off[i];
  const int* e = o.excl_idx.data() + o.excl_off[i + 1];
  return std::binary_search(b, e, j);
}

// ---------------------------------------------------------------- pair forms
// CHARMM switch, src/mem.cu:556-566: sw = (rc2-r2)^2 (rc2+2r2-3ron2)/(rc2-ron2)^3 for r > ron.
// Returns sw and dsw = -(dsw/dr)/r  (the reference's force expression at
// src/nonbonded_forces.cu:210-214 carries an extra Swcoeff2*invDist term, which is
// dimensionally inconsistent; the exact derivative is used here).
inline void switch_fn(double r2, double rc2, double ron2, double* sw, double* dsw) {
  if (r2 <= ron2) {
    *sw = 1.0;
    *dsw = 0.0;
    return;
  }
  const double c3 = 1.0 / ((rc2 - ron2) * (rc2 - ron2) * (rc2 - ron2));
  const double u = rc2 - r2;
  const double v = rc2 + 2.0 * r2 - 3.0 * ron2;
  *sw = u * u * v * c3;
  *dsw = 12.0 * u * (r2 - ron2) * c3;
}

// LJ (switched) + erfc Coulomb for one pair; returns F/r (force on i = fr * d, d = ri - rj)
inline double pair_lj_coul(double r2, double qq, double e4, double s2, double rc2, double ron2,
                           double beta, double* evdw, double* eelec) {
  const double r = std::sqrt(r2);
  const double ir2 = 1.0 / r2;
  const double br = beta * r;
  const double erfcv = std::erfc(br);
  const double ec = ORC_CC * qq * erfcv / r;
  const double fc = (ec + ORC_CC * qq * 2.0 / std::sqrt(kPi) * beta * std::exp(-br * br)) * ir2;
  const double s6 = s2 * s2 * s2 * ir2 * ir2 * ir2;
  const double a = e4 * s6, b = a * s6;
  const double elj = b - a;
  const double flj = (12.0 * b - 6.0 * a) * ir2;
  double sw, dsw;
  switch_fn(r2, rc2, ron2, &sw, &dsw);
  *evdw = elj * sw;
  *eelec = ec;
  return flj * sw + elj * dsw + fc;
}

// ---------------------------------------------------------------- FFT (FP64)
void fft_rec(const cplx* in, cplx* out, int n, int stride, int sign, cplx* tmp) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = 0;
  for (int f : {4, 2, 3, 5}) {
    if (n % f == 0) {
      p = f;
      break;
    }
  }
  if (!p) {
    for (p = 7; p * p <= n; p += 2)
      if (n % p == 0) break;
    if (n % p) p = n;
  }
  const int m = n / p;
  for (int r = 0; r < p; ++r) fft_rec(in + r * stride, out + r * m, m, stride * p, sign, tmp);
  // butterflies: X[k + s*m] = sum_r W_n^{(k+s m) r} Y_r[k]
  for (int k = 0; k < m; ++k) {
    for (int s2 = 0; s2 < p; ++s2) {
      cplx acc = 0;
      for (int r = 0; r < p; ++r) {
        const long long e = (long long)(k + s2 * m) * r % n;
        const double ang = sign * 2.0 * kPi * (double)e / (double)n;
        acc += out[r * m + k] * cplx(std::cos(ang), std::sin(ang));
      }
      tmp[k + s2 * m] = acc;
    }
  }
  for (int i = 0; i < n; ++i) out[i] = tmp[i];
}

void fft3d(cplx* d, int nx, int ny, int nz, int sign, int nth) {
  // x lines
#pragma omp parallel num_threads(nth)
  {
    std::vector<cplx> a(std::max(nx, std::max(ny, nz))), b(a.size()), t(a.size());
#pragma omp for schedule(static)
    for (int l = 0; l < ny * nz; ++l) {
      cplx* line = d + (size_t)l * nx;
      for (int i = 0; i < nx; ++i) a[i] = line[i];
      fft_rec(a.data(), b.data(), nx, 1, sign, t.data());
      for (int i = 0; i < nx; ++i) line[i] = b[i];
    }
#pragma omp for schedule(static)
    for (int l = 0; l < nx * nz; ++l) {
      const int x = l % nx, z = l / nx;
      cplx* base = d + (size_t)z * nx * ny + x;
      for (int i = 0; i < ny; ++i) a[i] = base[(size_t)i * nx];
      fft_rec(a.data(), b.data(), ny, 1, sign, t.data());
      for (int i = 0; i < ny; ++i) base[(size_t)i * nx] = b[i];
    }
#pragma omp for schedule(static)
    for (int l = 0; l < nx * ny; ++l) {
      cplx* base = d + l;
      for (int i = 0; i < nz; ++i) a[i] = base[(size_t)i * nx * ny];
      fft_rec(a.data(), b.data(), nz, 1, sign, t.data());
      for (int i = 0; i < nz; ++i) base[(size_t)i * nx * ny] = b[i];
    }
  }
}

// cubic B-spline M4 at t, t+1, t+2, t+3 and derivatives (t in [0,1))
inline void bspline4(double t, double* w, double* dw) {
  const double t2 = t * t, t3 = t2 * t, u = 1.0 - t;
  w[0] = t3 / 6.0;
  w[1] = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
  w[2] = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
  w[3] = u * u * u / 6.0;
  dw[0] = t2 / 2.0;
  dw[1] = (-3.0 * t2 + 2.0 * t + 1.0) / 2.0;
  dw[2] = (3.0 * t2 - 4.0 * t) / 2.0;
  dw[3] = -u * u / 2.0;
}

// |b(m)|^2 = 1 / |sum_{k=0}^{2} M4(k+1) e^{2 pi i m k / K}|^2  (src/cell_based_kernels.cu:1868-1903)
double bmod2(int m, int K) {
  const double M4v[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
  cplx den = 0;
  for (int k = 0; k < 3; ++k) {
    const double a = 2.0 * kPi * (double)m * k / K;
    den += M4v[k] * cplx(std::cos(a), std::sin(a));
  }
  return 1.0 / std::norm(den);
}

// C(m) = |b(m)|^2 exp(-pi^2 |m|^2 / beta^2) / |m|^2 with m the reciprocal vector of
// grid index (mx, my, mz) (aliased to [-K/2, K/2]); 0 at m = 0.  The factor the
// transformed charge grid is multiplied by, up to CC / (pi V) (src/cell_based_kernels.cu:1770-1826)
double influence(int mx, int my, int mz, const int* K, const double* L, double beta, const double* bx,
                 const double* by, const double* bz) {
  if (mx == 0 && my == 0 && mz == 0) return 0.0;
  const double fx = (mx <= K[0] / 2 ? mx : mx - K[0]) / L[0];
  const double fy = (my <= K[1] / 2 ? my : my - K[1]) / L[1];
  const double fz = (mz <= K[2] / 2 ? mz : mz - K[2]) / L[2];
  const double m2 = fx * fx + fy * fy + fz * fz;
  return bx[mx] * by[my] * bz[mz] * std::exp(-kPi * kPi * m2 / (beta * beta)) / m2;
}

void pme(const Orc& o, const double* pos, double* f, double* e) {
  const int Kx = o.s.K[0], Ky = o.s.K[1], Kz = o.s.K[2];
  const double* L = o.s.box;
  const int n = o.s.n;
  const size_t Kt = (size_t)Kx * Ky * Kz;
  std::vector<cplx> Q(Kt, 0.0);
  const int K[3] = {Kx, Ky, Kz};
  std::vector<int> k0(3 * (size_t)n);
  std::vector<double> W(12 * (size_t)n), dW(12 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      double s = pos[3 * i + c] / L[c];
      s -= std::floor(s);
      double u = s * K[c];
      int ki = (int)std::floor(u);
      double t = u - ki;
      if (ki >= K[c]) ki -= K[c];
      k0[3 * i + c] = ki;
      bspline4(t, &W[12 * i + 4 * c], &dW[12 * i + 4 * c]);
    }
  }
  // spread (serial, deterministic): grid point k0 - j gets M4(t + j)
  for (int i = 0; i < n; ++i) {
    const double qi = o.q[i];
    for (int jz = 0; jz < 4; ++jz) {
      const int gz = ((k0[3 * i + 2] - jz) % Kz + Kz) % Kz;
      for (int jy = 0; jy < 4; ++jy) {
        const int gy = ((k0[3 * i + 1] - jy) % Ky + Ky) % Ky;
        const double wzy = W[12 * i + 8 + jz] * W[12 * i + 4 + jy] * qi;
        for (int jx = 0; jx < 4; ++jx) {
          const int gx = ((k0[3 * i] - jx) % Kx + Kx) % Kx;
          Q[((size_t)gz * Ky + gy) * Kx + gx] += wzy * W[12 * i + jx];
        }
      }
    }
  }
  const int nth = o.nthreads;
  fft3d(Q.data(), Kx, Ky, Kz, -1, nth);
  const double V = L[0] * L[1] * L[2];
  std::vector<double> bx(Kx), by(Ky), bz(Kz);
  for (int m = 0; m < Kx; ++m) bx[m] = bmod2(m, Kx);
  for (int m = 0; m < Ky; ++m) by[m] = bmod2(m, Ky);
  for (int m = 0; m < Kz; ++m) bz[m] = bmod2(m, Kz);
  double E = 0;
  for (int mz = 0; mz < Kz; ++mz) {
    for (int my = 0; my < Ky; ++my) {
      for (int mx = 0; mx < Kx; ++mx) {
        const size_t idx = ((size_t)mz * Ky + my) * Kx + mx;
        if (idx == 0) {
          Q[idx] = 0;
          continue;
        }
        const double C = influence(mx, my, mz, K, L, o.s.beta, bx.data(), by.data(), bz.data());
        E += C * std::norm(Q[idx]);
        Q[idx] *= ORC_CC / (kPi * V) * C;
      }
    }
  }
  E *= ORC_CC / (2.0 * kPi * V);
  fft3d(Q.data(), Kx, Ky, Kz, +1, nth);
  // gather
#pragma omp parallel for num_threads(nth) schedule(static)
  for (int i = 0; i < n; ++i) {
    double g[3] = {0, 0, 0};
    for (int jz = 0; jz < 4; ++jz) {
      const int gz = ((k0[3 * i + 2] - jz) % Kz + Kz) % Kz;
      for (int jy = 0; jy < 4; ++jy) {
        const int gy = ((k0[3 * i + 1] - jy) % Ky + Ky) % Ky;
        for (int jx = 0; jx < 4; ++jx) {
          const int gx = ((k0[3 * i] - jx) % Kx + Kx) % Kx;
          const double phi = Q[((size_t)gz * Ky + gy) * Kx + gx].real();
          const double* w = &W[12 * i];
          const double* dw = &dW[12 * i];
          g[0] += phi * dw[jx] * w[4 + jy] * w[8 + jz];
          g[1] += phi * w[jx] * dw[4 + jy] * w[8 + jz];
          g[2] += phi * w[jx] * w[4 + jy] * dw[8 + jz];
        }
      }
    }
    for (int c = 0; c < 3; ++c) f[3 * i + c] -= o.q[i] * g[c] * K[c] / L[c];
  }
  e[ORC_E_PME] = E;
}

// ---------------------------------------------------------------- nonbonded (cell list)
void nonbonded(const Orc& o, const double* pos, double* f, double* e) {
  const int n = o.s.n;
  const double* L = o.s.box;
  const double rc = o.s.rc, rc2 = rc * rc, ron2 = o.s.ron * o.s.ron, beta = o.s.beta;
  int nc[3];
  for (int c = 0; c < 3; ++c) nc[c] = std::max(1, (int)std::floor(L[c] / rc));
  const int ncell = nc[0] * nc[1] * nc[2];
  std::vector<int> cell(n), head(ncell + 1, 0), list(n);
  for (int i = 0; i < n; ++i) {
    int ci[3];
    for (int c = 0; c < 3; ++c) {
      double s = pos[3 * i + c] / L[c];
      s -= std::floor(s);
      ci[c] = std::min(nc[c] - 1, (int)(s * nc[c]));
    }
    cell[i] = (ci[2] * nc[1] + ci[1]) * nc[0] + ci[0];
    head[cell[i] + 1]++;
  }
  for (int c = 0; c < ncell; ++c) head[c + 1] += head[c];
  {
    std::vector<int> fill(head.begin(), head.end() - 1);
    for (int i = 0; i < n; ++i) list[fill[cell[i]]++] = i;
  }
  const int nt = o.s.ntypes;
  double ev = 0, ee = 0;
#pragma omp parallel for num_threads(o.nthreads) schedule(dynamic, 64) reduction(+ : ev, ee)
  for (int i = 0; i < n; ++i) {
    const int c = cell[i];
    const int cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
    std::vector<int> nbr;
    nbr.reserve(27);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = ((cx + dx) % nc[0] + nc[0]) % nc[0];
          const int y = ((cy + dy) % nc[1] + nc[1]) % nc[1];
          const int z = ((cz + dz) % nc[2] + nc[2]) % nc[2];
          nbr.push_back((z * nc[1] + y) * nc[0] + x);
        }
    std::sort(nbr.begin(), nbr.end());
    nbr.erase(std::unique(nbr.begin(), nbr.end()), nbr.end());
    double fi[3] = {0, 0, 0};
    const int ti = o.type[i];
    for (int cc : nbr) {
      for (int p = head[cc]; p < head[cc + 1]; ++p) {
        const int j = list[p];
        if (j == i) continue;
        double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
        minimg(d, L);
        const double r2 = dot3(d, d);
        if (r2 >= rc2) continue;
        if (excluded(o, i, j)) continue;
        const int tj = o.type[j];
        double evdw, eel;
        const double fr = pair_lj_coul(r2, o.q[i] * o.q[j], o.eps4[ti * nt + tj], o.sig2[ti * nt + tj],
                                       rc2, ron2, beta, &evdw, &eel);
        fi[0] += fr * d[0];
        fi[1] += fr * d[1];
        fi[2] += fr * d[2];
        ev += 0.5 * evdw;
        ee += 0.5 * eel;
      }
    }
    f[3 * i] += fi[0];
    f[3 * i + 1] += fi[1];
    f[3 * i + 2] += fi[2];
  }
  e[ORC_E_VDW] += ev;
  e[ORC_E_ELEC] += ee;
}

// Ewald exclusion correction, src/mdcuda.cu:520-553: E = -CC qq erf(beta r)/r
void excl_correction(const Orc& o, const double* pos, double* f, double* e) {
  const double beta = o.s.beta;
  double E = 0;
  for (auto& pr : o.ew_pairs) {
    const int i = pr.first, j = pr.second;
    double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    minimg(d, o.s.box);
    const double r2 = dot3(d, d), r = std::sqrt(r2);
    const double qq = o.q[i] * o.q[j];
    const double erfv = std::erf(beta * r);
    E += -ORC_CC * qq * erfv / r;
    const double fr = ORC_CC * qq * (2.0 / std::sqrt(kPi) * beta * r * std::exp(-beta * beta * r2) - erfv) / (r2 * r);
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] += fr * d[c];
      f[3 * j + c] -= fr * d[c];
    }
  }
  e[ORC_E_EWEXCL] += E;
}

// 1-4 pairs: 1-4 LJ (switched) + erfc Coulomb, no cutoff test (src/bonded_forces.cu:1155-1268)
void pairs14(const Orc& o, const double* pos, double* f, double* e) {
  const int nt = o.s.ntypes;
  const double rc2 = o.s.rc * o.s.rc, ron2 = o.s.ron * o.s.ron;
  double ev = 0, ee = 0;
  for (auto& pr : o.p14_pairs) {
    const int i = pr.first, j = pr.second;
    double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    minimg(d, o.s.box);
    const double r2 = dot3(d, d);
    const int ti = o.type[i], tj = o.type[j];
    double evdw, eel;
    const double fr = pair_lj_coul(r2, o.q[i] * o.q[j], o.eps4_14[ti * nt + tj], o.sig2_14[ti * nt + tj], rc2, ron2,
                                   o.s.beta, &evdw, &eel);
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] += fr * d[c];
      f[3 * j + c] -= fr * d[c];
    }
    ev += evdw;
    ee += eel;
  }
  e[ORC_E_VDW] += ev;
  e[ORC_E_ELEC] += ee;
}

// ---------------------------------------------------------------- bonded
void bonds(const Orc& o, const double* pos, double* f, double* e) {
  double E = 0;
  for (int b = 0; b < o.s.nbond; ++b) {
    const int i = o.bond[2 * b], j = o.bond[2 * b + 1];
    double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    minimg(d, o.s.box);
    const double r = std::sqrt(dot3(d, d));
    const double dr = r - o.bond_r0[b];
    E += o.bond_k[b] * dr * dr;
    const double fr = -2.0 * o.bond_k[b] * dr / r;
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] += fr * d[c];
      f[3 * j + c] -= fr * d[c];
    }
  }
  e[ORC_E_BOND] += E;
}

void ureyb(const Orc& o, const double* pos, double* f, double* e) {
  double E = 0;
  for (int b = 0; b < o.s.nub; ++b) {
    const int i = o.ub[2 * b], j = o.ub[2 * b + 1];
    double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    minimg(d, o.s.box);
    const double r = std::sqrt(dot3(d, d));
    const double dr = r - o.ub_r0[b];
    E += o.ub_k[b] * dr * dr;
    const double fr = -2.0 * o.ub_k[b] * dr / r;
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] += fr * d[c];
      f[3 * j + c] -= fr * d[c];
    }
  }
  e[ORC_E_UREYB] += E;
}

void angles(const Orc& o, const double* pos, double* f, double* e) {
  double E = 0;
  for (int a = 0; a < o.s.nangle; ++a) {
    const int i = o.angle[3 * a], j = o.angle[3 * a + 1], k = o.angle[3 * a + 2];
    double u[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    double v[3] = {pos[3 * k] - pos[3 * j], pos[3 * k + 1] - pos[3 * j + 1], pos[3 * k + 2] - pos[3 * j + 2]};
    minimg(u, o.s.box);
    minimg(v, o.s.box);
    const double uu = dot3(u, u), vv = dot3(v, v), uv = dot3(u, v);
    const double ru = std::sqrt(uu), rv = std::sqrt(vv);
    double c = uv / (ru * rv);
    c = std::max(-1.0, std::min(1.0, c));
    double w[3];
    cross3(u, v, w);
    const double sn = std::sqrt(dot3(w, w)) / (ru * rv);
    const double th = std::atan2(sn, c);
    const double dth = th - o.angle_t0[a];
    E += o.angle_k[a] * dth * dth;
    const double dE = 2.0 * o.angle_k[a] * dth;  // dE/dtheta
    // dtheta/du = -(v/|v| - c u/|u|) / (|u| sin)
    const double s = std::max(sn, 1e-12);
    for (int cc = 0; cc < 3; ++cc) {
      const double gu = -(v[cc] / (ru * rv) - c * u[cc] / uu) / s;
      const double gv = -(u[cc] / (ru * rv) - c * v[cc] / vv) / s;
      f[3 * i + cc] -= dE * gu;
      f[3 * k + cc] -= dE * gv;
      f[3 * j + cc] += dE * (gu + gv);
    }
  }
  e[ORC_E_ANGLE] += E;
}

// dihedral angle (IUPAC sign) and its gradients, Blondel & Karplus, J. Comput. Chem. 17, 1132 (1996)
inline double dihedral_grad(const double* pos, const double* L, int i, int j, int k, int l, double gi[3],
                            double gj[3], double gk[3], double gl[3]) {
  double F[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
  double G[3] = {pos[3 * j] - pos[3 * k], pos[3 * j + 1] - pos[3 * k + 1], pos[3 * j + 2] - pos[3 * k + 2]};
  double H[3] = {pos[3 * l] - pos[3 * k], pos[3 * l + 1] - pos[3 * k + 1], pos[3 * l + 2] - pos[3 * k + 2]};
  minimg(F, L);
  minimg(G, L);
  minimg(H, L);
  double A[3], B[3];
  cross3(F, G, A);
  cross3(H, G, B);
  const double A2 = dot3(A, A), B2 = dot3(B, B), Gn = std::sqrt(dot3(G, G));
  double AxB[3];
  cross3(B, A, AxB);
  const double cphi = dot3(A, B);
  const double sphi = dot3(AxB, G) / Gn;
  const double phi = std::atan2(sphi, cphi);
  const double FG = dot3(F, G), HG = dot3(H, G);
  for (int c = 0; c < 3; ++c) {
    gi[c] = -Gn / A2 * A[c];
    gl[c] = Gn / B2 * B[c];
    gj[c] = Gn / A2 * A[c] + FG / (A2 * Gn) * A[c] - HG / (B2 * Gn) * B[c];
    gk[c] = -Gn / B2 * B[c] - FG / (A2 * Gn) * A[c] + HG / (B2 * Gn) * B[c];
  }
  return phi;
}

void dihedrals(const Orc& o, const double* pos, double* f, double* e) {
  double E = 0;
  for (int d = 0; d < o.s.ndihe; ++d) {
    const int i = o.dihe[4 * d], j = o.dihe[4 * d + 1], k = o.dihe[4 * d + 2], l = o.dihe[4 * d + 3];
    double gi[3], gj[3], gk[3], gl[3];
    const double phi = dihedral_grad(pos, o.s.box, i, j, k, l, gi, gj, gk, gl);
    const double K = o.dihe_k[d], nn = o.dihe_n[d], dl = o.dihe_d[d];
    E += K * (1.0 + std::cos(nn * phi - dl));
    const double dE = -K * nn * std::sin(nn * phi - dl);
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] -= dE * gi[c];
      f[3 * j + c] -= dE * gj[c];
      f[3 * k + c] -= dE * gk[c];
      f[3 * l + c] -= dE * gl[c];
    }
  }
  e[ORC_E_DIHED] += E;
}

// impropers: E = K (psi - psi0)^2 with the signed dihedral angle psi.  (The reference
// ignores psi0, src/bonded_forces.cu:216; identical whenever psi0 = 0.)
void impropers(const Orc& o, const double* pos, double* f, double* e) {
  double E = 0;
  for (int d = 0; d < o.s.nimpr; ++d) {
    const int i = o.impr[4 * d], j = o.impr[4 * d + 1], k = o.impr[4 * d + 2], l = o.impr[4 * d + 3];
    double gi[3], gj[3], gk[3], gl[3];
    const double psi = dihedral_grad(pos, o.s.box, i, j, k, l, gi, gj, gk, gl);
    double dp = psi - o.impr_p0[d];
    dp -= 2.0 * kPi * std::nearbyint(dp / (2.0 * kPi));
    E += o.impr_k[d] * dp * dp;
    const double dE = 2.0 * o.impr_k[d] * dp;
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] -= dE * gi[c];
      f[3 * j + c] -= dE * gj[c];
      f[3 * k + c] -= dE * gk[c];
      f[3 * l + c] -= dE * gl[c];
    }
  }
  e[ORC_E_IMPR] += E;
}

// ---------------------------------------------------------------- constraints
// SHAKE, Newton iteration with Gauss elimination per cluster (src/shake.cu:20-327), FP64.
bool gauss_solve(int n, double J[3][3], double* rhs, double* x) {
  for (int k = 0; k < n; ++k) {
    if (J[k][k] == 0.0) return false;
    for (int r = k + 1; r < n; ++r) {
      const double m = J[r][k] / J[k][k];
      for (int c = k + 1; c < n; ++c) J[r][c] -= m * J[k][c];
      rhs[r] -= m * rhs[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double t = rhs[k];
    for (int c = k + 1; c < n; ++c) t -= J[k][c] * x[c];
    x[k] = t / J[k][k];
  }
  return true;
}

int shake_cluster(const Orc& o, const Cluster& cl, const double* pref, double* pos, double* vel, double dtu,
                  double tol, int maxit) {
  const double* L = o.s.box;
  double rd[3][3], rn[4][3], im[4];
  for (int a = 0; a < cl.na; ++a) {
    im[a] = 1.0 / o.mass[cl.atom[a]];
    for (int c = 0; c < 3; ++c) rn[a][c] = pos[3 * cl.atom[a] + c];
  }
  for (int k = 0; k < cl.nc; ++k) {
    const int ga = cl.atom[cl.ca[k]], gb = cl.atom[cl.cb[k]];
    for (int c = 0; c < 3; ++c) rd[k][c] = pref[3 * ga + c] - pref[3 * gb + c];
    minimg(rd[k], L);
  }
  double lam[3] = {0, 0, 0};
  int it = 0;
  for (; it < maxit; ++it) {
    double dr[4][3] = {};
    for (int k = 0; k < cl.nc; ++k)
      for (int c = 0; c < 3; ++c) {
        dr[cl.ca[k]][c] += rd[k][c] * lam[k] * im[cl.ca[k]];
        dr[cl.cb[k]][c] -= rd[k][c] * lam[k] * im[cl.cb[k]];
      }
    double J[3][3] = {}, sig[3] = {};
    for (int k = 0; k < cl.nc; ++k) {
      const int a = cl.ca[k], b = cl.cb[k];
      double C[3];
      for (int c = 0; c < 3; ++c) C[c] = rn[a][c] - rn[b][c];
      minimg(C, L);
      for (int c = 0; c < 3; ++c) C[c] += dr[a][c] - dr[b][c];
      sig[k] = dot3(C, C) - cl.d[k] * cl.d[k];
      for (int l = 0; l < cl.nc; ++l) {
        double coef = 0;
        if (cl.ca[l] == a) coef += im[a];
        if (cl.cb[l] == a) coef -= im[a];
        if (cl.ca[l] == b) coef -= im[b];
        if (cl.cb[l] == b) coef += im[b];
        J[k][l] = 2.0 * coef * dot3(rd[l], C);
      }
    }
    double dl[3];
    if (!gauss_solve(cl.nc, J, sig, dl)) return -1;
    double t = 0;
    for (int k = 0; k < cl.nc; ++k) {
      lam[k] -= dl[k];
      t += dl[k] * dl[k];
    }
    if (t < tol) break;
  }
  double dr[4][3] = {};
  for (int k = 0; k < cl.nc; ++k)
    for (int c = 0; c < 3; ++c) {
      dr[cl.ca[k]][c] += rd[k][c] * lam[k] * im[cl.ca[k]];
      dr[cl.cb[k]][c] -= rd[k][c] * lam[k] * im[cl.cb[k]];
    }
  for (int a = 0; a < cl.na; ++a)
    for (int c = 0; c < 3; ++c) {
      pos[3 * cl.atom[a] + c] += dr[a][c];
      if (vel) vel[3 * cl.atom[a] + c] += dr[a][c] / dtu;
    }
  return it >= maxit ? 1 : 0;
}

// RATTLE velocity stage (src/shake.cu:330-615): linear system solved directly.
void rattle_cluster(const Orc& o, const Cluster& cl, const double* pos, double* vel) {
  double rd[3][3], im[4];
  for (int a = 0; a < cl.na; ++a) im[a] = 1.0 / o.mass[cl.atom[a]];
  for (int k = 0; k < cl.nc; ++k) {
    const int ga = cl.atom[cl.ca[k]], gb = cl.atom[cl.cb[k]];
    for (int c = 0; c < 3; ++c) rd[k][c] = pos[3 * ga + c] - pos[3 * gb + c];
    minimg(rd[k], o.s.box);
  }
  double J[3][3] = {}, rhs[3] = {}, mu[3];
  for (int k = 0; k < cl.nc; ++k) {
    const int a = cl.ca[k], b = cl.cb[k];
    double vab[3];
    for (int c = 0; c < 3; ++c) vab[c] = vel[3 * cl.atom[a] + c] - vel[3 * cl.atom[b] + c];
    rhs[k] = dot3(vab, rd[k]);
    for (int l = 0; l < cl.nc; ++l) {
      double coef = 0;
      if (cl.ca[l] == a) coef += im[a];
      if (cl.cb[l] == a) coef -= im[a];
      if (cl.ca[l] == b) coef -= im[b];
      if (cl.cb[l] == b) coef += im[b];
      J[k][l] = coef * dot3(rd[l], rd[k]);
    }
  }
  if (!gauss_solve(cl.nc, J, rhs, mu)) return;
  for (int k = 0; k < cl.nc; ++k)
    for (int c = 0; c < 3; ++c) {
      vel[3 * cl.atom[cl.ca[k]] + c] -= rd[k][c] * mu[k] * im[cl.ca[k]];
      vel[3 * cl.atom[cl.cb[k]] + c] += rd[k][c] * mu[k] * im[cl.cb[k]];
    }
}

// ---------------------------------------------------------------- RNG (splitmix64, Steele/Lea/Flood 2014)
inline uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double u01(uint64_t r) { return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

}  // namespace

// ====================================================================== C ABI
extern "C" {

void* orc_create(const orc_system* s) {
  Orc* o = new Orc();
  o->s = *s;
  const int n = s->n, nt = s->ntypes;
  o->q.assign(s->q, s->q + n);
  o->mass.assign(s->mass, s->mass + n);
  o->type.assign(s->type, s->type + n);
  o->eps4.assign(s->eps4, s->eps4 + nt * nt);
  o->sig2.assign(s->sig2, s->sig2 + nt * nt);
  o->eps4_14.assign(s->eps4_14, s->eps4_14 + nt * nt);
  o->sig2_14.assign(s->sig2_14, s->sig2_14 + nt * nt);
  auto cp_i = [](std::vector<int>& v, const int* p, size_t c) { v.assign(p, p + c); };
  auto cp_d = [](std::vector<double>& v, const double* p, size_t c) { v.assign(p, p + c); };
  cp_i(o->bond, s->bond, 2 * (size_t)s->nbond);
  cp_d(o->bond_k, s->bond_k, s->nbond);
  cp_d(o->bond_r0, s->bond_r0, s->nbond);
  cp_i(o->angle, s->angle, 3 * (size_t)s->nangle);
  cp_d(o->angle_k, s->angle_k, s->nangle);
  cp_d(o->angle_t0, s->angle_t0, s->nangle);
  cp_i(o->ub, s->ub, 2 * (size_t)s->nub);
  cp_d(o->ub_k, s->ub_k, s->nub);
  cp_d(o->ub_r0, s->ub_r0, s->nub);
  cp_i(o->dihe, s->dihe, 4 * (size_t)s->ndihe);
  cp_d(o->dihe_k, s->dihe_k, s->ndihe);
  cp_i(o->dihe_n, s->dihe_n, s->ndihe);
  cp_d(o->dihe_d, s->dihe_d, s->ndihe);
  cp_i(o->impr, s->impr, 4 * (size_t)s->nimpr);
  cp_d(o->impr_k, s->impr_k, s->nimpr);
  cp_d(o->impr_p0, s->impr_p0, s->nimpr);
  cp_i(o->cons, s->cons, 2 * (size_t)s->ncons);
  cp_d(o->cons_d, s->cons_d, s->ncons);
  o->s.q = o->q.data();
  o->s.mass = o->mass.data();
  o->s.type = o->type.data();
  o->nthreads = s->nthreads > 0 ? s->nthreads : 1;
#ifdef _OPENMP
  if (s->nthreads <= 0) o->nthreads = omp_get_max_threads();
#endif
  // exclusions, src/prmread.cu:2928-3062: 1-2 (bonds) + 1-3 (angle ends) -> Ewald list;
  // + 1-4 (dihedral ends) -> full exclusion list.
  std::set<std::pair<int, int>> ew, ex, p14;
  auto key = [](int a, int b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); };
  for (int b = 0; b < s->nbond; ++b)
    if (o->bond[2 * b] != o->bond[2 * b + 1]) ew.insert(key(o->bond[2 * b], o->bond[2 * b + 1]));
  for (int a = 0; a < s->nangle; ++a)
    if (o->angle[3 * a] != o->angle[3 * a + 2]) ew.insert(key(o->angle[3 * a], o->angle[3 * a + 2]));
  ex = ew;
  for (int d = 0; d < s->ndihe; ++d) {
    auto k = key(o->dihe[4 * d], o->dihe[4 * d + 3]);
    if (k.first == k.second) continue;
    ex.insert(k);
    if (!ew.count(k)) p14.insert(k);
  }
  o->ew_pairs.assign(ew.begin(), ew.end());
  o->p14_pairs.assign(p14.begin(), p14.end());
  std::vector<std::vector<int>> per(n);
  for (auto& pr : ex) {
    per[pr.first].push_back(pr.second);
    per[pr.second].push_back(pr.first);
  }
  o->excl_off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    std::sort(per[i].begin(), per[i].end());
    o->excl_off[i + 1] = o->excl_off[i] + (int)per[i].size();
  }
  o->excl_idx.reserve(o->excl_off[n]);
  for (int i = 0; i < n; ++i) o->excl_idx.insert(o->excl_idx.end(), per[i].begin(), per[i].end());
  // clusters = connected components of the constraint graph (src/prmread.cu:1192-1439)
  std::vector<int> parent(n);
  for (int i = 0; i < n; ++i) parent[i] = i;
  auto findf = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (int c = 0; c < s->ncons; ++c) {
    const int a = findf(o->cons[2 * c]), b = findf(o->cons[2 * c + 1]);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
  std::vector<int> cid(n, -1);
  for (int c = 0; c < s->ncons; ++c) {
    const int a = o->cons[2 * c], b = o->cons[2 * c + 1];
    const int r = findf(a);
    if (cid[r] < 0) {
      cid[r] = (int)o->clusters.size();
      o->clusters.emplace_back();
    }
    Cluster& cl = o->clusters[cid[r]];
    auto local = [&](int g) {
      for (int t = 0; t < cl.na; ++t)
        if (cl.atom[t] == g) return t;
      if (cl.na >= 4) return -1;
      cl.atom[cl.na] = g;
      return cl.na++;
    };
    const int la = local(a), lb = local(b);
    if (la < 0 || lb < 0 || cl.nc >= 3) {
      delete o;
      return nullptr;
    }
    cl.ca[cl.nc] = la;
    cl.cb[cl.nc] = lb;
    cl.d[cl.nc] = o->cons_d[c];
    cl.nc++;
  }
  return o;
}

void orc_destroy(void* h) { delete (Orc*)h; }

int orc_counts(void* h, int* out4) {
  Orc* o = (Orc*)h;
  out4[0] = (int)o->ew_pairs.size();
  out4[1] = (int)o->p14_pairs.size();
  out4[2] = (int)o->clusters.size();
  out4[3] = o->s.ncons;
  return 0;
}

int orc_forces(void* h, const double* pos, double* f, double* e, int terms) {
  Orc* o = (Orc*)h;
  for (int k = 0; k < ORC_NE; ++k) e[k] = 0;
  if (terms & ORC_T_NB) nonbonded(*o, pos, f, e);
  if (terms & ORC_T_EXCL) excl_correction(*o, pos, f, e);
  if (terms & ORC_T_P14) pairs14(*o, pos, f, e);
  if (terms & ORC_T_PME) pme(*o, pos, f, e);
  if (terms & ORC_T_BOND) bonds(*o, pos, f, e);
  if (terms & ORC_T_ANGLE) angles(*o, pos, f, e);
  if (terms & ORC_T_UREYB) ureyb(*o, pos, f, e);
  if (terms & ORC_T_DIHED) dihedrals(*o, pos, f, e);
  if (terms & ORC_T_IMPR) impropers(*o, pos, f, e);
  if (terms & ORC_T_SELF) {
    double s = 0;
    for (int i = 0; i < o->s.n; ++i) s += o->q[i] * o->q[i];
    e[ORC_E_EWSELF] = -ORC_CC * o->s.beta / std::sqrt(kPi) * s;
  }
  return 0;
}

int orc_ewald_recip(void* h, const double* pos, int kmax, double* f, double* e) {
  Orc* o = (Orc*)h;
  const int n = o->s.n;
  const double* L = o->s.box;
  const double V = L[0] * L[1] * L[2], b2 = o->s.beta * o->s.beta;
  const int nk = 2 * kmax + 1;
  // e^{2 pi i k x / L} tables
  std::vector<cplx> ex((size_t)n * nk), ey((size_t)n * nk), ez((size_t)n * nk);
  for (int i = 0; i < n; ++i)
    for (int k = -kmax; k <= kmax; ++k) {
      const double ax = 2 * kPi * k * pos[3 * i] / L[0], ay = 2 * kPi * k * pos[3 * i + 1] / L[1],
                   az = 2 * kPi * k * pos[3 * i + 2] / L[2];
      ex[(size_t)i * nk + k + kmax] = cplx(std::cos(ax), std::sin(ax));
      ey[(size_t)i * nk + k + kmax] = cplx(std::cos(ay), std::sin(ay));
      ez[(size_t)i * nk + k + kmax] = cplx(std::cos(az), std::sin(az));
    }
  const double lmin = std::min(L[0], std::min(L[1], L[2]));
  const double m2max = (kmax / lmin) * (kmax / lmin);
  std::vector<std::array<int, 3>> ms;
  for (int mx = 0; mx <= kmax; ++mx)
    for (int my = -kmax; my <= kmax; ++my)
      for (int mz = -kmax; mz <= kmax; ++mz) {
        // half space
        if (mx == 0 && (my < 0 || (my == 0 && mz <= 0))) continue;
        const double fx = mx / L[0], fy = my / L[1], fz = mz / L[2];
        if (fx * fx + fy * fy + fz * fz > m2max) continue;
        ms.push_back({mx, my, mz});
      }
  const int nth = o->nthreads;
  double E = 0;
  std::vector<double> fl((size_t)nth * 3 * n, 0.0);
#pragma omp parallel num_threads(nth) reduction(+ : E)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* myf = &fl[(size_t)tid * 3 * n];
    std::vector<cplx> eij(n);
#pragma omp for schedule(dynamic, 16)
    for (int t = 0; t < (int)ms.size(); ++t) {
      const int mx = ms[t][0], my = ms[t][1], mz = ms[t][2];
      const double fx = mx / L[0], fy = my / L[1], fz = mz / L[2];
      const double m2 = fx * fx + fy * fy + fz * fz;
      const double C = std::exp(-kPi * kPi * m2 / b2) / m2;
      cplx S = 0;
      for (int i = 0; i < n; ++i) {
        eij[i] = ex[(size_t)i * nk + mx + kmax] * ey[(size_t)i * nk + my + kmax] * ez[(size_t)i * nk + mz + kmax];
        S += o->q[i] * eij[i];
      }
      // half space: factor 2
      E += 2.0 * C * std::norm(S);
      for (int i = 0; i < n; ++i) {
        const double im = (std::conj(S) * eij[i]).imag();
        const double g = 2.0 * C * 4.0 * kPi * o->q[i] * im;
        myf[3 * i] += g * fx;
        myf[3 * i + 1] += g * fy;
        myf[3 * i + 2] += g * fz;
      }
    }
  }
  const double A = ORC_CC / (2.0 * kPi * V);
  for (int t = 0; t < nth; ++t)
    for (int i = 0; i < 3 * n; ++i) f[i] += A * fl[(size_t)t * 3 * n + i];
  e[0] = A * E;
  return 0;
}

int orc_fft3d(int nx, int ny, int nz, double* data, int sign) {
  fft3d(reinterpret_cast<cplx*>(data), nx, ny, nz, sign, 4);
  return 0;
}

int orc_pme_influence(const int* K, const double* L, double beta, double* G) {
  std::vector<double> b[3];
  for (int d = 0; d < 3; ++d) {
    b[d].resize(K[d]);
    for (int m = 0; m < K[d]; ++m) b[d][m] = bmod2(m, K[d]);
  }
  for (int mz = 0; mz < K[2]; ++mz)
    for (int my = 0; my < K[1]; ++my)
      for (int mx = 0; mx < K[0]; ++mx)
        G[((size_t)mz * K[1] + my) * K[0] + mx] =
            influence(mx, my, mz, K, L, beta, b[0].data(), b[1].data(), b[2].data());
  return 0;
}

long long orc_count_pairs(void* h, const double* pos, double rcut) {
  Orc* o = (Orc*)h;
  // reuse the nonbonded cell loop via brute force over cells
  const int n = o->s.n;
  const double* L = o->s.box;
  int nc[3];
  for (int c = 0; c < 3; ++c) nc[c] = std::max(1, (int)std::floor(L[c] / rcut));
  const int ncell = nc[0] * nc[1] * nc[2];
  std::vector<int> cell(n), head(ncell + 1, 0), list(n);
  for (int i = 0; i < n; ++i) {
    int ci[3];
    for (int c = 0; c < 3; ++c) {
      double s = pos[3 * i + c] / L[c];
      s -= std::floor(s);
      ci[c] = std::min(nc[c] - 1, (int)(s * nc[c]));
    }
    cell[i] = (ci[2] * nc[1] + ci[1]) * nc[0] + ci[0];
    head[cell[i] + 1]++;
  }
  for (int c = 0; c < ncell; ++c) head[c + 1] += head[c];
  {
    std::vector<int> fill(head.begin(), head.end() - 1);
    for (int i = 0; i < n; ++i) list[fill[cell[i]]++] = i;
  }
  long long cnt = 0;
  const double r2c = rcut * rcut;
#pragma omp parallel for num_threads(o->nthreads) schedule(dynamic, 64) reduction(+ : cnt)
  for (int i = 0; i < n; ++i) {
    const int c = cell[i];
    const int cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
    std::vector<int> nbr;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = ((cx + dx) % nc[0] + nc[0]) % nc[0];
          const int y = ((cy + dy) % nc[1] + nc[1]) % nc[1];
          const int z = ((cz + dz) % nc[2] + nc[2]) % nc[2];
          nbr.push_back((z * nc[1] + y) * nc[0] + x);
        }
    std::sort(nbr.begin(), nbr.end());
    nbr.erase(std::unique(nbr.begin(), nbr.end()), nbr.end());
    for (int cc : nbr)
      for (int p = head[cc]; p < head[cc + 1]; ++p) {
        const int j = list[p];
        if (j <= i) continue;
        double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
        minimg(d, L);
        if (dot3(d, d) < r2c && !excluded(*o, i, j)) cnt++;
      }
  }
  return cnt;
}

int orc_shake(void* h, const double* pos_ref, double* pos, double* vel, double dt_ps, double tol, int maxit) {
  Orc* o = (Orc*)h;
  const double dtu = dt_ps * ORC_TU;
  int bad = 0;
#pragma omp parallel for num_threads(o->nthreads) reduction(+ : bad)
  for (int c = 0; c < (int)o->clusters.size(); ++c)
    bad += shake_cluster(*o, o->clusters[c], pos_ref, pos, vel, dtu, tol, maxit) != 0;
  return bad;
}

int orc_rattle(void* h, const double* pos, double* vel) {
  Orc* o = (Orc*)h;
#pragma omp parallel for num_threads(o->nthreads)
  for (int c = 0; c < (int)o->clusters.size(); ++c) rattle_cluster(*o, o->clusters[c], pos, vel);
  return 0;
}

double orc_kinetic(void* h, const double* vel) {
  Orc* o = (Orc*)h;
  double k = 0;
  for (int i = 0; i < o->s.n; ++i)
    k += 0.5 * o->mass[i] * (vel[3 * i] * vel[3 * i] + vel[3 * i + 1] * vel[3 * i + 1] + vel[3 * i + 2] * vel[3 * i + 2]);
  return k;
}

int orc_md(void* h, double* pos, double* vel, int nsteps, double dt_ps, double tol, double* fout, double* epot,
           double* ekin) {
  Orc* o = (Orc*)h;
  const int n = o->s.n;
  const double dtu = dt_ps * ORC_TU;
  std::vector<double> f(3 * (size_t)n, 0.0), ref(3 * (size_t)n);
  double e[ORC_NE];
  orc_forces(h, pos, f.data(), e, ORC_T_ALL);
  int bad = 0;
  for (int s = 0; s < nsteps; ++s) {
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        vel[3 * i + c] += 0.5 * dtu * f[3 * i + c] / o->mass[i];
        ref[3 * i + c] = pos[3 * i + c];
        pos[3 * i + c] += dtu * vel[3 * i + c];
      }
    bad += orc_shake(h, ref.data(), pos, vel, dt_ps, tol, 1000);
    std::fill(f.begin(), f.end(), 0.0);
    orc_forces(h, pos, f.data(), e, ORC_T_ALL);
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) vel[3 * i + c] += 0.5 * dtu * f[3 * i + c] / o->mass[i];
    orc_rattle(h, pos, vel);
    if (epot) {
      double sum = 0;
      for (int k = 0; k < ORC_NE; ++k) sum += e[k];
      epot[s] = sum;
    }
    if (ekin) ekin[s] = orc_kinetic(h, vel);
  }
  if (fout) std::memcpy(fout, f.data(), sizeof(double) * 3 * n);
  return bad;
}

// Energy minimisation, the reference's MinimizeStep loop (src/dynamics.cu:491-620) with
// the moves of ConjugatedGradient / SteepestDescent (src/mdcuda.cu:126-351) and the
// factor schedule of main() (src/fenzi.cu:397-418), in FP64:
//   CG move per atom: gamma = |F|^2 / |F_prev|^2 (F_prev replaced by F when
//     |F_prev|^2 < 1e-8), H = (F + gamma H_prev) cgfac, r += H; F_prev = F, H_prev = H;
//   SD move per atom: r += F sdfac;
//   after the move the energy is evaluated; if it rose (never on the first move, where
//   the reference's previous energy is still its 0 sentinel) the move is undone, the
//   step is not counted, and CG switches to SD, SD ends the minimisation;
//   every 100 counted steps (step > 0) the current method's factor is multiplied by
//   rate x 100.
// Constrained units are kept rigid by SHAKE against the positions before the move
// (the reference moves those atoms freely).  pos in/out; energies[k] (may be NULL) is
// the potential energy after counted step k; methods[k] (may be NULL) the method of
// that step's move.  Returns the number of counted steps.
int orc_minimize(void* h, double* pos, int max_steps, double cgfac, double sdfac, double cgrate, double sdrate,
                 double* energies, int* methods) {
  Orc* o = (Orc*)h;
  const int n = o->s.n;
  std::vector<double> f(3 * (size_t)n), fprev(3 * (size_t)n, 0.0), dir(3 * (size_t)n, 0.0),
      pos0(3 * (size_t)n), vel(3 * (size_t)n, 0.0);
  double e[ORC_NE];
  auto evaluate = [&]() {
    std::fill(f.begin(), f.end(), 0.0);
    orc_forces(h, pos, f.data(), e, ORC_T_ALL);
    double u = 0;
    for (int k = 0; k < ORC_NE; ++k) u += e[k];
    return u;
  };
  int method = 1;
  double fac[3] = {0.0, cgfac, sdfac};
  const double rate[3] = {0.0, cgrate, sdrate};
  double cur = evaluate(), prev = 0.0;
  bool first = true;
  int step = 0;
  for (; step < max_steps && method != 0; ++step) {
    std::memcpy(pos0.data(), pos, sizeof(double) * 3 * n);
    const int used = method;
    for (int i = 0; i < n; ++i) {
      double* F = &f[3 * (size_t)i];
      double H[3];
      if (method == 1) {
        double* F1 = &fprev[3 * (size_t)i];
        const double ff = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
        double f11 = F1[0] * F1[0] + F1[1] * F1[1] + F1[2] * F1[2];
        if (f11 < 1e-8) f11 = ff;
        const double gamma = f11 > 0.0 ? ff / f11 : 0.0;
        for (int c = 0; c < 3; ++c) {
          H[c] = (F[c] + dir[3 * (size_t)i + c] * gamma) * fac[1];
          dir[3 * (size_t)i + c] = H[c];
          F1[c] = F[c];
        }
      } else {
        for (int c = 0; c < 3; ++c) H[c] = F[c] * fac[2];
      }
      for (int c = 0; c < 3; ++c) pos[3 * (size_t)i + c] += H[c];
    }
    if (o->s.ncons > 0) orc_shake(h, pos0.data(), pos, vel.data(), 1.0, 1e-12, 1000);
    prev = cur;
    cur = evaluate();
    if (cur > prev && !first) {
      std::memcpy(pos, pos0.data(), sizeof(double) * 3 * n);
      cur = evaluate();
      method = method == 1 ? 2 : 0;
      --step;
    } else {
      if (energies) energies[step] = cur;
      if (methods) methods[step] = used;
    }
    first = false;
    if (step > 0 && step % 100 == 0 && method != 0) fac[method] *= rate[method] * 100.0;
  }
  return step;
}

void orc_normals(int n, uint64_t seed, uint32_t counter, double* out) {
  const uint64_t z = splitmix64(seed ^ (0xD1B54A32D192ED03ULL * ((uint64_t)counter + 1)));
  for (int a = 0; a < n; ++a) {
    const uint64_t base = z + 4ULL * (uint64_t)a;
    const double u1 = u01(splitmix64(base)), u2 = u01(splitmix64(base + 1));
    const double u3 = u01(splitmix64(base + 2)), u4 = u01(splitmix64(base + 3));
    const double r1 = std::sqrt(-2.0 * std::log(u1)), r2 = std::sqrt(-2.0 * std::log(u3));
    out[3 * a] = r1 * std::cos(2.0 * kPi * u2);
    out[3 * a + 1] = r1 * std::sin(2.0 * kPi * u2);
    out[3 * a + 2] = r2 * std::cos(2.0 * kPi * u4);
  }
}

void orc_reassign_velocities(void* h, const double* pos, double T, uint64_t seed, uint32_t counter, double* vel) {
  Orc* o = (Orc*)h;
  const int n = o->s.n;
  orc_normals(n, seed, counter, vel);
  double p[3] = {0, 0, 0}, mt = 0;
  for (int i = 0; i < n; ++i) {
    const double sd = std::sqrt(ORC_RC * T / o->mass[i]);
    for (int c = 0; c < 3; ++c) {
      vel[3 * i + c] *= sd;
      p[c] += o->mass[i] * vel[3 * i + c];
    }
    mt += o->mass[i];
  }
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) vel[3 * i + c] -= p[c] / mt;
  orc_rattle(h, pos, vel);
}

}  // extern "C"

// ---------------------------------------------------------------- virial, pressure, Andersen barostat
namespace {

// integration units: SHAKE clusters and free atoms (the barostat's scaling groups)
std::vector<std::vector<int>> units_of(const Orc& o) {
  std::vector<std::vector<int>> u;
  std::vector<int> in_cl(o.s.n, 0);
  for (const Cluster& cl : o.clusters) {
    u.emplace_back(cl.atom, cl.atom + cl.na);
    for (int a = 0; a < cl.na; ++a) in_cl[cl.atom[a]] = 1;
  }
  for (int i = 0; i < o.s.n; ++i)
    if (!in_cl[i]) u.push_back({i});
  return u;
}

// mass centre of a unit (min-imaged about its first atom)
void centre(const Orc& o, const std::vector<int>& u, const double* pos, double* R) {
  double cm[3] = {0, 0, 0}, mt = 0;
  for (int i : u) {
    double d[3] = {pos[3 * i] - pos[3 * u[0]], pos[3 * i + 1] - pos[3 * u[0] + 1], pos[3 * i + 2] - pos[3 * u[0] + 2]};
    minimg(d, o.s.box);
    for (int c = 0; c < 3; ++c) cm[c] += o.mass[i] * d[c];
    mt += o.mass[i];
  }
  for (int c = 0; c < 3; ++c) R[c] = pos[3 * u[0] + c] + cm[c] / mt;
}

// W_aa = -L_a dU/dL_a by central differences of the energy at fixed fractional
// coordinates: of every atom (group = 0, the atomic virial) or of every unit's mass
// centre with the units moved rigidly (group = 1, the group virial).
void virial_fd(const Orc& o, const double* pos, double h, int terms, double* vir, int group) {
  const int n = o.s.n;
  std::vector<double> ps(3 * (size_t)n), f(3 * (size_t)n), R;
  std::vector<std::vector<int>> units;
  if (group) {
    units = units_of(o);
    R.resize(3 * units.size());
    for (size_t k = 0; k < units.size(); ++k) centre(o, units[k], pos, &R[3 * k]);
  }
  double e[ORC_NE];
  for (int a = 0; a < 3; ++a) {
    double u[2];
    for (int sgn = 0; sgn < 2; ++sgn) {
      const double sc = sgn ? 1.0 - h : 1.0 + h;
      Orc w = o;
      w.s.box[a] = o.s.box[a] * sc;
      for (int i = 0; i < 3 * n; ++i) ps[i] = pos[i];
      if (group) {  // the centre's image next to each atom, so wrapped units move rigidly
        for (size_t k = 0; k < units.size(); ++k)
          for (int i : units[k]) {
            const int a0 = units[k][0];
            double d[3] = {pos[3 * i] - pos[3 * a0], pos[3 * i + 1] - pos[3 * a0 + 1], pos[3 * i + 2] - pos[3 * a0 + 2]};
            double dm[3] = {d[0], d[1], d[2]};
            minimg(dm, o.s.box);
            ps[3 * i + a] += (sc - 1.0) * (R[3 * k + a] + d[a] - dm[a]);
          }
      } else {
        for (int i = 0; i < n; ++i) ps[3 * i + a] *= sc;
      }
      std::fill(f.begin(), f.end(), 0.0);
      orc_forces(&w, ps.data(), f.data(), e, terms);
      double t = 0;
      for (int k = 0; k < ORC_NE; ++k) t += e[k];
      u[sgn] = t;
    }
    vir[a] = -(u[0] - u[1]) / (2.0 * h);
  }
}

// kinetic energy of the unit centres
double com_kinetic(const Orc& o, const std::vector<std::vector<int>>& units, const double* vel) {
  double k = 0;
  for (const auto& u : units) {
    double p[3] = {0, 0, 0}, mt = 0;
    for (int i : u) {
      for (int c = 0; c < 3; ++c) p[c] += o.mass[i] * vel[3 * i + c];
      mt += o.mass[i];
    }
    k += 0.5 * dot3(p, p) / mt;
  }
  return k;
}

// scales every unit's centre-of-mass velocity by f
void scale_com(const Orc& o, const std::vector<std::vector<int>>& units, double* vel, double f) {
  for (const auto& u : units) {
    double p[3] = {0, 0, 0}, mt = 0;
    for (int i : u) {
      for (int c = 0; c < 3; ++c) p[c] += o.mass[i] * vel[3 * i + c];
      mt += o.mass[i];
    }
    for (int i : u)
      for (int c = 0; c < 3; ++c) vel[3 * i + c] += (f - 1.0) * p[c] / mt;
  }
}

// instantaneous constraint virial: multipliers keeping d2/dt2 |r_k|^2 = 0 given F and v
void constraint_virial(const Orc& o, const double* pos, const double* vel, const double* f, double* vir) {
  for (const Cluster& cl : o.clusters) {
    double rd[3][3], im[4];
    for (int a = 0; a < cl.na; ++a) im[a] = 1.0 / o.mass[cl.atom[a]];
    double J[3][3] = {}, rhs[3] = {}, lam[3];
    for (int k = 0; k < cl.nc; ++k) {
      const int ga = cl.atom[cl.ca[k]], gb = cl.atom[cl.cb[k]];
      for (int c = 0; c < 3; ++c) rd[k][c] = pos[3 * ga + c] - pos[3 * gb + c];
      minimg(rd[k], o.s.box);
    }
    for (int k = 0; k < cl.nc; ++k) {
      const int a = cl.ca[k], b = cl.cb[k];
      const int ga = cl.atom[a], gb = cl.atom[b];
      double vab[3], aab[3];
      for (int c = 0; c < 3; ++c) {
        vab[c] = vel[3 * ga + c] - vel[3 * gb + c];
        aab[c] = f[3 * ga + c] * im[a] - f[3 * gb + c] * im[b];
      }
      rhs[k] = -dot3(vab, vab) - dot3(rd[k], aab);
      for (int l = 0; l < cl.nc; ++l) {
        double coef = 0;
        if (cl.ca[l] == a) coef += im[a];
        if (cl.cb[l] == a) coef -= im[a];
        if (cl.ca[l] == b) coef -= im[b];
        if (cl.cb[l] == b) coef += im[b];
        J[k][l] = coef * dot3(rd[l], rd[k]);
      }
    }
    if (!gauss_solve(cl.nc, J, rhs, lam)) continue;
    for (int k = 0; k < cl.nc; ++k)
      for (int c = 0; c < 3; ++c) vir[c] += lam[k] * rd[k][c] * rd[k][c];
  }
}

const double kPUo = 1.4586e-5;             // atm -> kcal/mol/A^3 (src/defs.in.h:105)
const double kPatmO = 68558.64100846418;   // kcal/mol/A^3 -> atm (src/cell_based_kernels.cu:584)

}  // namespace

extern "C" {

int orc_virial_fd(void* h, const double* pos, double hrel, int terms, int group, double* vir3) {
  virial_fd(*(Orc*)h, pos, hrel, terms, vir3, group);
  return 0;
}

int orc_constraint_virial(void* h, const double* pos, const double* vel, const double* f, double* vir3) {
  vir3[0] = vir3[1] = vir3[2] = 0.0;
  constraint_virial(*(Orc*)h, pos, vel, f, vir3);
  return 0;
}

double orc_group_pressure(void* h, const double* pos, const double* vel, double hrel) {
  const Orc& o = *(Orc*)h;
  double w[3];
  virial_fd(o, pos, hrel, ORC_T_ALL, w, 1);
  const double V = o.s.box[0] * o.s.box[1] * o.s.box[2];
  return (2.0 * com_kinetic(o, units_of(o), vel) + w[0] + w[1] + w[2]) / (3.0 * V) * kPatmO;
}

int orc_npt(void* h, double* pos, double* vel, double* box3, double* lstate, int nsteps, double dt_ps, double tol,
            double pref_atm, double pmass, double hrel, double* Ltrace, double* Ptrace) {
  Orc w = *(Orc*)h;  // works on a copy whose box follows the piston
  const int n = w.s.n;
  const double dt = dt_ps * ORC_TU;
  for (int d = 0; d < 3; ++d) w.s.box[d] = box3[d];
  const double ratio[3] = {1.0, box3[1] / box3[0], box3[2] / box3[0]};
  double Ldot = lstate[0], Lacc = lstate[1];
  const std::vector<std::vector<int>> units = units_of(w);
  std::vector<double> f(3 * (size_t)n, 0.0), ref(3 * (size_t)n), R(3 * units.size());
  double e[ORC_NE];
  orc_forces(&w, pos, f.data(), e, ORC_T_ALL);
  int bad = 0;
  for (int s = 0; s < nsteps; ++s) {
    const double L = w.s.box[0];
    Ldot += 0.5 * dt * Lacc;
    const double Ln = L + dt * Ldot, lam = Ln / L;
    scale_com(w, units, vel, std::exp(-0.5 * dt * Ldot / L));
    // each atom moves by (lam - 1) x its unit's mass centre taken in the atom's own
    // periodic image, so the unit moves rigidly even when its atoms are wrapped apart
    for (size_t k = 0; k < units.size(); ++k) {
      centre(w, units[k], pos, &R[3 * k]);
      const int a0 = units[k][0];
      for (int i : units[k]) {
        double d[3] = {pos[3 * i] - pos[3 * a0], pos[3 * i + 1] - pos[3 * a0 + 1], pos[3 * i + 2] - pos[3 * a0 + 2]};
        double dm[3] = {d[0], d[1], d[2]};
        minimg(dm, w.s.box);
        for (int c = 0; c < 3; ++c)  // R + (d - dm): the centre's image next to atom i
          ref[3 * i + c] = pos[3 * i + c] + (lam - 1.0) * (R[3 * k + c] + d[c] - dm[c]);
      }
    }
    for (int d = 0; d < 3; ++d) w.s.box[d] = Ln * ratio[d];
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        vel[3 * i + c] += 0.5 * dt * f[3 * i + c] / w.mass[i];
        pos[3 * i + c] = ref[3 * i + c] + dt * vel[3 * i + c];
      }
    for (const Cluster& cl : w.clusters) bad += shake_cluster(w, cl, ref.data(), pos, vel, dt, tol, 1000) != 0;
    const double kc = com_kinetic(w, units, vel);
    std::fill(f.begin(), f.end(), 0.0);
    orc_forces(&w, pos, f.data(), e, ORC_T_ALL);
    double wf[3];
    virial_fd(w, pos, hrel, ORC_T_ALL, wf, 1);
    const double V = w.s.box[0] * w.s.box[1] * w.s.box[2];
    const double P = (2.0 * kc + wf[0] + wf[1] + wf[2]) / (3.0 * V);
    Lacc = (P - pref_atm * kPUo) / (3.0 * pmass * Ln * Ln) - 2.0 * Ldot * Ldot / Ln;
    Ldot += 0.5 * dt * Lacc;
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) vel[3 * i + c] += 0.5 * dt * f[3 * i + c] / w.mass[i];
    scale_com(w, units, vel, std::exp(-0.5 * dt * Ldot / Ln));
    for (const Cluster& cl : w.clusters) rattle_cluster(w, cl, pos, vel);
    if (Ltrace) Ltrace[s] = Ln;
    if (Ptrace) Ptrace[s] = P * kPatmO;
  }
  for (int d = 0; d < 3; ++d) box3[d] = w.s.box[d];
  lstate[0] = Ldot;
  lstate[1] = Lacc;
  return bad;
}

}  // extern "C"
