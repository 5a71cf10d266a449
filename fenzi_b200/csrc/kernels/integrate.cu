// Velocity Verlet with SHAKE/RATTLE in AKMA units, fused per integration unit
// (a SHAKE cluster of <= 4 atoms or a free atom).  Replaces HalfKickGPU,
// UpdateCoords, CoordsUpdate (src/mdcuda.cu:27-92, 354-478), solve_bond_constraints /
// solve_velocity_constraints (src/shake.cu:20-615) and the nupdated D2H flag of
// SingleStep (src/dynamics.cu:695-737): the displacement test raises a device flag
// read by the neighbour kernels, so no host synchronisation is needed per step.
// Constraint solves run in FP64 with an iteration cap (the reference loops without one,
// src/shake.cu:195-271) and report non-convergence in the status word.
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace fzk {

struct Unit {
  int na, nc;
  int atom[4];
  int ca[3], cb[3];
  double d[3];
};

// NA, NC > 0: the unit's class (atoms, constraints) is known at compile time, so the
// per-atom loops below fold to that size and the unit's arrays stay small in
// registers; NA = 0 reads both from the unit's metadata.
template <int NA, int NC>
__device__ __forceinline__ Unit load_unit(const IntegrateArgs& a, int u) {
  Unit U;
  const int4 at = a.unit_atoms[u];
  const int meta = a.unit_meta[u];
  const float4 dd = a.unit_d[u];
  U.atom[0] = at.x;
  U.atom[1] = at.y;
  U.atom[2] = at.z;
  U.atom[3] = at.w;
  U.na = NA > 0 ? NA : meta & 15;
  U.nc = NA > 0 ? NC : (meta >> 4) & 15;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    U.ca[k] = (meta >> (8 + 4 * k)) & 3;
    U.cb[k] = (meta >> (10 + 4 * k)) & 3;
  }
  U.d[0] = dd.x;
  U.d[1] = dd.y;
  U.d[2] = dd.z;
  return U;
}

__device__ __forceinline__ double3 force_of(const long long* facc, int n, int i) {
  const double s = 1.0 / kFixFd;
  return make_double3((double)facc[i] * s, (double)facc[n + i] * s, (double)facc[2 * n + i] * s);
}

// solves J x = r for n <= 3 (Cramer's rule); false if singular
__device__ __forceinline__ bool solve3(int n, const double J[3][3], const double* r, double* x) {
  if (n == 1) {
    if (J[0][0] == 0.0) return false;
    x[0] = r[0] / J[0][0];
    return true;
  }
  if (n == 2) {
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    if (det == 0.0) return false;
    const double id = 1.0 / det;
    x[0] = (r[0] * J[1][1] - J[0][1] * r[1]) * id;
    x[1] = (J[0][0] * r[1] - r[0] * J[1][0]) * id;
    return true;
  }
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  if (det == 0.0) return false;
  const double id = 1.0 / det;
  x[0] = (r[0] * c00 + J[0][1] * (r[2] * J[1][2] - r[1] * J[2][2]) + J[0][2] * (r[1] * J[2][1] - r[2] * J[1][1])) * id;
  x[1] = (J[0][0] * (r[1] * J[2][2] - r[2] * J[1][2]) + r[0] * c01 + J[0][2] * (r[2] * J[1][0] - r[1] * J[2][0])) * id;
  x[2] = (J[0][0] * (r[2] * J[1][1] - r[1] * J[2][1]) + J[0][1] * (r[1] * J[2][0] - r[2] * J[1][0]) + r[0] * c02) * id;
  return true;
}

__device__ __forceinline__ void minimg3(double* d, const IntegrateArgs& a) {
#pragma unroll
  for (int c = 0; c < 3; ++c) d[c] -= a.box_d[c] * rint(d[c] * a.inv_box_d[c]);
}

// Sign of atom `at` in constraint k: +1 first atom, -1 second, 0 absent.  All cluster
// indexing below runs through compile-time-unrolled loops over (atom, constraint) with
// these selects, so the per-cluster arrays stay in registers.
__device__ __forceinline__ double sgn(const Unit& U, int k, int at) {
  return (U.ca[k] == at ? 1.0 : 0.0) - (U.cb[k] == at ? 1.0 : 0.0);
}

// bond vector of constraint k from per-atom positions x (min-imaged)
__device__ __forceinline__ void bond_vec(const Unit& U, int k, const double x[4][3], double* out,
                                         const IntegrateArgs& a) {
  out[0] = out[1] = out[2] = 0.0;
#pragma unroll
  for (int at = 0; at < 4; ++at) {
    if (at >= U.na) continue;
    const double sg = sgn(U, k, at);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] += sg * x[at][c];
  }
  minimg3(out, a);
}

// c_kl = sum over atoms of sgn(k, at) sgn(l, at) / m_at
__device__ __forceinline__ void coef_matrix(const Unit& U, const double* im, double cf[3][3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      double c = 0.0;
#pragma unroll
      for (int at = 0; at < 4; ++at)
        if (at < U.na) c += sgn(U, k, at) * sgn(U, l, at) * im[at];
      cf[k][l] = c;
    }
}

// SHAKE: Newton iteration on |r_a - r_b + dr_a - dr_b|^2 = d^2 with displacements along
// the reference bond vectors (src/shake.cu:159-271).  With s_k the unconstrained bond
// vector and c_kl the inverse-mass coupling of constraints k and l,
// C_k = s_k + sum_l c_kl lambda_l rd_l.  rn: unconstrained positions (in/out).
__device__ __forceinline__ int shake_unit(const Unit& U, const double rref[4][3], double rn[4][3], const double* im,
                                          const IntegrateArgs& a) {
  double rd[3][3], s0[3][3], cf[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    bond_vec(U, k, rref, rd[k], a);
    bond_vec(U, k, rn, s0[k], a);
  }
  coef_matrix(U, im, cf);
  double lam[3] = {0, 0, 0};
  int it = 0;
  const int nc = U.nc;
  for (; it < a.shake_maxit; ++it) {
    double J[3][3], sig[3], dl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double C[3] = {s0[k][0], s0[k][1], s0[k][2]};
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        const double w = (l < nc) ? cf[k][l] * lam[l] : 0.0;
        C[0] += w * rd[l][0];
        C[1] += w * rd[l][1];
        C[2] += w * rd[l][2];
      }
      sig[k] = C[0] * C[0] + C[1] * C[1] + C[2] * C[2] - U.d[k] * U.d[k];
#pragma unroll
      for (int l = 0; l < 3; ++l) J[k][l] = 2.0 * cf[k][l] * (rd[l][0] * C[0] + rd[l][1] * C[1] + rd[l][2] * C[2]);
    }
    if (!solve3(nc, J, sig, dl)) return 2;
    double t = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (k < nc) {
        lam[k] -= dl[k];
        t += dl[k] * dl[k];
      }
    if (t < a.shake_tol) break;
  }
#pragma unroll
  for (int at = 0; at < 4; ++at)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (at >= U.na) continue;
      const double w = (k < nc) ? sgn(U, k, at) * lam[k] * im[at] : 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) rn[at][c] += w * rd[k][c];
    }
  return it >= a.shake_maxit ? 1 : 0;
}

__device__ __forceinline__ void cross3d(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3d(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void unit3d(double* a) {
  const double s = rsqrt(dot3d(a, a));
  a[0] *= s;
  a[1] *= s;
  a[2] *= s;
}

// SETTLE (Miyamoto and Kollman, J. Comput. Chem. 13, 952 (1992)): the closed-form
// solution of the SHAKE equations for a rigid triangle with an apex (atom 0) and two
// base atoms of equal mass at equal distance from it, constraints ordered (0,1),
// (0,2), (1,2).  The constraint displacements lie in the plane of r(t), so in a frame
// with n0 normal to that plane every atom keeps its n0 coordinate and the triangle
// is placed by three rotations (phi, psi, theta) solved in closed form; the result is
// the converged SHAKE solution without iterations.  Works on offsets from the apex's
// r(t) (min-imaged), so large coordinates do not enter; rn: unconstrained positions
// in, constrained out.  Returns false when the step is too large for a solution.
__device__ __forceinline__ bool settle_unit(const Unit& U, const double rref[4][3], double rn[4][3],
                                            const double* im, const IntegrateArgs& a) {
  const double mA = 1.0 / im[0], mB = 1.0 / im[1];
  const double wA = mA / (mA + 2.0 * mB), wB = mB / (mA + 2.0 * mB);
  const double rc = 0.5 * U.d[2];
  const double h = sqrt(U.d[0] * U.d[0] - rc * rc);
  const double ra = 2.0 * wB * h, rb = h - ra;
  double b0[3], c0[3], a1[3], b1[3], c1[3], D[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    b0[c] = rref[1][c] - rref[0][c];
    c0[c] = rref[2][c] - rref[0][c];
  }
  minimg3(b0, a);
  minimg3(c0, a);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    a1[c] = rn[0][c] - rref[0][c];
    b1[c] = b0[c] + (rn[1][c] - rref[1][c]);
    c1[c] = c0[c] + (rn[2][c] - rref[2][c]);
    D[c] = wA * a1[c] + wB * (b1[c] + c1[c]);
    a1[c] -= D[c];
    b1[c] -= D[c];
    c1[c] -= D[c];
  }
  double n0[3], n1[3], n2[3];
  cross3d(b0, c0, n0);
  cross3d(a1, n0, n1);
  cross3d(n0, n1, n2);
  unit3d(n0);
  unit3d(n1);
  unit3d(n2);
  const double b0x = dot3d(n1, b0), b0y = dot3d(n2, b0), c0x = dot3d(n1, c0), c0y = dot3d(n2, c0);
  const double a1z = dot3d(n0, a1);
  const double b1x = dot3d(n1, b1), b1y = dot3d(n2, b1), b1z = dot3d(n0, b1);
  const double c1x = dot3d(n1, c1), c1y = dot3d(n2, c1), c1z = dot3d(n0, c1);
  const double sinphi = a1z / ra;
  const double cphi2 = 1.0 - sinphi * sinphi;
  if (!(cphi2 > 0.0)) return false;
  const double cosphi = sqrt(cphi2);
  const double sinpsi = (b1z - c1z) / (2.0 * rc * cosphi);
  const double cpsi2 = 1.0 - sinpsi * sinpsi;
  if (!(cpsi2 > 0.0)) return false;
  const double cospsi = sqrt(cpsi2);
  const double ya2 = ra * cosphi, xb2 = -rc * cospsi;
  const double t1 = -rb * cosphi, t2 = rc * sinpsi * sinphi;
  const double yb2 = t1 - t2, yc2 = t1 + t2;
  const double al = xb2 * (b0x - c0x) + b0y * yb2 + c0y * yc2;
  const double be = xb2 * (c0y - b0y) + b0x * yb2 + c0x * yc2;
  const double ga = b0x * b1y - b1x * b0y + c0x * c1y - c1x * c0y;
  const double ab2 = al * al + be * be;
  const double disc = ab2 - ga * ga;
  if (!(disc >= 0.0) || !(ab2 > 0.0)) return false;
  const double sinth = (al * ga - be * sqrt(disc)) / ab2;
  const double costh = sqrt(fmax(0.0, 1.0 - sinth * sinth));
  // final offsets from D in the (n1, n2, n0) frame, minus the r(t) offsets from the apex
  const double p[3][3] = {{-ya2 * sinth, ya2 * costh, a1z},
                          {xb2 * costh - yb2 * sinth, xb2 * sinth + yb2 * costh, b1z},
                          {-xb2 * costh - yc2 * sinth, -xb2 * sinth + yc2 * costh, c1z}};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double x = D[c] + p[k][0] * n1[c] + p[k][1] * n2[c] + p[k][2] * n0[c];
      const double x0 = k == 0 ? 0.0 : (k == 1 ? b0[c] : c0[c]);
      rn[k][c] = rref[k][c] + (x - x0);
    }
  return true;
}

// RATTLE velocity stage: (v_a - v_b) . r_ab = 0, linear, solved directly
__device__ __forceinline__ void rattle_unit(const Unit& U, const double r[4][3], double v[4][3], const double* im,
                                            const IntegrateArgs& a) {
  double rd[3][3], vd[3][3], cf[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    bond_vec(U, k, r, rd[k], a);
    vd[k][0] = vd[k][1] = vd[k][2] = 0.0;
#pragma unroll
    for (int at = 0; at < 4; ++at) {
      if (at >= U.na) continue;
      const double sg = sgn(U, k, at);
#pragma unroll
      for (int c = 0; c < 3; ++c) vd[k][c] += sg * v[at][c];
    }
  }
  coef_matrix(U, im, cf);
  double J[3][3], rhs[3], mu[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    rhs[k] = vd[k][0] * rd[k][0] + vd[k][1] * rd[k][1] + vd[k][2] * rd[k][2];
#pragma unroll
    for (int l = 0; l < 3; ++l) J[k][l] = cf[k][l] * (rd[l][0] * rd[k][0] + rd[l][1] * rd[k][1] + rd[l][2] * rd[k][2]);
  }
  if (!solve3(U.nc, J, rhs, mu)) return;
#pragma unroll
  for (int at = 0; at < 4; ++at)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (at >= U.na) continue;
      const double w = (k < U.nc) ? sgn(U, k, at) * mu[k] * im[at] : 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[at][c] -= w * rd[k][c];
    }
}

// mass centre offset of a unit relative to its atom 0 (min-imaged) and total mass
__device__ __forceinline__ double unit_centre(const Unit& U, const double r[4][3], const double* im, double* cm,
                                              const IntegrateArgs& a) {
  double mt = 0.0;
  cm[0] = cm[1] = cm[2] = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= U.na) continue;
    const double m = im[k] > 0.0 ? 1.0 / im[k] : 0.0;
    double d[3] = {r[k][0] - r[0][0], r[k][1] - r[0][1], r[k][2] - r[0][2]};
    minimg3(d, a);
    for (int c = 0; c < 3; ++c) cm[c] += m * d[c];
    mt += m;
  }
  if (mt > 0.0)
    for (int c = 0; c < 3; ++c) cm[c] /= mt;
  return mt;
}

// scales the unit's centre-of-mass velocity by f (barostat friction on the peculiar
// centre-of-mass motion; internal motion is untouched)
__device__ __forceinline__ void scale_com_velocity(const Unit& U, double v[4][3], const double* im, double f) {
  double p[3] = {0.0, 0.0, 0.0}, mt = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= U.na) continue;
    const double m = im[k] > 0.0 ? 1.0 / im[k] : 0.0;
    for (int c = 0; c < 3; ++c) p[c] += m * v[k][c];
    mt += m;
  }
  if (mt <= 0.0) return;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < U.na)
      for (int c = 0; c < 3; ++c) v[k][c] += (f - 1.0) * p[c] / mt;
}

// v += (dt/2) F / m, one rounding per component (the same in every pass that kicks)
__device__ __forceinline__ void half_kick(double* v, double3 F, double im, const IntegrateArgs& a) {
  const double h = 0.5 * a.dtu * im;
  v[0] = fma(h, F.x, v[0]);
  v[1] = fma(h, F.y, v[1]);
  v[2] = fma(h, F.z, v[2]);
}

// brings a line into L1 ahead of a load that comes after stores the compiler cannot
// move it past (pointers that may alias), so that load does not wait on DRAM
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// NPT (Andersen barostat step with the integration units as scaling groups): the unit
// moves rigidly with its mass centre scaled by a.lam about the origin (the box changed
// by a.lam), and its centre-of-mass velocity is scaled by a.vfric before the kick.
// CLOSE (not with NPT): the unit first finishes the previous step as the kick + RATTLE
// pass does (half kick with the same forces, velocity constraints, velocities rounded
// to the stored float), so one pass replaces the previous step's closing launch and
// this step's opening one with bit-identical results.
template <bool NPT, int NA, int NC, bool SETTLE, bool CLOSE = false>
__device__ __forceinline__ void kick_drift_body(const IntegrateArgs& a, int bid) {
  static_assert(!(NPT && CLOSE), "the closing pass is for constant-volume steps");
  griddep_wait();
  const int u = a.u_begin + bid * blockDim.x + threadIdx.x;
  if (u >= a.u_end) return;
  const Unit U = load_unit<NA, NC>(a, u);
  const int n = a.p.n;
  double r0[4][3], rn[4][3], v[4][3], im[4];
  double3 F[4];
  float q[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    im[k] = 0.0;
    q[k] = 0.f;
    F[k] = make_double3(0.0, 0.0, 0.0);
    for (int c = 0; c < 3; ++c) r0[k][c] = rn[k][c] = v[k][c] = 0.0;
    if (k < U.na) {
      const int i = U.atom[k];
      const float4 pr = a.pos4[i], vl = a.vel4[i];
      F[k] = force_of(a.facc, n, i);
      prefetch_l1(a.pos_build + i);
      prefetch_l1(a.pos_prune + i);
      prefetch_l1(a.inv_perm + i);
      im[k] = vl.w;
      q[k] = pr.w;
      v[k][0] = vl.x;
      v[k][1] = vl.y;
      v[k][2] = vl.z;
      r0[k][0] = pr.x;
      r0[k][1] = pr.y;
      r0[k][2] = pr.z;
    }
  }
  if (CLOSE) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < U.na) half_kick(v[k], F[k], im[k], a);
    if (U.nc > 0) rattle_unit(U, r0, v, im, a);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) v[k][c] = (double)(float)v[k][c];
  }
  if (NPT) scale_com_velocity(U, v, im, a.vfric);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= U.na) continue;
    const int i = U.atom[k];
    a.facc[i] = 0;
    a.facc[n + i] = 0;
    a.facc[2 * n + i] = 0;
    half_kick(v[k], F[k], im[k], a);
  }
  if (NPT) {
    // Each atom moves by (lam - 1) x the unit's mass centre taken in the atom's own
    // periodic image (atoms of a unit can sit on opposite sides of the box after the
    // rebuild wraps them), so every min-imaged intra-unit vector is unchanged in the
    // new box and the unit moves rigidly.  Offsets are min-imaged in the old box
    // (a.box_d / a.lam), the frame the positions are in.
    double d[4][3], cm[3] = {0.0, 0.0, 0.0}, mt = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      for (int c = 0; c < 3; ++c) {
        const double L0 = a.box_d[c] / a.lam;
        const double x = r0[k][c] - r0[0][c];
        d[k][c] = x - L0 * rint(x / L0);
      }
      if (k < U.na && im[k] > 0.0) {
        for (int c = 0; c < 3; ++c) cm[c] += d[k][c] / im[k];
        mt += 1.0 / im[k];
      }
    }
    if (mt > 0.0)
      for (int c = 0; c < 3; ++c) cm[c] /= mt;
    const double s = a.lam - 1.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < U.na)
        for (int c = 0; c < 3; ++c) r0[k][c] += s * (r0[k][c] - d[k][c] + cm[c]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) rn[k][c] = r0[k][c] + a.dtu * v[k][c];
  if (U.nc > 0) {
    int st;
    if constexpr (SETTLE) st = settle_unit(U, r0, rn, im, a) ? 0 : 1;
    else st = shake_unit(U, r0, rn, im, a);
    if (st) atomicOr(a.status, ST_SHAKE_NOCONV);
    const double idt = 1.0 / a.dtu;
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) v[k][c] = (rn[k][c] - r0[k][c]) * idt;  // v += dr/(dt TU)
  }
  bool far = false, moved = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= U.na) continue;
    const int i = U.atom[k];
    const float4 np = make_float4((float)rn[k][0], (float)rn[k][1], (float)rn[k][2], q[k]);
    a.pos4[i] = np;
    a.vel4[i] = make_float4((float)v[k][0], (float)v[k][1], (float)v[k][2], (float)im[k]);
    a.xyzq_s[a.inv_perm[i]] = np;
    const float4 pb = a.pos_build[i];
    const float dx = np.x - pb.x, dy = np.y - pb.y, dz = np.z - pb.z;
    far |= dx * dx + dy * dy + dz * dz > a.p.skin_half2;
    const float4 pp = a.pos_prune[i];
    const float ex = np.x - pp.x, ey = np.y - pp.y, ez = np.z - pp.z;
    moved |= ex * ex + ey * ey + ez * ez > a.prune_half2;
  }
  // one store per warp: on a step where many atoms cross the threshold, per-thread
  // stores to the same word would queue at one L2 slice
  const unsigned am = __activemask();
  const bool lead = (threadIdx.x & 31) == __ffs(am) - 1;
  if (__any_sync(am, far) && lead) *a.flag = 1;
  if (__any_sync(am, moved) && lead) *a.flag_prune = 1;
}

template <bool NPT, int NA, int NC, bool SETTLE = false>
__global__ void __launch_bounds__(128) k_kick_drift(IntegrateArgs a) { griddep_wait(); kick_drift_body<NPT, NA, NC, SETTLE>(a, blockIdx.x); }

template <int NA, int NC, bool SETTLE>
__global__ void __launch_bounds__(128, SETTLE ? 4 : 1) k_close_kick_drift(IntegrateArgs a) {
  griddep_wait();
  kick_drift_body<false, NA, NC, SETTLE, true>(a, blockIdx.x);
}

template <int NA, int NC, bool SETTLE>
__global__ void __launch_bounds__(128, SETTLE ? 4 : 1) k_close_kick_drift_b(const IntegrateArgs* __restrict__ args,
                                                                           const int4* __restrict__ tab) {
  griddep_wait();
  const int4 t = tab[blockIdx.x];
  const IntegrateArgs a = args[t.x];
  kick_drift_body<false, NA, NC, SETTLE, true>(a, t.y);
}

template <int NA, int NC, bool SETTLE>
__global__ void __launch_bounds__(128) k_kick_drift_b(const IntegrateArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const IntegrateArgs a = args[t.x];
  kick_drift_body<false, NA, NC, SETTLE>(a, t.y);
}

// Group (unit) virial terms of a barostat step, after the forces: the centre-of-mass
// kinetic energy of the half-step velocities into EN_KIN_HALF and, into the virial
// slots, minus the intra-unit part sum_a (r_a - R_unit) . F_a, which turns the atomic
// force virial into the virial of the unit centres (constraint forces are internal to
// a unit and drop out).
template <int NA, int NC>
__global__ void __launch_bounds__(128) k_unit_virial(IntegrateArgs a) { griddep_wait();
  const int u = a.u_begin + blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0, vir[3] = {0.0, 0.0, 0.0};
  if (u < a.u_end) {
    const Unit U = load_unit<NA, NC>(a, u);
    const int n = a.p.n;
    double r[4][3], im[4], p[3] = {0.0, 0.0, 0.0}, mt = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      im[k] = 0.0;
      for (int c = 0; c < 3; ++c) r[k][c] = 0.0;
      if (k >= U.na) continue;
      const int i = U.atom[k];
      const float4 pr = a.pos4[i], vl = a.vel4[i];
      im[k] = vl.w;
      r[k][0] = pr.x;
      r[k][1] = pr.y;
      r[k][2] = pr.z;
      const double m = im[k] > 0.0 ? 1.0 / im[k] : 0.0;
      p[0] += m * vl.x;
      p[1] += m * vl.y;
      p[2] += m * vl.z;
      mt += m;
    }
    if (mt > 0.0) ke = 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / mt;
    if (U.na > 1) {
      double cm[3];
      unit_centre(U, r, im, cm, a);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k >= U.na) continue;
        const double3 F = force_of(a.facc, n, U.atom[k]);
        double d[3] = {r[k][0] - r[0][0], r[k][1] - r[0][1], r[k][2] - r[0][2]};
        minimg3(d, a);
        vir[0] -= (d[0] - cm[0]) * F.x;
        vir[1] -= (d[1] - cm[1]) * F.y;
        vir[2] -= (d[2] - cm[2]) * F.z;
      }
    }
  }
  energy_add(a.energy + EN_KIN_HALF, ke);
  energy_add(a.energy + EN_VIR_X, vir[0]);
  energy_add(a.energy + EN_VIR_Y, vir[1]);
  energy_add(a.energy + EN_VIR_Z, vir[2]);
}

template <bool KIN, int NA, int NC>
__device__ __forceinline__ void kick_rattle_body(const IntegrateArgs& a, int kick, int bid) {
  griddep_wait();
  const int u = a.u_begin + bid * blockDim.x + threadIdx.x;
  double ke = 0.0;
  if (u < a.u_end) {
    const Unit U = load_unit<NA, NC>(a, u);
    const int n = a.p.n;
    double r[4][3], v[4][3], im[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      im[k] = 0.0;
      for (int c = 0; c < 3; ++c) r[k][c] = v[k][c] = 0.0;
      if (k >= U.na) continue;
      const int i = U.atom[k];
      const float4 pr = a.pos4[i], vl = a.vel4[i];
      im[k] = vl.w;
      v[k][0] = vl.x;
      v[k][1] = vl.y;
      v[k][2] = vl.z;
      if (kick) half_kick(v[k], force_of(a.facc, n, i), im[k], a);
      r[k][0] = pr.x;
      r[k][1] = pr.y;
      r[k][2] = pr.z;
    }
    if (kick && a.vfric != 1.0) scale_com_velocity(U, v, im, a.vfric);
    if (U.nc > 0) rattle_unit(U, r, v, im, a);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= U.na) continue;
      const int i = U.atom[k];
      a.vel4[i] = make_float4((float)v[k][0], (float)v[k][1], (float)v[k][2], (float)im[k]);
      if (KIN && im[k] > 0.0) {
        const double vx = (float)v[k][0], vy = (float)v[k][1], vz = (float)v[k][2];
        ke += 0.5 / im[k] * (vx * vx + vy * vy + vz * vz);
      }
    }
  }
  if (KIN) energy_add(a.energy + EN_KIN, ke);
}

template <bool KIN, int NA, int NC>
__global__ void __launch_bounds__(128) k_kick_rattle(IntegrateArgs a, int kick) { griddep_wait(); kick_rattle_body<KIN, NA, NC>(a, kick, blockIdx.x); }

template <int NA, int NC>
__global__ void __launch_bounds__(128) k_kick_rattle_b(const IntegrateArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const IntegrateArgs a = args[t.x];
  kick_rattle_body<false, NA, NC>(a, 1, t.y);
}

__global__ void __launch_bounds__(256) k_kinetic(IntegrateArgs a) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0;
  if (i < a.p.n) {
    const float4 v = a.vel4[i];
    if (v.w > 0.f) ke = 0.5 / (double)v.w * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  }
  energy_add(a.energy + EN_KIN, ke);
}

// Instantaneous constraint virial of the current state: the multipliers that keep the
// second time derivative of every constraint length at zero given the forces F and the
// velocities v, sum_l c_kl (r_k . r_l) lambda_l = -|v_k|^2 - r_k . (sum_a sgn_ka F_a / m_a),
// give constraint forces G_a = sum_l sgn_la lambda_l r_l and the virial
// sum_l lambda_l r_l (x) r_l (diagonal), added to the virial slots.
template <int NA, int NC>
__global__ void __launch_bounds__(128) k_constraint_virial(IntegrateArgs a) { griddep_wait();
  const int u = a.u_begin + blockIdx.x * blockDim.x + threadIdx.x;
  double vir[3] = {0.0, 0.0, 0.0};
  if (u < a.u_end) {
    const Unit U = load_unit<NA, NC>(a, u);
    if (U.nc > 0) {
      const int n = a.p.n;
      double r[4][3], v[4][3], f[4][3], im[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        im[k] = 0.0;
        for (int c = 0; c < 3; ++c) r[k][c] = v[k][c] = f[k][c] = 0.0;
        if (k >= U.na) continue;
        const int i = U.atom[k];
        const float4 pr = a.pos4[i], vl = a.vel4[i];
        const double3 F = force_of(a.facc, n, i);
        im[k] = vl.w;
        r[k][0] = pr.x;
        r[k][1] = pr.y;
        r[k][2] = pr.z;
        v[k][0] = vl.x;
        v[k][1] = vl.y;
        v[k][2] = vl.z;
        f[k][0] = F.x * im[k];
        f[k][1] = F.y * im[k];
        f[k][2] = F.z * im[k];
      }
      double rd[3][3], vd[3][3], ad[3][3], cf[3][3], J[3][3], rhs[3], lam[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        bond_vec(U, k, r, rd[k], a);
        for (int c = 0; c < 3; ++c) vd[k][c] = ad[k][c] = 0.0;
#pragma unroll
        for (int at = 0; at < 4; ++at) {
          const double sg = sgn(U, k, at);
          for (int c = 0; c < 3; ++c) {
            vd[k][c] += sg * v[at][c];
            ad[k][c] += sg * f[at][c];
          }
        }
      }
      coef_matrix(U, im, cf);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        rhs[k] = -(vd[k][0] * vd[k][0] + vd[k][1] * vd[k][1] + vd[k][2] * vd[k][2]) -
                 (rd[k][0] * ad[k][0] + rd[k][1] * ad[k][1] + rd[k][2] * ad[k][2]);
#pragma unroll
        for (int l = 0; l < 3; ++l)
          J[k][l] = cf[k][l] * (rd[l][0] * rd[k][0] + rd[l][1] * rd[k][1] + rd[l][2] * rd[k][2]);
      }
      if (solve3(U.nc, J, rhs, lam)) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (k < U.nc)
            for (int c = 0; c < 3; ++c) vir[c] += lam[k] * rd[k][c] * rd[k][c];
      }
    }
  }
  energy_add(a.energy + EN_VIR_X, vir[0]);
  energy_add(a.energy + EN_VIR_Y, vir[1]);
  energy_add(a.energy + EN_VIR_Z, vir[2]);
}

// Minimiser move of one unit: ConjugatedGradient / SteepestDescent (src/mdcuda.cu:126-351).
// Conjugate gradient, per atom as the reference: gamma = |F|^2 / |F_prev|^2 (F_prev = F
// when |F_prev|^2 < 1e-8), direction H = (F + gamma H_prev) x fac; steepest descent:
// step F x fac.  Unlike the reference, which moves constrained atoms freely, SHAKE then
// puts the unit back on its constraints (the old positions as reference vectors), so
// minimised rigid waters stay rigid.  Velocities are zeroed as in the reference.
template <int NA, int NC>
__global__ void __launch_bounds__(128) k_min_step(IntegrateArgs a) { griddep_wait();
  const int u = a.u_begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.u_end) return;
  const Unit U = load_unit<NA, NC>(a, u);
  const int n = a.p.n;
  double r0[4][3], rn[4][3], im[4];
  float q[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    im[k] = 0.0;
    q[k] = 0.f;
    for (int c = 0; c < 3; ++c) r0[k][c] = rn[k][c] = 0.0;
    if (k >= U.na) continue;
    const int i = U.atom[k];
    const float4 pr = a.pos4[i];
    im[k] = a.vel4[i].w;
    q[k] = pr.w;
    r0[k][0] = pr.x;
    r0[k][1] = pr.y;
    r0[k][2] = pr.z;
    const double3 F = force_of(a.facc, n, i);
    a.facc[i] = 0;
    a.facc[n + i] = 0;
    a.facc[2 * n + i] = 0;
    float3 step;
    if (a.min_method == 1) {
      float4 f1 = a.min_prev_f[i];
      const float3 f = make_float3((float)F.x, (float)F.y, (float)F.z);
      const float ff = f.x * f.x + f.y * f.y + f.z * f.z;
      float f11 = f1.x * f1.x + f1.y * f1.y + f1.z * f1.z;
      if (f11 < 1e-8f) f11 = ff;
      const float gamma = f11 > 0.f ? ff / f11 : 0.f;
      const float4 h0 = a.min_dir[i];
      step = make_float3((f.x + h0.x * gamma) * a.min_fac, (f.y + h0.y * gamma) * a.min_fac,
                         (f.z + h0.z * gamma) * a.min_fac);
      a.min_dir[i] = make_float4(step.x, step.y, step.z, 0.f);
      a.min_prev_f[i] = make_float4(f.x, f.y, f.z, 0.f);
    } else {
      step = make_float3((float)F.x * a.min_fac, (float)F.y * a.min_fac, (float)F.z * a.min_fac);
    }
    if (im[k] == 0.0) step = make_float3(0.f, 0.f, 0.f);  // fixed (consfix) atom
    rn[k][0] = r0[k][0] + step.x;
    rn[k][1] = r0[k][1] + step.y;
    rn[k][2] = r0[k][2] + step.z;
  }
  if (U.nc > 0 && shake_unit(U, r0, rn, im, a)) atomicOr(a.status, ST_SHAKE_NOCONV);
  bool far = false, moved = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= U.na) continue;
    const int i = U.atom[k];
    const float4 np = make_float4((float)rn[k][0], (float)rn[k][1], (float)rn[k][2], q[k]);
    a.pos4[i] = np;
    a.vel4[i] = make_float4(0.f, 0.f, 0.f, (float)im[k]);
    a.xyzq_s[a.inv_perm[i]] = np;
    const float4 pb = a.pos_build[i];
    const float dx = np.x - pb.x, dy = np.y - pb.y, dz = np.z - pb.z;
    far |= dx * dx + dy * dy + dz * dz > a.p.skin_half2;
    const float4 pp = a.pos_prune[i];
    const float ex = np.x - pp.x, ey = np.y - pp.y, ez = np.z - pp.z;
    moved |= ex * ex + ey * ey + ez * ez > a.prune_half2;
  }
  // one store per warp: on a step where many atoms cross the threshold, per-thread
  // stores to the same word would queue at one L2 slice
  const unsigned am = __activemask();
  const bool lead = (threadIdx.x & 31) == __ffs(am) - 1;
  if (__any_sync(am, far) && lead) *a.flag = 1;
  if (__any_sync(am, moved) && lead) *a.flag_prune = 1;
}

// ---------------------------------------------------------------- velocity reassignment
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t r) { return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

constexpr double kFixP = 1099511627776.0;  // momentum sums, 2^40

__global__ void __launch_bounds__(256) k_reassign_draw(IntegrateArgs a, double T, uint64_t seed, uint32_t counter,
                                                       long long* psum) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double px = 0, py = 0, pz = 0;
  if (i < a.p.n) {
    const uint64_t z = splitmix64(seed ^ (0xD1B54A32D192ED03ULL * ((uint64_t)counter + 1)));
    const uint64_t base = z + 4ULL * (uint64_t)i;
    const double u1 = u01(splitmix64(base)), u2 = u01(splitmix64(base + 1));
    const double u3 = u01(splitmix64(base + 2)), u4 = u01(splitmix64(base + 3));
    const double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
    const double n0 = r1 * cos(2.0 * kPi * u2), n1 = r1 * sin(2.0 * kPi * u2), n2 = r2 * cos(2.0 * kPi * u4);
    const float4 v = a.vel4[i];
    const double im = v.w;
    const double sd = im > 0 ? sqrt(kRC * T * im) : 0.0;
    const double vx = n0 * sd, vy = n1 * sd, vz = n2 * sd;
    a.vel4[i] = make_float4((float)vx, (float)vy, (float)vz, v.w);
    if (im > 0) {
      px = vx / im;
      py = vy / im;
      pz = vz / im;
    }
  }
  px = warp_sum_d(px);
  py = warp_sum_d(py);
  pz = warp_sum_d(pz);
  if ((threadIdx.x & 31) == 0) {
    red_add(psum + 0, __double2ll_rn(px * kFixP));
    red_add(psum + 1, __double2ll_rn(py * kFixP));
    red_add(psum + 2, __double2ll_rn(pz * kFixP));
  }
}

__global__ void __launch_bounds__(256) k_reassign_shift(IntegrateArgs a, const long long* psum, double inv_mtot) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.p.n) return;
  const double s = inv_mtot / kFixP;
  float4 v = a.vel4[i];
  if (v.w > 0.f) {
    v.x = (float)((double)v.x - (double)psum[0] * s);
    v.y = (float)((double)v.y - (double)psum[1] * s);
    v.z = (float)((double)v.z - (double)psum[2] * s);
  }
  a.vel4[i] = v;
}

__global__ void k_zero_ll(long long* p, int n) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0;
}

template <int V>
using IC = std::integral_constant<int, V>;

// Runs f(args over one unit class, IC<NA>, IC<NC>) for every non-empty unit class,
// with the compile-time specialisations free atom (1, 0), (2, 1), (3, 2), (3, 3) and
// (4, 3), and the runtime form (0, 0) for any other class.
template <class F>
void for_classes(const IntegrateArgs& a0, F f) {
  for (int c = 0; c < a0.ncls; ++c) {
    IntegrateArgs a = a0;
    a.u_begin = a0.cls_begin[c];
    a.u_end = a0.cls_begin[c + 1];
    if (a.u_end <= a.u_begin) continue;
    const int na = a0.cls_na[c], nc = a0.cls_nc[c];
    if (na == 1 && nc == 0)
      f(a, IC<1>(), IC<0>());
    else if (na == 2 && nc == 1)
      f(a, IC<2>(), IC<1>());
    else if (na == 3 && nc == 2)
      f(a, IC<3>(), IC<2>());
    else if (na == 3 && nc == 3)
      f(a, IC<3>(), IC<3>());
    else if (na == 4 && nc == 3)
      f(a, IC<4>(), IC<3>());
    else
      f(a, IC<0>(), IC<0>());
  }
}

static int unit_grid(const IntegrateArgs& a) { return (a.u_end - a.u_begin + 127) / 128; }

// (3, 3) units go to the SETTLE instantiation when every one of them is a symmetric
// triangle (a.settle), which keeps its registers apart from the Newton solver's
template <bool NPT>
static void kick_drift_classes(const IntegrateArgs& a, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    constexpr int NA = decltype(na)::value, NC = decltype(nc)::value;
    if constexpr (NA == 3 && NC == 3) {
      if (x.settle) {
        launch_pdl(k_kick_drift<NPT, 3, 3, true>, dim3(unit_grid(x)), dim3(128), 0, st, x);
        return;
      }
    }
    launch_pdl(k_kick_drift<NPT, NA, NC>, dim3(unit_grid(x)), dim3(128), 0, st, x);
  });
}

void launch_kick_drift(const IntegrateArgs& a, cudaStream_t st) { kick_drift_classes<false>(a, st); }

void launch_close_kick_drift(const IntegrateArgs& a, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    constexpr int NA = decltype(na)::value, NC = decltype(nc)::value;
    if constexpr (NA == 3 && NC == 3) {
      if (x.settle) {
        launch_pdl(k_close_kick_drift<3, 3, true>, dim3(unit_grid(x)), dim3(128), 0, st, x);
        return;
      }
    }
    launch_pdl(k_close_kick_drift<NA, NC, false>, dim3(unit_grid(x)), dim3(128), 0, st, x);
  });
}

// batched: one launch per unit class over every system's units of that class
template <class F>
static void class_dispatch(int na, int nc, F f) {
  if (na == 1 && nc == 0) f(IC<1>(), IC<0>());
  else if (na == 2 && nc == 1) f(IC<2>(), IC<1>());
  else if (na == 3 && nc == 2) f(IC<3>(), IC<2>());
  else if (na == 3 && nc == 3) f(IC<3>(), IC<3>());
  else if (na == 4 && nc == 3) f(IC<4>(), IC<3>());
  else f(IC<0>(), IC<0>());
}

void launch_kick_drift_b(const ClassBatch& c, cudaStream_t st) {
  if (c.nblocks <= 0) return;
  class_dispatch(c.na, c.nc, [&](auto na, auto nc) {
    constexpr int NA = decltype(na)::value, NC = decltype(nc)::value;
    if constexpr (NA == 3 && NC == 3) {
      if (c.settle) {
        launch_pdl(k_kick_drift_b<3, 3, true>, dim3(c.nblocks), dim3(128), 0, st, c.args, c.tab);
        return;
      }
    }
    launch_pdl(k_kick_drift_b<NA, NC, false>, dim3(c.nblocks), dim3(128), 0, st, c.args, c.tab);
  });
}

void launch_close_kick_drift_b(const ClassBatch& c, cudaStream_t st) {
  if (c.nblocks <= 0) return;
  class_dispatch(c.na, c.nc, [&](auto na, auto nc) {
    constexpr int NA = decltype(na)::value, NC = decltype(nc)::value;
    if constexpr (NA == 3 && NC == 3) {
      if (c.settle) {
        launch_pdl(k_close_kick_drift_b<3, 3, true>, dim3(c.nblocks), dim3(128), 0, st, c.args, c.tab);
        return;
      }
    }
    launch_pdl(k_close_kick_drift_b<NA, NC, false>, dim3(c.nblocks), dim3(128), 0, st, c.args, c.tab);
  });
}

void launch_kick_rattle_b(const ClassBatch& c, cudaStream_t st) {
  if (c.nblocks <= 0) return;
  class_dispatch(c.na, c.nc, [&](auto na, auto nc) {
    k_kick_rattle_b<decltype(na)::value, decltype(nc)::value><<<c.nblocks, 128, 0, st>>>(c.args, c.tab);
  });
}

void launch_kick_drift_npt(const IntegrateArgs& a, cudaStream_t st) { kick_drift_classes<true>(a, st); }

void launch_unit_virial(const IntegrateArgs& a, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    k_unit_virial<decltype(na)::value, decltype(nc)::value><<<unit_grid(x), 128, 0, st>>>(x);
  });
}

void launch_constraint_virial(const IntegrateArgs& a, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    k_constraint_virial<decltype(na)::value, decltype(nc)::value><<<unit_grid(x), 128, 0, st>>>(x);
  });
}

void launch_kick_rattle(const IntegrateArgs& a, bool kinetic, bool kick, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    constexpr int NA = decltype(na)::value, NC = decltype(nc)::value;
    if (kinetic)
      launch_pdl(k_kick_rattle<true, NA, NC>, dim3(unit_grid(x)), dim3(128), 0, st, x, kick ? 1 : 0);
    else
      launch_pdl(k_kick_rattle<false, NA, NC>, dim3(unit_grid(x)), dim3(128), 0, st, x, kick ? 1 : 0);
  });
}

void launch_min_step(const IntegrateArgs& a, cudaStream_t st) {
  for_classes(a, [&](const IntegrateArgs& x, auto na, auto nc) {
    k_min_step<decltype(na)::value, decltype(nc)::value><<<unit_grid(x), 128, 0, st>>>(x);
  });
}

void launch_kinetic(const IntegrateArgs& a, cudaStream_t st) {
  launch_pdl(k_kinetic, dim3((a.p.n + 255) / 256), dim3(256), 0, st, a);
}

void launch_reassign(const IntegrateArgs& a, double T, uint64_t seed, uint32_t counter, double inv_mtot,
                     long long* psum, cudaStream_t st) {
  launch_pdl(k_zero_ll, dim3(1), dim3(32), 0, st, psum, 3);
  launch_pdl(k_reassign_draw, dim3((a.p.n + 255) / 256), dim3(256), 0, st, a, T, seed, counter, psum);
  launch_pdl(k_reassign_shift, dim3((a.p.n + 255) / 256), dim3(256), 0, st, a, psum, inv_mtot);
  launch_kick_rattle(a, false, false, st);
}

}  // namespace fzk
