// Velocity Verlet with SHAKE/RATTLE in AKMA units, fused per integration unit
// (a SHAKE cluster of <= 4 atoms or a free atom).  Replaces HalfKickGPU,
// UpdateCoords, CoordsUpdate (src/mdcuda.cu:27-92, 354-478), solve_bond_constraints /
// solve_velocity_constraints (src/shake.cu:20-615) and the nupdated D2H flag of
// SingleStep (src/dynamics.cu:695-737): the displacement test raises a device flag
// read by the neighbour kernels, so no host synchronisation is needed per step.
// Constraint solves run in FP64 with an iteration cap (the reference loops without one,
// src/shake.cu:195-271) and report non-convergence in the status word.
#include "common.cuh"
#include "kernels.h"

namespace fzk {

struct Unit {
  int na, nc;
  int atom[4];
  int ca[3], cb[3];
  double d[3];
};

__device__ __forceinline__ Unit load_unit(const IntegrateArgs& a, int u) {
  Unit U;
  const int4 at = a.unit_atoms[u];
  const int meta = a.unit_meta[u];
  const float4 dd = a.unit_d[u];
  U.atom[0] = at.x;
  U.atom[1] = at.y;
  U.atom[2] = at.z;
  U.atom[3] = at.w;
  U.na = meta & 15;
  U.nc = (meta >> 4) & 15;
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

__device__ bool gauss3(int n, double J[3][3], double* rhs, double* x) {
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

__device__ __forceinline__ double coef_of(const Unit& U, int k, int l, const double* im) {
  const int a = U.ca[k], b = U.cb[k];
  double c = 0;
  if (U.ca[l] == a) c += im[a];
  if (U.cb[l] == a) c -= im[a];
  if (U.ca[l] == b) c -= im[b];
  if (U.cb[l] == b) c += im[b];
  return c;
}

// SHAKE: Newton iteration on |r_a - r_b + dr_a - dr_b|^2 = d^2 with displacements along
// the reference bond vectors (src/shake.cu:159-271).  rn: unconstrained positions (in/out)
__device__ int shake_unit(const Unit& U, const double rref[4][3], double rn[4][3], const double* im,
                          const SysParams& p, double tol, int maxit) {
  double rd[3][3];
  for (int k = 0; k < U.nc; ++k) {
    for (int c = 0; c < 3; ++c) rd[k][c] = rref[U.ca[k]][c] - rref[U.cb[k]][c];
    min_image_d(rd[k], p);
  }
  double lam[3] = {0, 0, 0};
  int it = 0;
  for (; it < maxit; ++it) {
    double dr[4][3] = {};
    for (int k = 0; k < U.nc; ++k)
      for (int c = 0; c < 3; ++c) {
        dr[U.ca[k]][c] += rd[k][c] * lam[k] * im[U.ca[k]];
        dr[U.cb[k]][c] -= rd[k][c] * lam[k] * im[U.cb[k]];
      }
    double J[3][3], sig[3], dl[3];
    for (int k = 0; k < U.nc; ++k) {
      double C[3];
      for (int c = 0; c < 3; ++c) C[c] = rn[U.ca[k]][c] - rn[U.cb[k]][c];
      min_image_d(C, p);
      for (int c = 0; c < 3; ++c) C[c] += dr[U.ca[k]][c] - dr[U.cb[k]][c];
      sig[k] = C[0] * C[0] + C[1] * C[1] + C[2] * C[2] - U.d[k] * U.d[k];
      for (int l = 0; l < U.nc; ++l)
        J[k][l] = 2.0 * coef_of(U, k, l, im) * (rd[l][0] * C[0] + rd[l][1] * C[1] + rd[l][2] * C[2]);
    }
    if (!gauss3(U.nc, J, sig, dl)) return 2;
    double t = 0;
    for (int k = 0; k < U.nc; ++k) {
      lam[k] -= dl[k];
      t += dl[k] * dl[k];
    }
    if (t < tol) break;
  }
  double dr[4][3] = {};
  for (int k = 0; k < U.nc; ++k)
    for (int c = 0; c < 3; ++c) {
      dr[U.ca[k]][c] += rd[k][c] * lam[k] * im[U.ca[k]];
      dr[U.cb[k]][c] -= rd[k][c] * lam[k] * im[U.cb[k]];
    }
  for (int a = 0; a < U.na; ++a)
    for (int c = 0; c < 3; ++c) rn[a][c] += dr[a][c];
  return it >= maxit ? 1 : 0;
}

// RATTLE velocity stage: (v_a - v_b) . r_ab = 0, linear, solved directly
__device__ void rattle_unit(const Unit& U, const double r[4][3], double v[4][3], const double* im,
                            const SysParams& p) {
  double rd[3][3];
  for (int k = 0; k < U.nc; ++k) {
    for (int c = 0; c < 3; ++c) rd[k][c] = r[U.ca[k]][c] - r[U.cb[k]][c];
    min_image_d(rd[k], p);
  }
  double J[3][3], rhs[3], mu[3];
  for (int k = 0; k < U.nc; ++k) {
    double vab[3];
    for (int c = 0; c < 3; ++c) vab[c] = v[U.ca[k]][c] - v[U.cb[k]][c];
    rhs[k] = vab[0] * rd[k][0] + vab[1] * rd[k][1] + vab[2] * rd[k][2];
    for (int l = 0; l < U.nc; ++l)
      J[k][l] = coef_of(U, k, l, im) * (rd[l][0] * rd[k][0] + rd[l][1] * rd[k][1] + rd[l][2] * rd[k][2]);
  }
  if (!gauss3(U.nc, J, rhs, mu)) return;
  for (int k = 0; k < U.nc; ++k)
    for (int c = 0; c < 3; ++c) {
      v[U.ca[k]][c] -= rd[k][c] * mu[k] * im[U.ca[k]];
      v[U.cb[k]][c] += rd[k][c] * mu[k] * im[U.cb[k]];
    }
}

__global__ void __launch_bounds__(128) k_kick_drift(IntegrateArgs a) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.nunits) return;
  const Unit U = load_unit(a, u);
  const int n = a.p.n;
  double r0[4][3], rn[4][3], v[4][3], im[4];
  float q[4];
  for (int k = 0; k < U.na; ++k) {
    const int i = U.atom[k];
    const float4 pr = a.pos4[i], vl = a.vel4[i];
    const double3 F = force_of(a.facc, n, i);
    a.facc[i] = 0;
    a.facc[n + i] = 0;
    a.facc[2 * n + i] = 0;
    im[k] = vl.w;
    q[k] = pr.w;
    const double h = 0.5 * a.dtu * im[k];
    v[k][0] = vl.x + h * F.x;
    v[k][1] = vl.y + h * F.y;
    v[k][2] = vl.z + h * F.z;
    r0[k][0] = pr.x;
    r0[k][1] = pr.y;
    r0[k][2] = pr.z;
    for (int c = 0; c < 3; ++c) rn[k][c] = r0[k][c] + a.dtu * v[k][c];
  }
  if (U.nc > 0) {
    const int st = shake_unit(U, r0, rn, im, a.p, a.shake_tol, a.shake_maxit);
    if (st) atomicOr(a.status, ST_SHAKE_NOCONV);
    for (int k = 0; k < U.na; ++k)
      for (int c = 0; c < 3; ++c) v[k][c] = (rn[k][c] - r0[k][c]) / a.dtu;  // v += dr/(dt TU)
  }
  bool far = false;
  for (int k = 0; k < U.na; ++k) {
    const int i = U.atom[k];
    const float4 np = make_float4((float)rn[k][0], (float)rn[k][1], (float)rn[k][2], q[k]);
    a.pos4[i] = np;
    a.vel4[i] = make_float4((float)v[k][0], (float)v[k][1], (float)v[k][2], (float)im[k]);
    a.xyzq_s[a.inv_perm[i]] = np;
    const float4 pb = a.pos_build[i];
    const float dx = np.x - pb.x, dy = np.y - pb.y, dz = np.z - pb.z;
    far |= dx * dx + dy * dy + dz * dz > a.p.skin_half2;
  }
  if (far) *a.flag = 1;
}

template <bool KIN>
__global__ void __launch_bounds__(128) k_kick_rattle(IntegrateArgs a, int kick) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0;
  if (u < a.nunits) {
    const Unit U = load_unit(a, u);
    const int n = a.p.n;
    double r[4][3], v[4][3], im[4];
    for (int k = 0; k < U.na; ++k) {
      const int i = U.atom[k];
      const float4 pr = a.pos4[i], vl = a.vel4[i];
      im[k] = vl.w;
      v[k][0] = vl.x;
      v[k][1] = vl.y;
      v[k][2] = vl.z;
      if (kick) {
        const double3 F = force_of(a.facc, n, i);
        const double h = 0.5 * a.dtu * im[k];
        v[k][0] += h * F.x;
        v[k][1] += h * F.y;
        v[k][2] += h * F.z;
      }
      r[k][0] = pr.x;
      r[k][1] = pr.y;
      r[k][2] = pr.z;
    }
    if (U.nc > 0) rattle_unit(U, r, v, im, a.p);
    for (int k = 0; k < U.na; ++k) {
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

__global__ void __launch_bounds__(256) k_kinetic(IntegrateArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0;
  if (i < a.p.n) {
    const float4 v = a.vel4[i];
    if (v.w > 0.f) ke = 0.5 / (double)v.w * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  }
  energy_add(a.energy + EN_KIN, ke);
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
                                                       long long* psum) {
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

__global__ void __launch_bounds__(256) k_reassign_shift(IntegrateArgs a, const long long* psum, double inv_mtot) {
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

__global__ void k_zero_ll(long long* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0;
}

void launch_kick_drift(const IntegrateArgs& a, cudaStream_t st) {
  k_kick_drift<<<(a.nunits + 127) / 128, 128, 0, st>>>(a);
}

void launch_kick_rattle(const IntegrateArgs& a, bool kinetic, bool kick, cudaStream_t st) {
  if (kinetic)
    k_kick_rattle<true><<<(a.nunits + 127) / 128, 128, 0, st>>>(a, kick ? 1 : 0);
  else
    k_kick_rattle<false><<<(a.nunits + 127) / 128, 128, 0, st>>>(a, kick ? 1 : 0);
}

void launch_kinetic(const IntegrateArgs& a, cudaStream_t st) {
  k_kinetic<<<(a.p.n + 255) / 256, 256, 0, st>>>(a);
}

void launch_reassign(const IntegrateArgs& a, double T, uint64_t seed, uint32_t counter, double inv_mtot,
                     long long* psum, cudaStream_t st) {
  k_zero_ll<<<1, 32, 0, st>>>(psum, 3);
  k_reassign_draw<<<(a.p.n + 255) / 256, 256, 0, st>>>(a, T, seed, counter, psum);
  k_reassign_shift<<<(a.p.n + 255) / 256, 256, 0, st>>>(a, psum, inv_mtot);
  k_kick_rattle<false><<<(a.nunits + 127) / 128, 128, 0, st>>>(a, 0);
}

}  // namespace fzk
