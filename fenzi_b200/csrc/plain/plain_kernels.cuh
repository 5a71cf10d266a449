// Kernels of the plain comparator path (fenzi_plain.h), templated on the arithmetic
// type: T = float is the reference's precision, T = double the all-FP64 variant.
// Every stage is one launch with one thread per atom, term, cluster or grid point,
// as in the reference's kernels cited beside each one.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

namespace fzp {

template <class T> struct Vec;
template <> struct Vec<float> {
  using v4 = float4;
  using cplx = cufftComplex;
};
template <> struct Vec<double> {
  using v4 = double4;
  using cplx = cufftDoubleComplex;
};

__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_rint(float x) { return rintf(x); }
__device__ __forceinline__ double m_rint(double x) { return rint(x); }
__device__ __forceinline__ float m_floor(float x) { return floorf(x); }
__device__ __forceinline__ double m_floor(double x) { return floor(x); }
__device__ __forceinline__ float m_erfc(float x) { return erfcf(x); }
__device__ __forceinline__ double m_erfc(double x) { return erfc(x); }
__device__ __forceinline__ float m_erf(float x) { return erff(x); }
__device__ __forceinline__ double m_erf(double x) { return erf(x); }
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_atan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double m_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float m_cos(float x) { return cosf(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ float m_sin(float x) { return sinf(x); }
__device__ __forceinline__ double m_sin(double x) { return sin(x); }

// status bits
enum : int { PS_CELL_OVF = 1, PS_LIST_OVF = 2, PS_LATTICE_OVF = 4, PS_SHAKE = 8, PS_BAD_COORD = 16 };

// energy accumulator slots (double, on the device)
enum : int { PE_BOND, PE_ANGLE, PE_UREYB, PE_DIHED, PE_IMPR, PE_VDW, PE_ELEC, PE_PME, PE_EWEXCL, PE_KIN2, PE_N };

template <class T> struct Prm {
  int n, nt;
  T L[3], iL[3];
  T rc2, ron2, rl2, beta, cc, sw_c3;
  int K[3];
  int nc[3], cell_cap, maxnb;
};

template <class T> __device__ __forceinline__ void min_image(const Prm<T>& p, T& dx, T& dy, T& dz) {
  dx -= p.L[0] * m_rint(dx * p.iL[0]);
  dy -= p.L[1] * m_rint(dy * p.iL[1]);
  dz -= p.L[2] * m_rint(dz * p.iL[2]);
}

template <class T> __device__ __forceinline__ int cell_coord(const Prm<T>& p, T x, int d) {
  int c = (int)m_floor((x * p.iL[d] + T(0.5)) * (T)p.nc[d]);
  return c < 0 ? 0 : (c >= p.nc[d] ? p.nc[d] - 1 : c);
}

// positions wrapped into [-L/2, L/2), the build positions recorded, atoms binned into
// cells of edge >= pairlistdist (CellBuild, src/cell_based_kernels.cu:198-290)
template <class T>
__global__ void k_cells(Prm<T> p, typename Vec<T>::v4* pos, typename Vec<T>::v4* pos_build, int* cell_n,
                        int* cell_atoms, int* status) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= p.n) return;
  typename Vec<T>::v4 r = pos[a];
  if (!(fabs((double)r.x) < 1e7 && fabs((double)r.y) < 1e7 && fabs((double)r.z) < 1e7)) {
    atomicOr(status, PS_BAD_COORD);
    r.x = r.y = r.z = 0;
  }
  r.x -= p.L[0] * m_floor(r.x * p.iL[0] + T(0.5));
  r.y -= p.L[1] * m_floor(r.y * p.iL[1] + T(0.5));
  r.z -= p.L[2] * m_floor(r.z * p.iL[2] + T(0.5));
  pos[a] = r;
  pos_build[a] = r;
  const int c = (cell_coord(p, r.x, 0) * p.nc[1] + cell_coord(p, r.y, 1)) * p.nc[2] + cell_coord(p, r.z, 2);
  const int k = atomicAdd(&cell_n[c], 1);
  if (k < p.cell_cap) cell_atoms[(size_t)c * p.cell_cap + k] = a;
  else atomicOr(status, PS_CELL_OVF);
}

__device__ __forceinline__ bool is_excluded(const int* __restrict__ off, const int* __restrict__ idx, int i, int j) {
  int lo = off[i], hi = off[i + 1];
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    const int v = idx[m];
    if (v == j) return true;
    if (v < j) lo = m + 1;
    else hi = m;
  }
  return false;
}

// distinct neighbour cells along one dimension (1, 2 or 3 of them)
__device__ __forceinline__ int cell_range(int c, int nc, int* out) {
  if (nc == 1) {
    out[0] = 0;
    return 1;
  }
  if (nc == 2) {
    out[0] = 0;
    out[1] = 1;
    return 2;
  }
  out[0] = (c + nc - 1) % nc;
  out[1] = c;
  out[2] = (c + 1) % nc;
  return 3;
}

// per-atom full neighbour list, 27-cell search, excluded pairs (1-2, 1-3, 1-4) left
// out; stored transposed (entry k of atom i at k * n + i) as the reference's list
// (nbbuild_excllist, src/cell_based_kernels.cu:1259-1493)
template <class T>
__global__ void k_nblist(Prm<T> p, const typename Vec<T>::v4* __restrict__ pos, const int* __restrict__ cell_n,
                         const int* __restrict__ cell_atoms, const int* __restrict__ excl_off,
                         const int* __restrict__ excl_idx, int* nbl, int* nbn, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const typename Vec<T>::v4 ri = pos[i];
  int cx[3], cy[3], cz[3];
  const int nx = cell_range(cell_coord(p, ri.x, 0), p.nc[0], cx);
  const int ny = cell_range(cell_coord(p, ri.y, 1), p.nc[1], cy);
  const int nz = cell_range(cell_coord(p, ri.z, 2), p.nc[2], cz);
  int k = 0;
  for (int a = 0; a < nx; ++a)
    for (int b = 0; b < ny; ++b)
      for (int c = 0; c < nz; ++c) {
        const int cell = (cx[a] * p.nc[1] + cy[b]) * p.nc[2] + cz[c];
        const int m = min(cell_n[cell], p.cell_cap);
        const int* at = cell_atoms + (size_t)cell * p.cell_cap;
        for (int q = 0; q < m; ++q) {
          const int j = at[q];
          if (j == i) continue;
          const typename Vec<T>::v4 rj = pos[j];
          T dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - rj.z;
          min_image(p, dx, dy, dz);
          if (dx * dx + dy * dy + dz * dz >= p.rl2) continue;
          if (is_excluded(excl_off, excl_idx, i, j)) continue;
          if (k < p.maxnb) nbl[(size_t)k * p.n + i] = j;
          ++k;
        }
      }
  nbn[i] = k;
  if (k > p.maxnb) atomicOr(status, PS_LIST_OVF);
}

// CHARMM switch for r > ron: sw = (rc2-r2)^2 (rc2+2r2-3ron2)/(rc2-ron2)^3 and
// dsw = -(d sw/dr)/r (src/mem.cu:556-566)
template <class T> __device__ __forceinline__ void switch_fn(const Prm<T>& p, T r2, T& sw, T& dsw) {
  if (r2 <= p.ron2) {
    sw = 1;
    dsw = 0;
    return;
  }
  const T u = p.rc2 - r2, v = p.rc2 + 2 * r2 - 3 * p.ron2;
  sw = u * u * v * p.sw_c3;
  dsw = 12 * u * (r2 - p.ron2) * p.sw_c3;
}

// switched LJ + erfc Coulomb of one pair: returns F/r (force on i = fr * d) and the
// pair energies (nonbondforce, src/nonbonded_forces.cu:137-214)
template <class T>
__device__ __forceinline__ T pair_force(const Prm<T>& p, T r2, T qq, T e4, T s2, T& evdw, T& eelec) {
  const T r = m_sqrt(r2), ir2 = T(1) / r2;
  const T br = p.beta * r;
  const T ec = p.cc * qq * m_erfc(br) / r;
  const T fc = (ec + p.cc * qq * T(1.1283791670955126) * p.beta * m_exp(-br * br)) * ir2;
  const T s6 = s2 * s2 * s2 * ir2 * ir2 * ir2;
  const T a = e4 * s6, b = a * s6;
  const T elj = b - a, flj = (12 * b - 6 * a) * ir2;
  T sw, dsw;
  switch_fn(p, r2, sw, dsw);
  evdw = elj * sw;
  eelec = ec;
  return flj * sw + elj * dsw + fc;
}

// thread per atom over its full list; each pair is met twice, so half of each pair
// energy is kept (nonbondforce, src/nonbonded_forces.cu:25-270).  Writes (not adds)
// the force: the first force stage of a step.
template <class T>
__global__ void k_nonbonded(Prm<T> p, const typename Vec<T>::v4* __restrict__ pos, const int* __restrict__ type,
                            const T* __restrict__ eps4, const T* __restrict__ sig2, const int* __restrict__ nbl,
                            const int* __restrict__ nbn, typename Vec<T>::v4* force, T* evdw_a, T* eelec_a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const typename Vec<T>::v4 ri = pos[i];
  const int ti = type[i] * p.nt;
  const int m = min(nbn[i], p.maxnb);
  T fx = 0, fy = 0, fz = 0, ev = 0, ee = 0;
  for (int k = 0; k < m; ++k) {
    const int j = nbl[(size_t)k * p.n + i];
    const typename Vec<T>::v4 rj = pos[j];
    T dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - rj.z;
    min_image(p, dx, dy, dz);
    const T r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= p.rc2) continue;
    const int t = ti + type[j];
    T e1, e2;
    const T fr = pair_force(p, r2, ri.w * rj.w, eps4[t], sig2[t], e1, e2);
    fx += fr * dx;
    fy += fr * dy;
    fz += fr * dz;
    ev += e1;
    ee += e2;
  }
  typename Vec<T>::v4 f;
  f.x = fx;
  f.y = fy;
  f.z = fz;
  f.w = 0;
  force[i] = f;
  evdw_a[i] = T(0.5) * ev;
  eelec_a[i] = T(0.5) * ee;
}

}  // namespace fzp
