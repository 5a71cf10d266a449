// Plain path: PME (per-grid-point atom lists, gather-style spread, influence-function
// multiply, thread-per-atom gather) and the velocity-Verlet/SHAKE/RATTLE kernels.
#pragma once
#include "plain_kernels.cuh"

namespace fzp {

constexpr int kLatCap = 64;  // atoms per grid-point list (the reference's 64, src/defs.in.h)

// order-4 B-spline weights of the points floor(u)-3+j, j = 0..3, at fractional part f,
// and their derivatives with respect to u
template <class T> __device__ __forceinline__ void bspline4(T f, T* w, T* dw) {
  const T f2 = f * f, f3 = f2 * f, g = 1 - f;
  w[0] = g * g * g / 6;
  w[1] = (3 * f3 - 6 * f2 + 4) / 6;
  w[2] = (-3 * f3 + 3 * f2 + 3 * f + 1) / 6;
  w[3] = f3 / 6;
  dw[0] = -g * g / 2;
  dw[1] = T(1.5) * f2 - 2 * f;
  dw[2] = T(-1.5) * f2 + f + T(0.5);
  dw[3] = f2 / 2;
}

// scaled coordinate u in [0, K): its floor and fraction
template <class T> __device__ __forceinline__ int grid_base(const Prm<T>& p, T x, int d, T& f) {
  T s = x * p.iL[d];
  s -= m_floor(s);
  const T u = s * (T)p.K[d];
  const T fl = m_floor(u);
  f = u - fl;
  return (int)fl;
}

// every atom appends itself to the lists of the 4x4x4 grid points its spline covers
// (LatticeBuild/LatticeUpdate, src/cell_based_kernels.cu:1557-1767)
template <class T>
__global__ void k_lattice(Prm<T> p, const typename Vec<T>::v4* __restrict__ pos, int* lat_n, int* lat_list,
                          int* status) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= p.n) return;
  const typename Vec<T>::v4 r = pos[a];
  T f;
  const int bx = grid_base(p, r.x, 0, f) - 3 + 4 * p.K[0];
  const int by = grid_base(p, r.y, 1, f) - 3 + 4 * p.K[1];
  const int bz = grid_base(p, r.z, 2, f) - 3 + 4 * p.K[2];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const int g = (((bx + i) % p.K[0]) * p.K[1] + (by + j) % p.K[1]) * p.K[2] + (bz + k) % p.K[2];
        const int s = atomicAdd(&lat_n[g], 1);
        if (s < kLatCap) lat_list[(size_t)g * kLatCap + s] = a;
        else atomicOr(status, PS_LATTICE_OVF);
      }
}

// thread per grid point: Q(g) = sum over its list of q M4 M4 M4 (ChargeSpread,
// src/pme_kernels.cu:20-239); the grid is complex with zero imaginary part
template <class T>
__global__ void k_spread(Prm<T> p, const typename Vec<T>::v4* __restrict__ pos, const int* __restrict__ lat_n,
                         const int* __restrict__ lat_list, typename Vec<T>::cplx* grid) {
  const int Kt = p.K[0] * p.K[1] * p.K[2];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= Kt) return;
  const int gz = g % p.K[2], gy = (g / p.K[2]) % p.K[1], gx = g / (p.K[1] * p.K[2]);
  const int m = min(lat_n[g], kLatCap);
  T q = 0;
  for (int s = 0; s < m; ++s) {
    const typename Vec<T>::v4 r = pos[lat_list[(size_t)g * kLatCap + s]];
    T fx, fy, fz, w[4], dw[4];
    const int jx = (gx - (grid_base(p, r.x, 0, fx) - 3) + 4 * p.K[0]) % p.K[0];
    const int jy = (gy - (grid_base(p, r.y, 1, fy) - 3) + 4 * p.K[1]) % p.K[1];
    const int jz = (gz - (grid_base(p, r.z, 2, fz) - 3) + 4 * p.K[2]) % p.K[2];
    bspline4(fx, w, dw);
    T t = r.w * w[jx & 3];
    bspline4(fy, w, dw);
    t *= w[jy & 3];
    bspline4(fz, w, dw);
    q += t * w[jz & 3];
  }
  typename Vec<T>::cplx c;
  c.x = q;
  c.y = 0;
  grid[g] = c;
}

// Q^(m) *= C(m) (BCMultiply, src/cell_based_kernels.cu:1770-1826)
template <class T> __global__ void k_bcmult(int Kt, typename Vec<T>::cplx* grid, const T* __restrict__ infl) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= Kt) return;
  const T c = infl[g];
  grid[g].x *= c;
  grid[g].y *= c;
}

// thread per atom: E_i = 1/2 q sum theta phi, F_i = -q sum grad(theta) phi
// (PMEForce, src/pme_kernels.cu:381-770); adds to the force array
template <class T>
__global__ void k_gather(Prm<T> p, const typename Vec<T>::v4* __restrict__ pos,
                         const typename Vec<T>::cplx* __restrict__ grid, typename Vec<T>::v4* force, T* epme) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= p.n) return;
  const typename Vec<T>::v4 r = pos[a];
  T f[3], w[3][4], dw[3][4];
  const int bx = grid_base(p, r.x, 0, f[0]) - 3 + 4 * p.K[0];
  const int by = grid_base(p, r.y, 1, f[1]) - 3 + 4 * p.K[1];
  const int bz = grid_base(p, r.z, 2, f[2]) - 3 + 4 * p.K[2];
  for (int d = 0; d < 3; ++d) bspline4(f[d], w[d], dw[d]);
  T e = 0, gx = 0, gy = 0, gz = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 4; ++k) {
        const int g = (((bx + i) % p.K[0]) * p.K[1] + (by + j) % p.K[1]) * p.K[2] + (bz + k) % p.K[2];
        const T phi = grid[g].x;
        e += w[0][i] * w[1][j] * w[2][k] * phi;
        gx += dw[0][i] * w[1][j] * w[2][k] * phi;
        gy += w[0][i] * dw[1][j] * w[2][k] * phi;
        gz += w[0][i] * w[1][j] * dw[2][k] * phi;
      }
  typename Vec<T>::v4 fo = force[a];
  fo.x -= r.w * gx * (T)p.K[0] * p.iL[0];
  fo.y -= r.w * gy * (T)p.K[1] * p.iL[1];
  fo.z -= r.w * gz * (T)p.K[2] * p.iL[2];
  force[a] = fo;
  epme[a] = T(0.5) * r.w * e;
}

// ------------------------------------------------------------------ integration
// v += (dt/2) F / m (HalfKickGPU, src/mdcuda.cu:27-92)
template <class T>
__global__ void k_kick(int n, T hdt, const typename Vec<T>::v4* __restrict__ force, const T* __restrict__ inv_m,
                       typename Vec<T>::v4* vel) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const T s = hdt * inv_m[a];
  const typename Vec<T>::v4 f = force[a];
  typename Vec<T>::v4 v = vel[a];
  v.x += s * f.x;
  v.y += s * f.y;
  v.z += s * f.z;
  vel[a] = v;
}

// r(t) kept for SHAKE, r += dt v (UpdateCoords, src/mdcuda.cu:354-375)
template <class T>
__global__ void k_drift(int n, T dt, typename Vec<T>::v4* pos, const typename Vec<T>::v4* __restrict__ vel,
                        typename Vec<T>::v4* pos_old) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  typename Vec<T>::v4 r = pos[a];
  pos_old[a] = r;
  const typename Vec<T>::v4 v = vel[a];
  r.x += dt * v.x;
  r.y += dt * v.y;
  r.z += dt * v.z;
  pos[a] = r;
}

struct Clusters {
  int n;
  const int4* atoms;  // -1 padded
  const int4* pairs;  // (na, nc, a0 | b0 << 2 | a1 << 4 | b1 << 6 | a2 << 8 | b2 << 10, 0)
};

// iterative SHAKE per cluster: each constraint k moves its two atoms along the bond
// vector of r(t) until |r_ab|^2 is within 2 tol d^2 of d^2 for every bond
// (solve_bond_constraints, src/shake.cu:20-327); velocities take the same correction / dt
template <class T>
__global__ void k_shake(Prm<T> p, Clusters c, const typename Vec<T>::v4* __restrict__ cl_d,
                        const typename Vec<T>::v4* __restrict__ pos_old, typename Vec<T>::v4* pos,
                        typename Vec<T>::v4* vel, const T* __restrict__ inv_m, T idt, T tol, int maxit, int* status) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= c.n) return;
  const int4 at4 = c.atoms[u], pr = c.pairs[u];
  const int at[4] = {at4.x, at4.y, at4.z, at4.w};
  const int na = pr.x, nc = pr.y;
  const typename Vec<T>::v4 dd = cl_d[u];
  const T d2[3] = {dd.x * dd.x, dd.y * dd.y, dd.z * dd.z};
  const typename Vec<T>::v4 o0 = pos_old[at[0]], n0 = pos[at[0]];
  T ro[4][3], rn[4][3], rn0[4][3], im[4];
  for (int k = 0; k < na; ++k) {
    const typename Vec<T>::v4 o = pos_old[at[k]], q = pos[at[k]];
    T x = o.x - o0.x, y = o.y - o0.y, z = o.z - o0.z;
    min_image(p, x, y, z);
    ro[k][0] = x;
    ro[k][1] = y;
    ro[k][2] = z;
    x = q.x - n0.x;
    y = q.y - n0.y;
    z = q.z - n0.z;
    min_image(p, x, y, z);
    rn[k][0] = rn0[k][0] = x;
    rn[k][1] = rn0[k][1] = y;
    rn[k][2] = rn0[k][2] = z;
    im[k] = inv_m[at[k]];
  }
  int it = 0;
  for (; it < maxit; ++it) {
    bool done = true;
    for (int k = 0; k < nc; ++k) {
      const int a = (pr.z >> (4 * k)) & 3, b = (pr.z >> (4 * k + 2)) & 3;
      const T sx = rn[a][0] - rn[b][0], sy = rn[a][1] - rn[b][1], sz = rn[a][2] - rn[b][2];
      const T diff = d2[k] - (sx * sx + sy * sy + sz * sz);
      if (fabs((double)diff) <= 2.0 * (double)tol * (double)d2[k]) continue;
      done = false;
      const T rx = ro[a][0] - ro[b][0], ry = ro[a][1] - ro[b][1], rz = ro[a][2] - ro[b][2];
      const T g = diff / (2 * (sx * rx + sy * ry + sz * rz) * (im[a] + im[b]));
      rn[a][0] += g * im[a] * rx;
      rn[a][1] += g * im[a] * ry;
      rn[a][2] += g * im[a] * rz;
      rn[b][0] -= g * im[b] * rx;
      rn[b][1] -= g * im[b] * ry;
      rn[b][2] -= g * im[b] * rz;
    }
    if (done) break;
  }
  if (it >= maxit) atomicOr(status, PS_SHAKE);
  for (int k = 0; k < na; ++k) {
    typename Vec<T>::v4 q = pos[at[k]], v = vel[at[k]];
    const T dx = rn[k][0] - rn0[k][0], dy = rn[k][1] - rn0[k][1], dz = rn[k][2] - rn0[k][2];
    q.x += dx;
    q.y += dy;
    q.z += dz;
    v.x += dx * idt;
    v.y += dy * idt;
    v.z += dz * idt;
    pos[at[k]] = q;
    vel[at[k]] = v;
  }
}

// iterative RATTLE velocity stage: (v_a - v_b) . r_ab = 0 for every bond
// (solve_velocity_constraints, src/shake.cu:330-615)
template <class T>
__global__ void k_rattle(Prm<T> p, Clusters c, const typename Vec<T>::v4* __restrict__ cl_d,
                         const typename Vec<T>::v4* __restrict__ pos, typename Vec<T>::v4* vel,
                         const T* __restrict__ inv_m, T tol, int maxit, int* status) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= c.n) return;
  const int4 at4 = c.atoms[u], pr = c.pairs[u];
  const int at[4] = {at4.x, at4.y, at4.z, at4.w};
  const int na = pr.x, nc = pr.y;
  const typename Vec<T>::v4 dd = cl_d[u];
  const T d2[3] = {dd.x * dd.x, dd.y * dd.y, dd.z * dd.z};
  const typename Vec<T>::v4 p0 = pos[at[0]];
  T r[4][3], v[4][3], v0[4][3], im[4];
  for (int k = 0; k < na; ++k) {
    const typename Vec<T>::v4 q = pos[at[k]], w = vel[at[k]];
    T x = q.x - p0.x, y = q.y - p0.y, z = q.z - p0.z;
    min_image(p, x, y, z);
    r[k][0] = x;
    r[k][1] = y;
    r[k][2] = z;
    v[k][0] = v0[k][0] = w.x;
    v[k][1] = v0[k][1] = w.y;
    v[k][2] = v0[k][2] = w.z;
    im[k] = inv_m[at[k]];
  }
  int it = 0;
  for (; it < maxit; ++it) {
    bool done = true;
    for (int k = 0; k < nc; ++k) {
      const int a = (pr.z >> (4 * k)) & 3, b = (pr.z >> (4 * k + 2)) & 3;
      const T rx = r[a][0] - r[b][0], ry = r[a][1] - r[b][1], rz = r[a][2] - r[b][2];
      const T vr = (v[a][0] - v[b][0]) * rx + (v[a][1] - v[b][1]) * ry + (v[a][2] - v[b][2]) * rz;
      if (fabs((double)vr) <= (double)tol * (double)d2[k]) continue;
      done = false;
      const T g = vr / ((rx * rx + ry * ry + rz * rz) * (im[a] + im[b]));
      v[a][0] -= g * im[a] * rx;
      v[a][1] -= g * im[a] * ry;
      v[a][2] -= g * im[a] * rz;
      v[b][0] += g * im[b] * rx;
      v[b][1] += g * im[b] * ry;
      v[b][2] += g * im[b] * rz;
    }
    if (done) break;
  }
  if (it >= maxit) atomicOr(status, PS_SHAKE);
  for (int k = 0; k < na; ++k) {
    typename Vec<T>::v4 w = vel[at[k]];
    w.x = v[k][0];
    w.y = v[k][1];
    w.z = v[k][2];
    vel[at[k]] = w;
  }
}

// wrap into [-L/2, L/2) (CoordsUpdate, src/mdcuda.cu:419-436) and the largest squared
// displacement since the last list build, for the host's rebuild decision
template <class T>
__global__ void k_wrap_disp(Prm<T> p, typename Vec<T>::v4* pos, const typename Vec<T>::v4* __restrict__ pos_build,
                            unsigned int* dmax) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f;
  if (a < p.n) {
    typename Vec<T>::v4 r = pos[a];
    r.x -= p.L[0] * m_floor(r.x * p.iL[0] + T(0.5));
    r.y -= p.L[1] * m_floor(r.y * p.iL[1] + T(0.5));
    r.z -= p.L[2] * m_floor(r.z * p.iL[2] + T(0.5));
    pos[a] = r;
    const typename Vec<T>::v4 b = pos_build[a];
    T dx = r.x - b.x, dy = r.y - b.y, dz = r.z - b.z;
    min_image(p, dx, dy, dz);
    d2 = (float)(dx * dx + dy * dy + dz * dz);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dmax, __float_as_uint(d2));
}

// per-atom energies and 2 KE summed in FP64 (Scan_Energy/reduce_PE,
// src/cell_based_kernels.cu:604-710)
template <class T>
__global__ void k_energy(int n, const T* __restrict__ evdw, const T* __restrict__ eelec, const T* __restrict__ epme,
                         const typename Vec<T>::v4* __restrict__ vel, const T* __restrict__ mass, double* e_acc) {
  __shared__ double sh[4][32];
  double s[4] = {0, 0, 0, 0};
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    s[0] += (double)evdw[a];
    s[1] += (double)eelec[a];
    s[2] += (double)epme[a];
    const typename Vec<T>::v4 v = vel[a];
    s[3] += (double)mass[a] * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < 4; ++k) {
    double x = s[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < 4; ++k) {
      double x = threadIdx.x < nw ? sh[k][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) {
        const int slot[4] = {PE_VDW, PE_ELEC, PE_PME, PE_KIN2};
        atomicAdd(&e_acc[slot[k]], x);
      }
    }
  }
}

}  // namespace fzp
