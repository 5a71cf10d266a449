// Smooth PME, order 4: charge spreading, hand-written 3-D R2C/C2R FFT with the
// influence function fused between the forward and inverse z passes, force gather.
// Replaces ChargeSpread_small/_medium (src/pme_kernels.cu:20-239), the cuFFT C2C
// pair and BCMultiply (src/mdcuda.cu:748,780, src/cell_based_kernels.cu:1770-1826)
// and PMEForce_medium/_large (src/pme_kernels.cu:381-770).
//
// Spreading: the grid is cut into bricks and atoms are binned by the brick of their
// base grid point every step; one CTA per brick spreads each of its atoms once into a
// shared-memory region (the brick grown by the 3-point stencil reach on its low side)
// with int32 fixed-point atomics, then adds the region into the int32 charge grid with
// one global atomic add per nonzero point (a point gets <= 8 such adds, from the
// regions covering it).  Integer sums are order independent, so the grid is
// bit-reproducible; there are no per-grid-point lists.  B-splines are evaluated analytically
// (the reference samples a 1001-point table with a truncating index).
#include "common.cuh"
#include "kernels.h"
#include <cstdlib>

namespace fzk {

struct FftPlan {
  int n;
  int nrad;
  int rad[12];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// base grid point k0 and fraction t of coordinate x along a dimension of K points
__device__ __forceinline__ int grid_base(float x, float invL, int K, float* t) {
  float s = x * invL;
  s -= floorf(s);
  const float u = s * (float)K;
  int k0 = (int)u;
  float f = u - (float)k0;
  if (k0 >= K) {
    k0 -= K;
    f = 0.f;
  }
  *t = f;
  return k0;
}

// cubic B-spline weights M4(t+j) for grid points k0-j, j = 0..3, and derivatives
__device__ __forceinline__ void bsp4(float t, float* w, float* dw) {
  const float t2 = t * t, t3 = t2 * t, u = 1.f - t;
  const float s = 1.f / 6.f;
  w[0] = t3 * s;
  w[1] = fmaf(-3.f, t3, fmaf(3.f, t2, fmaf(3.f, t, 1.f))) * s;
  w[2] = fmaf(3.f, t3, fmaf(-6.f, t2, 4.f)) * s;
  w[3] = u * u * u * s;
  if (dw) {
    dw[0] = 0.5f * t2;
    dw[1] = 0.5f * fmaf(-3.f, t2, fmaf(2.f, t, 1.f));
    dw[2] = 0.5f * fmaf(3.f, t2, -4.f * t);
    dw[3] = -0.5f * u * u;
  }
}

__device__ __forceinline__ void pme_zero_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  int* cnt = a.brick_count;
  int* cur = a.brick_cursor;
  const int nb = a.nb[0] * a.nb[1] * a.nb[2];
  for (int i = bid * blockDim.x + threadIdx.x; i < nb; i += nbid * blockDim.x) {
    cnt[i] = 0;
    cur[i] = 0;
  }
}

__global__ void k_pme_zero(PmeArgs a) { griddep_wait(); pme_zero_body(a, blockIdx.x, gridDim.x); }
__global__ void k_pme_zero_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_zero_body(a, t.y, t.z);
}


__device__ __forceinline__ void pme_bin_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  const int i = bid * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const float4 r = a.pos4[i];
  float t;
  const int kx = grid_base(r.x, a.p.inv_box.x, a.K[0], &t);
  const int ky = grid_base(r.y, a.p.inv_box.y, a.K[1], &t);
  const int kz = grid_base(r.z, a.p.inv_box.z, a.K[2], &t);
  const int b = ((kz / a.B[2]) * a.nb[1] + ky / a.B[1]) * a.nb[0] + kx / a.B[0];
  a.brick_of[i] = b;
  // warp-aggregated increment: one atomic per distinct brick in the warp
  const unsigned peers = __match_any_sync(__activemask(), b);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&a.brick_count[b], __popc(peers));
}

__global__ void k_pme_bin(PmeArgs a) { griddep_wait(); pme_bin_body(a, blockIdx.x, gridDim.x); }
__global__ void k_pme_bin_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_bin_body(a, t.y, t.z);
}


__device__ __forceinline__ void pme_scan_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  const int nbr = a.nb[0] * a.nb[1] * a.nb[2];
  __shared__ int part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (nbr + nt - 1) / nt;
  const int b = t * per, e = min(nbr, b + per);
  int s = 0;
  for (int c = b; c < e; ++c) s += a.brick_count[c];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - s;
  for (int c = b; c < e; ++c) {
    a.brick_start[c] = run;
    run += a.brick_count[c];
  }
  if (t == nt - 1) a.brick_start[nbr] = part[t];
}

__global__ void k_pme_scan(PmeArgs a) { griddep_wait(); pme_scan_body(a, blockIdx.x, gridDim.x); }
__global__ void k_pme_scan_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_scan_body(a, t.y, t.z);
}


__device__ __forceinline__ void pme_scatter_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  const int i = bid * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int b = a.brick_of[i];
  const unsigned peers = __match_any_sync(__activemask(), b);
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if ((threadIdx.x & 31) == leader) base = atomicAdd(&a.brick_cursor[b], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  const int k = base + __popc(peers & ((1u << (threadIdx.x & 31)) - 1u));
  a.brick_atoms[a.brick_start[b] + k] = i;
}

__global__ void k_pme_scatter(PmeArgs a) { griddep_wait(); pme_scatter_body(a, blockIdx.x, gridDim.x); }
__global__ void k_pme_scatter_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_scatter_body(a, t.y, t.z);
}


constexpr float kFixQ32 = 16777216.0f;  // charge grid fixed point, 2^24 per e

// the grid buffer holds int32 fixed-point charges from the spread until the x pass
// reads them, and the float potential from the inverse x pass until the gather
__device__ __forceinline__ float charge_at(const PmeArgs& a, size_t i) {
  return (float)reinterpret_cast<const int*>(a.grid)[i] * (1.0f / kFixQ32);
}

// One CTA per brick processes the atoms binned to that brick exactly once: their
// 4x4x4 stencils (grid points k0-3..k0 per dimension) all fall inside the brick grown
// by 3 points on the low side, accumulated in shared memory with int32 fixed-point
// atomics (2^24 per e; values stay far below +-128 e).  The region is then added to
// the int32 charge grid; integer sums are exact, so the grid is bit-reproducible.
__device__ __forceinline__ void pme_spread_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  extern __shared__ int acc[];
  const int Bx = a.B[0], By = a.B[1], Bz = a.B[2];
  const int Ex = Bx + 3, Ey = By + 3, Ez = Bz + 3;
  const int nbx = a.nb[0], nby = a.nb[1];
  const int b = bid;
  const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const int vol = Ex * Ey * Ez;
  for (int k = threadIdx.x; k < vol; k += blockDim.x) acc[k] = 0;
  __syncthreads();
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  // region origin: brick origin - 3
  const int ox = bx * Bx - 3, oy = by * By - 3, oz = bz * Bz - 3;
  const int s0 = a.brick_start[b], s1 = a.brick_start[b + 1];
  for (int idx = s0 + threadIdx.x; idx < s1; idx += blockDim.x) {
    const float4 r = a.pos4[a.brick_atoms[idx]];
    float tx, ty, tz, wx[4], wy[4], wz[4];
    const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx) - ox;
    const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty) - oy;
    const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz) - oz;
    bsp4(tx, wx, nullptr);
    bsp4(ty, wy, nullptr);
    bsp4(tz, wz, nullptr);
    const float q = r.w * kFixQ32;
#pragma unroll
    for (int jz = 0; jz < 4; ++jz)
#pragma unroll
      for (int jy = 0; jy < 4; ++jy) {
        const float qzy = q * wz[jz] * wy[jy];
        int* row = acc + ((kz - jz) * Ey + (ky - jy)) * Ex + kx;
#pragma unroll
        for (int jx = 0; jx < 4; ++jx) atomicAdd(row - jx, __float2int_rn(qzy * wx[jx]));
      }
  }
  __syncthreads();
  // add the region into the int32 charge grid (zeroed before the spread); the low-side
  // halo wraps periodically, the region never passes the grid's upper end.  A point of
  // the brick more than 3 below its upper faces (region index 3 .. B-1 on every axis)
  // lies in no other brick's region, so it takes a plain store; the rest are shared
  // with the neighbouring bricks' halos and take atomic adds.
  // Each thread keeps one (x, y) column of the region and walks it along z (the two
  // halves of the block take alternate z), so the column's grid address and ownership
  // are worked out once instead of dividing every region index by the extents.
  int* g = reinterpret_cast<int*>(a.grid);
  const int plane = Ex * Ey, half = blockDim.x >> 1;
  const size_t zstride = (size_t)Ky * Kx;
  for (int t = threadIdx.x % half; t < plane; t += half) {
    const int ry = t / Ex, rx = t - ry * Ex;
    int gx = ox + rx, gy = oy + ry;
    gx += gx < 0 ? Kx : 0;
    gy += gy < 0 ? Ky : 0;
    const bool own_xy = rx >= 3 && rx < Bx && ry >= 3 && ry < By;
    int* col = g + (size_t)gy * Kx + gx;
    for (int rz = threadIdx.x / half; rz < Ez; rz += 2) {
      const int v = acc[rz * plane + t];
      if (v == 0) continue;
      int gz = oz + rz;
      gz += gz < 0 ? Kz : 0;
      int* dst = col + (size_t)gz * zstride;
      if (own_xy && rz >= 3 && rz < Bz) *dst = v;
      else atomicAdd(dst, v);
    }
  }
}

__global__ void __launch_bounds__(256) k_pme_spread(PmeArgs a) { griddep_wait(); pme_spread_body(a, blockIdx.x, gridDim.x); }

// One thread per atom, each of its 64 weights added straight into the int32 charge grid
// (RED atomics in L2; the grid of a small system stays there).  The values added are the
// brick spread's own (same expressions), and integer sums do not depend on the order, so
// the grid is bit-identical to the brick spread's; with no brick lists the bin, scan and
// scatter launches disappear, which is what a small system's step is made of.
// Four threads per atom, one z layer of its stencil each (more threads in flight for
// the small systems this mode serves).
__global__ void __launch_bounds__(256) k_pme_spread_atoms(PmeArgs a) {
  griddep_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t >> 2, jz = t & 3;
  if (i >= a.n) return;
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  const float4 r = a.pos4[i];
  float tx, ty, tz, wx[4], wy[4], wz[4];
  const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx);
  const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty);
  const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz);
  bsp4(tx, wx, nullptr);
  bsp4(ty, wy, nullptr);
  bsp4(tz, wz, nullptr);
  const float q = r.w * kFixQ32;
  int* g = reinterpret_cast<int*>(a.grid);
  const float wzj = jz == 0 ? wz[0] : (jz == 1 ? wz[1] : (jz == 2 ? wz[2] : wz[3]));
  {
    int z = kz - jz;
    z += z < 0 ? Kz : 0;
#pragma unroll
    for (int jy = 0; jy < 4; ++jy) {
      int y = ky - jy;
      y += y < 0 ? Ky : 0;
      const float qzy = q * wzj * wy[jy];
      int* row = g + ((size_t)z * Ky + y) * Kx;
#pragma unroll
      for (int jx = 0; jx < 4; ++jx) {
        int x = kx - jx;
        x += x < 0 ? Kx : 0;
        atomicAdd(row + x, __float2int_rn(qzy * wx[jx]));
      }
    }
  }
}
__global__ void __launch_bounds__(256) k_pme_spread_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_spread_body(a, t.y, t.z);
}



// ------------------------------------------------------------------ FFT
// Stockham autosort FFT of nl lines of length n in shared memory (x at a[l*n + i]).
// Returns the buffer holding the result.
__device__ float2* fft_lines(float2* a, float2* b, const float2* tw, const FftPlan& pl, int nl, bool inv) {
  const int n = pl.n, ld = n + 1;
  int Ns = 1;
  for (int s = 0; s < pl.nrad; ++s) {
    const int R = pl.rad[s];
    const int nbf = n / R;
    const int step = n / (Ns * R);
    for (int idx = threadIdx.x; idx < nl * nbf; idx += blockDim.x) {
      const int l = idx / nbf, j = idx - l * nbf;
      const float2* x = a + l * ld;
      float2* y = b + l * ld;
      const int k = j % Ns;
      float2 v[5], V[5];
#pragma unroll
      for (int r = 0; r < 5; ++r)
        if (r < R) v[r] = x[j + r * nbf];
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < 5; ++r)
          if (r < R) {
            float2 w = tw[r * k * step];
            if (inv) w.y = -w.y;
            v[r] = cmul(v[r], w);
          }
      }
      if (R == 2) {
        V[0] = make_float2(v[0].x + v[1].x, v[0].y + v[1].y);
        V[1] = make_float2(v[0].x - v[1].x, v[0].y - v[1].y);
      } else if (R == 4) {
        const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
        const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
        const float2 b0 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
        const float2 b1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
        V[0] = make_float2(a0.x + b0.x, a0.y + b0.y);
        V[2] = make_float2(a0.x - b0.x, a0.y - b0.y);
        if (!inv) {  // -i * b1 = (b1.y, -b1.x)
          V[1] = make_float2(a1.x + b1.y, a1.y - b1.x);
          V[3] = make_float2(a1.x - b1.y, a1.y + b1.x);
        } else {
          V[1] = make_float2(a1.x - b1.y, a1.y + b1.x);
          V[3] = make_float2(a1.x + b1.y, a1.y - b1.x);
        }
      } else {
        const int st = n / R;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          if (q >= R) continue;
          float2 acc = v[0];
#pragma unroll
          for (int r = 1; r < 5; ++r) {
            if (r >= R) continue;
            float2 w = tw[((r * q) % R) * st];
            if (inv) w.y = -w.y;
            const float2 t = cmul(v[r], w);
            acc.x += t.x;
            acc.y += t.y;
          }
          V[q] = acc;
        }
      }
      const int o = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < 5; ++r)
        if (r < R) y[o + r * Ns] = V[r];
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

__device__ __forceinline__ void load_tw(float2* s, const float2* g, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// x pass forward: real rows -> half spectrum (mx = 0..Kx/2)
__global__ void __launch_bounds__(256) k_fft_x_r2c(PmeArgs a, FftPlan pl, int nl) { griddep_wait();
  extern __shared__ float2 sm[];
  const int Kx = a.K[0], Kxh = Kx / 2 + 1;
  const int nrows = a.K[1] * a.K[2];
  const int ld = Kx + 1;
  float2* tw = sm;
  float2* A = sm + Kx;
  float2* B = A + nl * ld;
  load_tw(tw, a.tw[0], Kx);
  const int r0 = blockIdx.x * nl;
  for (int idx = threadIdx.x; idx < nl * Kx; idx += blockDim.x) {
    const int l = idx / Kx, x = idx - l * Kx;
    const int row = r0 + l;
    A[l * ld + x] = make_float2(row < nrows ? charge_at(a, (size_t)row * Kx + x) : 0.f, 0.f);
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, tw, pl, nl, false);
  for (int idx = threadIdx.x; idx < nl * Kxh; idx += blockDim.x) {
    const int l = idx / Kxh, m = idx - l * Kxh;
    const int row = r0 + l;
    if (row < nrows) a.cgrid[(size_t)row * Kxh + m] = R[l * ld + m];
  }
}

// y pass (forward or inverse): lines along y for nl consecutive mx at fixed z
__global__ void __launch_bounds__(256) k_fft_y(PmeArgs a, FftPlan pl, int nl, int inv) { griddep_wait();
  extern __shared__ float2 sm[];
  const int Kx = a.K[0], Ky = a.K[1], Kxh = Kx / 2 + 1;
  const int ng = (Kxh + nl - 1) / nl;
  const int z = blockIdx.x / ng, mx0 = (blockIdx.x % ng) * nl;
  const int ld = Ky + 1;
  float2* tw = sm;
  float2* A = sm + Ky;
  float2* B = A + nl * ld;
  load_tw(tw, a.tw[1], Ky);
  for (int idx = threadIdx.x; idx < nl * Ky; idx += blockDim.x) {
    const int y = idx / nl, l = idx - y * nl;
    const int mx = mx0 + l;
    A[l * ld + y] = mx < Kxh ? a.cgrid[((size_t)z * Ky + y) * Kxh + mx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, tw, pl, nl, inv != 0);
  for (int idx = threadIdx.x; idx < nl * Ky; idx += blockDim.x) {
    const int y = idx / nl, l = idx - y * nl;
    const int mx = mx0 + l;
    if (mx < Kxh) a.cgrid[((size_t)z * Ky + y) * Kxh + mx] = R[l * ld + y];
  }
}

// z pass: forward, influence function (and reciprocal energy), inverse
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_fft_z_conv(PmeArgs a, FftPlan pl, int nl) { griddep_wait();
  extern __shared__ float2 sm[];
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2], Kxh = Kx / 2 + 1;
  const int ng = (Kxh + nl - 1) / nl;
  const int y = blockIdx.x / ng, mx0 = (blockIdx.x % ng) * nl;
  const int ld = Kz + 1;
  float2* tw = sm;
  float2* A = sm + Kz;
  float2* B = A + nl * ld;
  load_tw(tw, a.tw[2], Kz);
  for (int idx = threadIdx.x; idx < nl * Kz; idx += blockDim.x) {
    const int z = idx / nl, l = idx - z * nl;
    const int mx = mx0 + l;
    A[l * ld + z] = mx < Kxh ? a.cgrid[((size_t)z * Ky + y) * Kxh + mx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* R = fft_lines(A, B, tw, pl, nl, false);
  float2* O = (R == A) ? B : A;
  double e = 0.0, w0 = 0.0, w1 = 0.0, w2 = 0.0;
  const float gy = a.gfac[1][y], fy2 = a.f2[1][y];
  for (int idx = threadIdx.x; idx < nl * Kz; idx += blockDim.x) {
    const int l = idx / Kz, z = idx - l * Kz;
    const int mx = mx0 + l;
    float2 v = R[l * ld + z];
    float G = 0.f;
    if (mx < Kxh && (mx | y | z) != 0) {
      const float den = a.f2[0][mx] + fy2 + a.f2[2][z];
      G = a.gscale * a.gfac[0][mx] * gy * a.gfac[2][z] / den;
    }
    if (ENERGY && mx < Kxh && G != 0.f) {
      // energy of this mode and its virial diagonal E (1 - 2 (1 + pi^2 m^2/beta^2) m_a^2 / m^2)
      const double wmx = (mx == 0 || (2 * mx == Kx)) ? 1.0 : 2.0;
      const double em = wmx * 0.5 * (double)G * ((double)v.x * v.x + (double)v.y * v.y);
      const double fx2 = a.f2[0][mx], fz2 = a.f2[2][z];
      const double m2 = fx2 + fy2 + fz2;
      const double k = 2.0 * (1.0 + kPi * kPi * m2 / ((double)a.p.beta * a.p.beta)) / m2;
      e += em;
      w0 += em * (1.0 - k * fx2);
      w1 += em * (1.0 - k * fy2);
      w2 += em * (1.0 - k * fz2);
    }
    v.x *= G;
    v.y *= G;
    R[l * ld + z] = v;
  }
  __syncthreads();
  const float2* Q = fft_lines(R, O, tw, pl, nl, true);
  for (int idx = threadIdx.x; idx < nl * Kz; idx += blockDim.x) {
    const int z = idx / nl, l = idx - z * nl;
    const int mx = mx0 + l;
    if (mx < Kxh) a.cgrid[((size_t)z * Ky + y) * Kxh + mx] = Q[l * ld + z];
  }
  if (ENERGY) {
    energy_add(a.energy + EN_PME, e);
    energy_add(a.energy + EN_VIR_X, w0);
    energy_add(a.energy + EN_VIR_Y, w1);
    energy_add(a.energy + EN_VIR_Z, w2);
  }
}

// x pass inverse: Hermitian half rows -> real potential rows
__global__ void __launch_bounds__(256) k_fft_x_c2r(PmeArgs a, FftPlan pl, int nl) { griddep_wait();
  extern __shared__ float2 sm[];
  const int Kx = a.K[0], Kxh = Kx / 2 + 1;
  const int nrows = a.K[1] * a.K[2];
  const int ld = Kx + 1;
  float2* tw = sm;
  float2* A = sm + Kx;
  float2* B = A + nl * ld;
  load_tw(tw, a.tw[0], Kx);
  const int r0 = blockIdx.x * nl;
  for (int idx = threadIdx.x; idx < nl * Kx; idx += blockDim.x) {
    const int l = idx / Kx, m = idx - l * Kx;
    const int row = r0 + l;
    float2 v = make_float2(0.f, 0.f);
    if (row < nrows) {
      if (m < Kxh) v = a.cgrid[(size_t)row * Kxh + m];
      else {
        v = a.cgrid[(size_t)row * Kxh + (Kx - m)];
        v.y = -v.y;
      }
    }
    A[l * ld + m] = v;
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, tw, pl, nl, true);
  for (int idx = threadIdx.x; idx < nl * Kx; idx += blockDim.x) {
    const int l = idx / Kx, x = idx - l * Kx;
    const int row = r0 + l;
    if (row < nrows) a.grid[(size_t)row * Kx + x] = R[l * ld + x].x;
  }
}

// One thread per atom, atoms taken in brick order so a warp reads neighbouring grid
// lines from L2; used when bricks hold many atoms (one CTA per brick would then load
// its region and compute in two long serial phases).
__device__ __forceinline__ void pme_gather_atoms_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  // four threads per atom, one z layer of its stencil each; the layer sums meet as
  // (l0 + l1) + (l2 + l3), the order every gather uses
  const int t = bid * blockDim.x + threadIdx.x;
  const int ta = t >> 2, jz = t & 3;
  const bool valid = ta < a.n;
  const int i = !valid ? 0 : (a.gather == 3 ? ta : a.brick_atoms[ta]);  // mode 3: atom order
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  const float4 r = a.pos4[i];
  float tx, ty, tz, wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
  const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx);
  const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty);
  const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz);
  bsp4(tx, wx, dx);
  bsp4(ty, wy, dy);
  bsp4(tz, wz, dz);
  const float wzj = jz == 0 ? wz[0] : (jz == 1 ? wz[1] : (jz == 2 ? wz[2] : wz[3]));
  const float dzj = jz == 0 ? dz[0] : (jz == 1 ? dz[1] : (jz == 2 ? dz[2] : dz[3]));
  int z = kz - jz;
  z += z < 0 ? Kz : 0;
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int jy = 0; jy < 4; ++jy) {
    int y = ky - jy;
    y += y < 0 ? Ky : 0;
    const float* row = a.grid + ((size_t)z * Ky + y) * Kx;
    float sx = 0.f, sdx = 0.f;
#pragma unroll
    for (int jx = 0; jx < 4; ++jx) {
      int x = kx - jx;
      x += x < 0 ? Kx : 0;
      const float phi = valid ? __ldg(row + x) : 0.f;
      sx = fmaf(wx[jx], phi, sx);
      sdx = fmaf(dx[jx], phi, sdx);
    }
    gx = fmaf(sdx, wy[jy] * wzj, gx);
    gy = fmaf(sx, dy[jy] * wzj, gy);
    gz = fmaf(sx, wy[jy] * dzj, gz);
  }
  gx += __shfl_xor_sync(0xffffffffu, gx, 1);
  gy += __shfl_xor_sync(0xffffffffu, gy, 1);
  gz += __shfl_xor_sync(0xffffffffu, gz, 1);
  gx += __shfl_xor_sync(0xffffffffu, gx, 2);
  gy += __shfl_xor_sync(0xffffffffu, gy, 2);
  gz += __shfl_xor_sync(0xffffffffu, gz, 2);
  if (!valid || jz != 0) return;
  const float q = r.w;
  const int n = a.n;
  red_add(a.facc + i, to_fix(-q * gx * (float)Kx * a.p.inv_box.x));
  red_add(a.facc + n + i, to_fix(-q * gy * (float)Ky * a.p.inv_box.y));
  red_add(a.facc + 2 * n + i, to_fix(-q * gz * (float)Kz * a.p.inv_box.z));
}

__global__ void __launch_bounds__(256) k_pme_gather_atoms(PmeArgs a) { griddep_wait(); pme_gather_atoms_body(a, blockIdx.x, gridDim.x); }

// One CTA per brick, as the spread: the brick's region of the potential (the brick
// grown by 3 points on the low side, wrapped periodically) is loaded into shared
// memory row by row, then each thread gathers the force of the brick's atoms from
// there, 64 shared-memory reads per atom instead of 64 scattered global loads.  Used
// when bricks hold few atoms; both gathers sum in the same order (identical forces).
__device__ __forceinline__ void pme_gather_body(const PmeArgs& a, int bid, int nbid) {
  griddep_wait();
  extern __shared__ float phi_reg[];
  const int Bx = a.B[0], By = a.B[1], Bz = a.B[2];
  const int Ex = Bx + 3, Ey = By + 3, Ez = Bz + 3;
  const int nbx = a.nb[0], nby = a.nb[1];
  const int b = bid;
  const int s0 = a.brick_start[b], s1 = a.brick_start[b + 1];
  if (s0 == s1) return;
  const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  const int ox = bx * Bx - 3, oy = by * By - 3, oz = bz * Bz - 3;
  // region load by (x, y) columns walked along z, as the spread's flush
  const int plane = Ex * Ey, half = blockDim.x >> 1;
  const size_t zstride = (size_t)Ky * Kx;
  for (int t = threadIdx.x % half; t < plane; t += half) {
    const int ry = t / Ex, rx = t - ry * Ex;
    int gx = ox + rx, gy = oy + ry;
    gx += gx < 0 ? Kx : 0;
    gy += gy < 0 ? Ky : 0;
    const float* col = a.grid + (size_t)gy * Kx + gx;
    for (int rz = threadIdx.x / half; rz < Ez; rz += 2) {
      int gz = oz + rz;
      gz += gz < 0 ? Kz : 0;
      phi_reg[rz * plane + t] = __ldg(col + (size_t)gz * zstride);
    }
  }
  __syncthreads();
  const int n = a.n;
  for (int idx = s0 + threadIdx.x; idx < s1; idx += blockDim.x) {
    const int i = a.brick_atoms[idx];
    const float4 r = a.pos4[i];
    float tx, ty, tz, wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx) - ox;
    const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty) - oy;
    const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz) - oz;
    bsp4(tx, wx, dx);
    bsp4(ty, wy, dy);
    bsp4(tz, wz, dz);
    // one partial per z layer of the stencil, summed as (l0 + l1) + (l2 + l3): the
    // order of the four-thread per-atom gather, so both give the same forces
    float gx = 0.f, gy = 0.f, gz = 0.f, hx = 0.f, hy = 0.f, hz = 0.f;
#pragma unroll
    for (int jz = 0; jz < 4; ++jz) {
      float lx = 0.f, ly = 0.f, lz = 0.f;
#pragma unroll
      for (int jy = 0; jy < 4; ++jy) {
        const float* row = phi_reg + ((kz - jz) * Ey + (ky - jy)) * Ex + kx;
        float sx = 0.f, sdx = 0.f;
#pragma unroll
        for (int jx = 0; jx < 4; ++jx) {
          const float phi = row[-jx];
          sx = fmaf(wx[jx], phi, sx);
          sdx = fmaf(dx[jx], phi, sdx);
        }
        lx = fmaf(sdx, wy[jy] * wz[jz], lx);
        ly = fmaf(sx, dy[jy] * wz[jz], ly);
        lz = fmaf(sx, wy[jy] * dz[jz], lz);
      }
      // layers 0 and 1 into g, layers 2 and 3 into h
      if (jz == 0 || jz == 2) {
        (jz == 0 ? gx : hx) = lx;
        (jz == 0 ? gy : hy) = ly;
        (jz == 0 ? gz : hz) = lz;
      } else {
        (jz == 1 ? gx : hx) += lx;
        (jz == 1 ? gy : hy) += ly;
        (jz == 1 ? gz : hz) += lz;
      }
    }
    gx += hx;
    gy += hy;
    gz += hz;
    const float q = r.w;
    red_add(a.facc + i, to_fix(-q * gx * (float)Kx * a.p.inv_box.x));
    red_add(a.facc + n + i, to_fix(-q * gy * (float)Ky * a.p.inv_box.y));
    red_add(a.facc + 2 * n + i, to_fix(-q * gz * (float)Kz * a.p.inv_box.z));
  }
}

__global__ void __launch_bounds__(256) k_pme_gather(PmeArgs a) { griddep_wait(); pme_gather_body(a, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) k_pme_gather_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  pme_gather_body(a, t.y, t.z);
}


// ------------------------------------------------------------------ compile-time FFT
// The same Stockham autosort algorithm with the line length N a template parameter:
// radices, strides and twiddle steps are constants, the small DFTs use constant roots.
// Radices 16 and 8 come first (128 = 16 x 8: two passes through shared memory per
// line instead of four with radix 4), each DFT held in registers.
__host__ __device__ constexpr int radix_of(int m) {
  return m % 16 == 0 ? 16 : (m % 8 == 0 ? 8 : (m % 4 == 0 ? 4 : (m % 2 == 0 ? 2 : (m % 3 == 0 ? 3 : 5))));
}

// Shared-memory layout of a contiguous line: element i sits at sk(i) = i + i / 16 and
// lines are fft_ld(N) apart.  A radix-R stage's first pass stores each thread's R
// outputs at stride R; the pad slot every 16 elements spreads those stores over all
// banks instead of a few (stride 16 float2 would put a half-warp on one bank).
__host__ __device__ constexpr int fft_ld(int n) { return n + n / 16 + 1; }
__device__ __forceinline__ int sk(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int radix_at(int n, int s) {
  int m = n, r = 1;
  for (int k = 0; k <= s; ++k) {
    r = radix_of(m);
    m /= r;
  }
  return r;
}
__host__ __device__ constexpr int nstages(int n) {
  int m = n, c = 0;
  while (m > 1) {
    m /= radix_of(m);
    ++c;
  }
  return c;
}

// v e^{sg 2 pi i m / 16} for m known after unrolling (sg = -1 forward, +1 inverse);
// the quarter turns are exact swaps and sign flips
template <bool INV>
__device__ __forceinline__ float2 rot16(float2 v, int m) {
  const float sg = INV ? 1.f : -1.f;
  constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
  switch (m & 15) {
    case 0: return v;
    case 4: return make_float2(-sg * v.y, sg * v.x);
    case 8: return make_float2(-v.x, -v.y);
    case 12: return make_float2(sg * v.y, -sg * v.x);
    case 1: return cmul(v, make_float2(c1, sg * s1));
    case 2: return cmul(v, make_float2(h, sg * h));
    case 3: return cmul(v, make_float2(s1, sg * c1));
    case 5: return cmul(v, make_float2(-s1, sg * c1));
    case 6: return cmul(v, make_float2(-h, sg * h));
    case 7: return cmul(v, make_float2(-c1, sg * s1));
    case 9: return cmul(v, make_float2(-c1, -sg * s1));
    case 10: return cmul(v, make_float2(-h, -sg * h));
    case 11: return cmul(v, make_float2(-s1, -sg * c1));
    case 13: return cmul(v, make_float2(s1, -sg * c1));
    case 14: return cmul(v, make_float2(h, -sg * h));
    default: return cmul(v, make_float2(c1, -sg * s1));
  }
}

template <int R, bool INV>
__device__ __forceinline__ void small_dft(float2* v) {
  const float sg = INV ? 1.f : -1.f;  // exponent sign
  if constexpr (R == 16) {
    // 16 = 4 x 4: with n = r + 4q and k = k1 + 4 k2, W16^{nk} = W4^{q k1} W16^{r k1} W4^{r k2}
    float2 t[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
      for (int q = 0; q < 4; ++q) t[r][q] = v[r + 4 * q];
      small_dft<4, INV>(t[r]);
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) t[r][k1] = rot16<INV>(t[r][k1], r * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 u[4] = {t[0][k1], t[1][k1], t[2][k1], t[3][k1]};
      small_dft<4, INV>(u);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = u[k2];
    }
  } else if constexpr (R == 8) {
    // 8 = 2 x 4: even and odd halves, the odd one turned by W8^k
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    small_dft<4, INV>(e);
    small_dft<4, INV>(o);
#pragma unroll
    for (int k = 1; k < 4; ++k) o[k] = rot16<INV>(o[k], 2 * k);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = make_float2(e[k].x + o[k].x, e[k].y + o[k].y);
      v[k + 4] = make_float2(e[k].x - o[k].x, e[k].y - o[k].y);
    }
  } else if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
    const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
    const float2 b0 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
    const float2 b1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
    // sg * i * b1 = (-sg b1.y, sg b1.x)
    v[0] = make_float2(a0.x + b0.x, a0.y + b0.y);
    v[2] = make_float2(a0.x - b0.x, a0.y - b0.y);
    v[1] = make_float2(a1.x - sg * b1.y, a1.y + sg * b1.x);
    v[3] = make_float2(a1.x + sg * b1.y, a1.y - sg * b1.x);
  } else if constexpr (R == 3) {
    const float c1 = -0.5f, s1 = sg * 0.86602540378443865f;  // e^{sg 2 pi i/3}
    const float2 t = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
    const float2 d = make_float2(v[1].x - v[2].x, v[1].y - v[2].y);
    const float2 m = make_float2(v[0].x + c1 * t.x, v[0].y + c1 * t.y);
    v[0] = make_float2(v[0].x + t.x, v[0].y + t.y);
    v[1] = make_float2(m.x - s1 * d.y, m.y + s1 * d.x);
    v[2] = make_float2(m.x + s1 * d.y, m.y - s1 * d.x);
  } else {  // R == 5
    const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
    const float s1 = sg * 0.95105651629515357f, s2 = sg * 0.58778525229247313f;
    const float2 t1 = make_float2(v[1].x + v[4].x, v[1].y + v[4].y);
    const float2 d1 = make_float2(v[1].x - v[4].x, v[1].y - v[4].y);
    const float2 t2 = make_float2(v[2].x + v[3].x, v[2].y + v[3].y);
    const float2 d2 = make_float2(v[2].x - v[3].x, v[2].y - v[3].y);
    const float2 m1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const float2 m2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const float2 n1 = make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    const float2 n2 = make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    v[0] = make_float2(v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y);
    v[1] = make_float2(m1.x - n1.y, m1.y + n1.x);
    v[4] = make_float2(m1.x + n1.y, m1.y - n1.x);
    v[2] = make_float2(m2.x - n2.y, m2.y + n2.x);
    v[3] = make_float2(m2.x + n2.y, m2.y - n2.x);
  }
}

// Threads per block of the compile-time FFT kernels (all are launched with 256) and
// lines per block, both constants so the index arithmetic of every load, store and
// butterfly loop folds to shifts and multiplies and the loops unroll.
constexpr int kFftThreads = 256;
// (8 lines for every size: a small grid's passes then have several CTAs per SM's worth
// of blocks instead of one block per plane row; 48^3: 61.8 -> 61.5 us per MD step)
__host__ __device__ constexpr int fft_lines_per_block(int) { return 8; }

template <int N, int R, int NS, bool INV>
__device__ __forceinline__ void fft_stage_t(const float2* x, float2* y, const float2* tw, int nl) {
  constexpr int NB = N / R, STEP = N / (NS * R), LD = fft_ld(N);
  for (int idx = threadIdx.x; idx < nl * NB; idx += kFftThreads) {
    const int l = idx / NB, j = idx - l * NB;
    const int k = j % NS;
    const float2* xl = x + l * LD;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = xl[sk(j + r * NB)];
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * k * STEP];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    small_dft<R, INV>(v);
    float2* yl = y + l * LD;
    const int o = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) yl[sk(o + r * NS)] = v[r];
  }
}

template <int N, int S, int NS, bool INV>
__device__ __forceinline__ float2* fft_run_t(float2* a, float2* b, const float2* tw, int nl) {
  if constexpr (S == nstages(N)) {
    return a;
  } else {
    constexpr int R = radix_at(N, S);
    fft_stage_t<N, R, NS, INV>(a, b, tw, nl);
    __syncthreads();
    return fft_run_t<N, S + 1, NS * R, INV>(b, a, tw, nl);
  }
}

// Real rows in pairs: rows 2p and 2p+1 of the block are the real and imaginary parts of
// one complex line, so each complex FFT transforms two rows; with Z its transform,
// X0(m) = (Z(m) + conj Z(N-m)) / 2 and X1(m) = (Z(m) - conj Z(N-m)) / 2i.
template <int N>
__global__ void __launch_bounds__(256) k_fft_x_r2c_t(PmeArgs a, int) { griddep_wait();
  constexpr int nl = fft_lines_per_block(N);  // complex lines = row pairs per block
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N), NH = N / 2 + 1;
  const int nrows = a.K[1] * a.K[2];
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + nl * LD;
  load_tw(tw, a.tw[0], N);
  const int r0 = blockIdx.x * 2 * nl;
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int l = idx / N, x = idx - l * N;
    const int row = r0 + 2 * l;
    A[l * LD + sk(x)] = make_float2(row < nrows ? charge_at(a, (size_t)row * N + x) : 0.f,
                                row + 1 < nrows ? charge_at(a, (size_t)(row + 1) * N + x) : 0.f);
  }
  __syncthreads();
  const float2* R = fft_run_t<N, 0, 1, false>(A, B, tw, nl);
  for (int idx = threadIdx.x; idx < nl * NH; idx += kFftThreads) {
    const int l = idx / NH, m = idx - l * NH;
    const int row = r0 + 2 * l;
    const float2 z = R[l * LD + sk(m)], w = R[l * LD + sk(m == 0 ? 0 : N - m)];  // w = Z(N-m)
    if (row < nrows) a.cgrid[(size_t)row * NH + m] = make_float2(0.5f * (z.x + w.x), 0.5f * (z.y - w.y));
    if (row + 1 < nrows) a.cgrid[(size_t)(row + 1) * NH + m] = make_float2(0.5f * (z.y + w.y), 0.5f * (w.x - z.x));
  }
}

template <int N, bool INV>
__global__ void __launch_bounds__(256) k_fft_y_t(PmeArgs a, int) { griddep_wait();
  constexpr int nl = fft_lines_per_block(N);
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N);
  const int Kxh = a.K[0] / 2 + 1;
  const int ng = (Kxh + nl - 1) / nl;
  const int z = blockIdx.x / ng, mx0 = (blockIdx.x % ng) * nl;
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + nl * LD;
  load_tw(tw, a.tw[1], N);
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int y = idx / nl, l = idx - y * nl;
    const int mx = mx0 + l;
    A[l * LD + sk(y)] = mx < Kxh ? a.cgrid[((size_t)z * N + y) * Kxh + mx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* R = fft_run_t<N, 0, 1, INV>(A, B, tw, nl);
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int y = idx / nl, l = idx - y * nl;
    const int mx = mx0 + l;
    if (mx < Kxh) a.cgrid[((size_t)z * N + y) * Kxh + mx] = R[l * LD + sk(y)];
  }
}

template <int N, bool ENERGY>
__device__ __forceinline__ void fft_z_conv_body(const PmeArgs& a, int bid) {
  griddep_wait();
  constexpr int nl = fft_lines_per_block(N);
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N);
  const int Kx = a.K[0], Ky = a.K[1], Kxh = Kx / 2 + 1;
  const int ng = (Kxh + nl - 1) / nl;
  const int y = bid / ng, mx0 = (bid % ng) * nl;
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + nl * LD;
  load_tw(tw, a.tw[2], N);
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int z = idx / nl, l = idx - z * nl;
    const int mx = mx0 + l;
    A[l * LD + sk(z)] = mx < Kxh ? a.cgrid[((size_t)z * Ky + y) * Kxh + mx] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* R = fft_run_t<N, 0, 1, false>(A, B, tw, nl);
  float2* O = (R == A) ? B : A;
  double e = 0.0, w0 = 0.0, w1 = 0.0, w2 = 0.0;
  const float gy = a.gfac[1][y], fy2 = a.f2[1][y];
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int l = idx / N, z = idx - l * N;
    const int mx = mx0 + l;
    float2 v = R[l * LD + sk(z)];
    float G = 0.f;
    if (mx < Kxh && (mx | y | z) != 0) G = a.gscale * a.gfac[0][mx] * gy * a.gfac[2][z] / (a.f2[0][mx] + fy2 + a.f2[2][z]);
    if (ENERGY && mx < Kxh && G != 0.f) {
      // energy of this mode and its virial diagonal E (1 - 2 (1 + pi^2 m^2/beta^2) m_a^2 / m^2)
      const double wmx = (mx == 0 || (2 * mx == Kx)) ? 1.0 : 2.0;
      const double em = wmx * 0.5 * (double)G * ((double)v.x * v.x + (double)v.y * v.y);
      const double fx2 = a.f2[0][mx], fz2 = a.f2[2][z];
      const double m2 = fx2 + fy2 + fz2;
      const double k = 2.0 * (1.0 + kPi * kPi * m2 / ((double)a.p.beta * a.p.beta)) / m2;
      e += em;
      w0 += em * (1.0 - k * fx2);
      w1 += em * (1.0 - k * fy2);
      w2 += em * (1.0 - k * fz2);
    }
    v.x *= G;
    v.y *= G;
    R[l * LD + sk(z)] = v;
  }
  __syncthreads();
  const float2* Q = fft_run_t<N, 0, 1, true>(R, O, tw, nl);
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int z = idx / nl, l = idx - z * nl;
    const int mx = mx0 + l;
    if (mx < Kxh) a.cgrid[((size_t)z * Ky + y) * Kxh + mx] = Q[l * LD + sk(z)];
  }
  if (ENERGY) {
    energy_add(a.energy + EN_PME, e);
    energy_add(a.energy + EN_VIR_X, w0);
    energy_add(a.energy + EN_VIR_Y, w1);
    energy_add(a.energy + EN_VIR_Z, w2);
  }
}

template <int N, bool ENERGY>
__global__ void __launch_bounds__(256) k_fft_z_conv_t(PmeArgs a, int) { griddep_wait(); fft_z_conv_body<N, ENERGY>(a, blockIdx.x); }
template <int N>
__global__ void __launch_bounds__(256) k_fft_z_conv_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  fft_z_conv_body<N, false>(a, t.y);
}


// Inverse of the pairing above: Z(m) = X0(m) + i X1(m) over the full line (Hermitian
// extension for m > N/2) transforms back to row 2p + i row 2p+1.
template <int N>
__global__ void __launch_bounds__(256) k_fft_x_c2r_t(PmeArgs a, int) { griddep_wait();
  constexpr int nl = fft_lines_per_block(N);
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N), NH = N / 2 + 1;
  const int nrows = a.K[1] * a.K[2];
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + nl * LD;
  load_tw(tw, a.tw[0], N);
  const int r0 = blockIdx.x * 2 * nl;
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int l = idx / N, m = idx - l * N;
    const int row = r0 + 2 * l;
    const bool lo = m < NH;
    const int mm = lo ? m : N - m;
    float2 x0 = make_float2(0.f, 0.f), x1 = make_float2(0.f, 0.f);
    if (row < nrows) x0 = a.cgrid[(size_t)row * NH + mm];
    if (row + 1 < nrows) x1 = a.cgrid[(size_t)(row + 1) * NH + mm];
    if (!lo) {
      x0.y = -x0.y;
      x1.y = -x1.y;
    }
    A[l * LD + sk(m)] = make_float2(x0.x - x1.y, x0.y + x1.x);
  }
  __syncthreads();
  const float2* R = fft_run_t<N, 0, 1, true>(A, B, tw, nl);
  for (int idx = threadIdx.x; idx < nl * N; idx += kFftThreads) {
    const int l = idx / N, x = idx - l * N;
    const int row = r0 + 2 * l;
    const float2 v = R[l * LD + sk(x)];
    if (row < nrows) a.grid[(size_t)row * N + x] = v.x;
    if (row + 1 < nrows) a.grid[(size_t)(row + 1) * N + x] = v.y;
  }
}

// ------------------------------------------------------------------ plane FFTs
// One CTA per z-plane of a grid with Kx = Ky = N: the x transform (two real rows per
// complex line) and the y transform of the whole plane in shared memory, so the plane
// is read and written once, in whole rows (the separate x and y passes each read and
// wrote the complex grid).  The stage below is the Stockham stage above with compile-
// time element stride ES and line stride LS; for strided lines (ES > 1) consecutive
// threads take consecutive lines, so their shared-memory accesses are consecutive.
constexpr int kPlaneThreads = 1024;

template <int N, int R, int NS, bool INV, int ES, int LS, int NL>
__device__ __forceinline__ void fft_stage_g(const float2* x, float2* y, const float2* tw) {
  constexpr int NB = N / R, STEP = N / (NS * R);
  for (int idx = threadIdx.x; idx < NL * NB; idx += kPlaneThreads) {
    int l, j;
    if constexpr (ES == 1) {
      l = idx / NB;
      j = idx - l * NB;
    } else {
      j = idx / NL;
      l = idx - j * NL;
    }
    const int k = j % NS;
    const float2* xl = x + l * LS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = xl[ES == 1 ? sk(j + r * NB) : (j + r * NB) * ES];
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * k * STEP];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    small_dft<R, INV>(v);
    float2* yl = y + l * LS;
    const int o = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) yl[ES == 1 ? sk(o + r * NS) : (o + r * NS) * ES] = v[r];
  }
}

template <int N, int S, int NS, bool INV, int ES, int LS, int NL>
__device__ __forceinline__ float2* fft_run_g(float2* a, float2* b, const float2* tw) {
  if constexpr (S == nstages(N)) {
    return a;
  } else {
    constexpr int R = radix_at(N, S);
    fft_stage_g<N, R, NS, INV, ES, LS, NL>(a, b, tw);
    __syncthreads();
    return fft_run_g<N, S + 1, NS * R, INV, ES, LS, NL>(b, a, tw);
  }
}

// rows pair up as (2l, 2l+1); an odd N leaves the last line with one row and a zero
template <int N>
__host__ __device__ constexpr int plane_words() {
  constexpr int NH = N / 2 + 1, LD = fft_ld(N), NP = (N + 1) / 2;
  return (N * NH > NP * LD) ? N * NH : NP * LD;
}
template <int N>
constexpr size_t plane_smem_bytes() {
  return (size_t)(N + 2 * plane_words<N>()) * sizeof(float2);
}

// forward: real plane z -> half spectrum along x, full spectrum along y, cgrid[z][y][mx]
template <int N>
__device__ __forceinline__ void fft_xy_plane_body(const PmeArgs& a, int z) {
  griddep_wait();
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N), NH = N / 2 + 1, NP = (N + 1) / 2, W = plane_words<N>();
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + W;
  load_tw(tw, a.tw[0], N);
  const size_t row0 = (size_t)z * N;
  for (int idx = threadIdx.x; idx < NP * N; idx += kPlaneThreads) {
    const int l = idx / N, x = idx - l * N;
    A[l * LD + sk(x)] = make_float2(charge_at(a, (row0 + 2 * l) * N + x),
                                2 * l + 1 < N ? charge_at(a, (row0 + 2 * l + 1) * N + x) : 0.f);
  }
  __syncthreads();
  float2* R = fft_run_g<N, 0, 1, false, 1, LD, NP>(A, B, tw);
  float2* P = (R == A) ? B : A;  // plane [y][mx], row length NH
  for (int idx = threadIdx.x; idx < NP * NH; idx += kPlaneThreads) {
    const int l = idx / NH, m = idx - l * NH;
    const float2 u = R[l * LD + sk(m)], w = R[l * LD + sk(m == 0 ? 0 : N - m)];
    P[(2 * l) * NH + m] = make_float2(0.5f * (u.x + w.x), 0.5f * (u.y - w.y));
    if (2 * l + 1 < N) P[(2 * l + 1) * NH + m] = make_float2(0.5f * (u.y + w.y), 0.5f * (w.x - u.x));
  }
  __syncthreads();
  // the y twiddles equal the x twiddles (Kx = Ky)
  const float2* Q = fft_run_g<N, 0, 1, false, NH, 1, NH>(P, R, tw);
  for (int idx = threadIdx.x; idx < N * NH; idx += kPlaneThreads) a.cgrid[row0 * NH + idx] = Q[idx];
}

// inverse: cgrid[z][y][mx] -> inverse y, then two rows per complex line through the
// inverse x transform -> real potential plane z
template <int N>
__device__ __forceinline__ void fft_yx_plane_body(const PmeArgs& a, int z) {
  griddep_wait();
  extern __shared__ float2 sm[];
  constexpr int LD = fft_ld(N), NH = N / 2 + 1, NP = (N + 1) / 2, W = plane_words<N>();
  float2* tw = sm;
  float2* A = sm + N;
  float2* B = A + W;
  load_tw(tw, a.tw[0], N);
  const size_t row0 = (size_t)z * N;
  for (int idx = threadIdx.x; idx < N * NH; idx += kPlaneThreads) A[idx] = a.cgrid[row0 * NH + idx];
  __syncthreads();
  float2* Q = fft_run_g<N, 0, 1, true, NH, 1, NH>(A, B, tw);
  float2* L = (Q == A) ? B : A;  // complex lines of row pairs, length N, stride LD
  for (int idx = threadIdx.x; idx < NP * N; idx += kPlaneThreads) {
    const int l = idx / N, m = idx - l * N;
    const bool lo = m < NH;
    const int mm = lo ? m : N - m;
    float2 x0 = Q[(2 * l) * NH + mm];
    float2 x1 = 2 * l + 1 < N ? Q[(2 * l + 1) * NH + mm] : make_float2(0.f, 0.f);
    if (!lo) {
      x0.y = -x0.y;
      x1.y = -x1.y;
    }
    L[l * LD + sk(m)] = make_float2(x0.x - x1.y, x0.y + x1.x);
  }
  __syncthreads();
  const float2* R = fft_run_g<N, 0, 1, true, 1, LD, NP>(L, Q, tw);
  for (int idx = threadIdx.x; idx < NP * N; idx += kPlaneThreads) {
    const int l = idx / N, x = idx - l * N;
    const float2 v = R[l * LD + sk(x)];
    a.grid[(row0 + 2 * l) * N + x] = v.x;
    if (2 * l + 1 < N) a.grid[(row0 + 2 * l + 1) * N + x] = v.y;
  }
}

template <int N>
__global__ void __launch_bounds__(kPlaneThreads) k_fft_xy_plane(PmeArgs a) { griddep_wait(); fft_xy_plane_body<N>(a, blockIdx.x); }
template <int N>
__global__ void __launch_bounds__(kPlaneThreads) k_fft_yx_plane(PmeArgs a) { griddep_wait(); fft_yx_plane_body<N>(a, blockIdx.x); }
template <int N>
__global__ void __launch_bounds__(kPlaneThreads) k_fft_xy_plane_b(const PmeArgs* __restrict__ args,
                                                                  const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  fft_xy_plane_body<N>(a, t.y);
}
template <int N>
__global__ void __launch_bounds__(kPlaneThreads) k_fft_yx_plane_b(const PmeArgs* __restrict__ args,
                                                                  const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  fft_yx_plane_body<N>(a, t.y);
}

#define FZ_FFT_SIZES(X) \
  X(16) X(18) X(20) X(24) X(25) X(27) X(30) X(32) X(36) X(40) X(45) X(48) X(50) X(54) X(60) X(64) X(72) X(80) \
  X(90) X(96) X(100) X(108) X(120) X(128)

static bool fft_x_r2c_t(const PmeArgs& a, int nl, dim3 g, size_t sm, cudaStream_t st) {
  switch (a.K[0]) {
#define FZ_C(N) case N: launch_pdl(k_fft_x_r2c_t<N>, dim3(g), dim3(256), sm, st, a, nl); return true;
    FZ_FFT_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}
static bool fft_y_t(const PmeArgs& a, int nl, bool inv, dim3 g, size_t sm, cudaStream_t st) {
  switch (a.K[1]) {
#define FZ_C(N)                                                   \
  case N:                                                         \
    if (inv) launch_pdl(k_fft_y_t<N, true>, dim3(g), dim3(256), sm, st, a, nl);        \
    else launch_pdl(k_fft_y_t<N, false>, dim3(g), dim3(256), sm, st, a, nl);           \
    return true;
    FZ_FFT_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}
static bool fft_z_t(const PmeArgs& a, int nl, bool energy, dim3 g, size_t sm, cudaStream_t st) {
  switch (a.K[2]) {
#define FZ_C(N)                                                      \
  case N:                                                            \
    if (energy) launch_pdl(k_fft_z_conv_t<N, true>, dim3(g), dim3(256), sm, st, a, nl);   \
    else launch_pdl(k_fft_z_conv_t<N, false>, dim3(g), dim3(256), sm, st, a, nl);         \
    return true;
    FZ_FFT_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}
// plane kernels for grids with Kx = Ky of the compiled sizes; false if not available
#define FZ_PLANE_SIZES(X) FZ_FFT_SIZES(X)
static bool use_plane_fft(const PmeArgs& a) {
  static const bool on = !std::getenv("FZ_PLANE_FFT") || std::atoi(std::getenv("FZ_PLANE_FFT")) != 0;
  if (!on || a.K[0] != a.K[1]) return false;
  switch (a.K[0]) {
#define FZ_C(N) case N: return true;
    FZ_PLANE_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}
static void fft_plane(const PmeArgs& a, bool inverse, cudaStream_t st) {
  switch (a.K[0]) {
#define FZ_C(N)                                                                                        \
  case N: {                                                                                            \
    constexpr size_t sm = plane_smem_bytes<N>();                                                       \
    static const bool attr = [] {                                                                      \
      cudaFuncSetAttribute(k_fft_xy_plane<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);   \
      cudaFuncSetAttribute(k_fft_yx_plane<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);   \
      return true;                                                                                     \
    }();                                                                                               \
    (void)attr;                                                                                        \
    if (inverse) launch_pdl(k_fft_yx_plane<N>, dim3(a.K[2]), dim3(kPlaneThreads), sm, st, a);                              \
    else launch_pdl(k_fft_xy_plane<N>, dim3(a.K[2]), dim3(kPlaneThreads), sm, st, a);                                      \
    return;                                                                                            \
  }
    FZ_PLANE_SIZES(FZ_C)
#undef FZ_C
  }
}

static bool fft_size_compiled(int n) {
  switch (n) {
#define FZ_C(N) case N: return true;
    FZ_FFT_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}

static bool fft_x_c2r_t(const PmeArgs& a, int nl, dim3 g, size_t sm, cudaStream_t st) {
  switch (a.K[0]) {
#define FZ_C(N) case N: launch_pdl(k_fft_x_c2r_t<N>, dim3(g), dim3(256), sm, st, a, nl); return true;
    FZ_FFT_SIZES(FZ_C)
#undef FZ_C
  }
  return false;
}

static FftPlan make_plan(int n) {
  FftPlan p{};
  p.n = n;
  int m = n;
  while (m % 4 == 0 && p.nrad < 12) { p.rad[p.nrad++] = 4; m /= 4; }
  while (m % 2 == 0 && p.nrad < 12) { p.rad[p.nrad++] = 2; m /= 2; }
  while (m % 3 == 0 && p.nrad < 12) { p.rad[p.nrad++] = 3; m /= 3; }
  while (m % 5 == 0 && p.nrad < 12) { p.rad[p.nrad++] = 5; m /= 5; }
  return p;  // m == 1 checked by the caller (grid sizes are 2^a 3^b 5^c)
}

static int lines_for(int n) { return fft_lines_per_block(n); }

// largest mean atoms per brick for which the gather runs one CTA per brick (measured:
// 18 atoms per brick, 9,000 atoms on 48^3, 2.7 % faster per step; 450 per brick,
// 230,400 atoms on 128^3, 0.4 % slower than one thread per atom)
constexpr int kGatherBrickAtoms = 128;

// zero, bin, scan, scatter, spread, 3 or 5 FFT kernels, gather
// gather / spread mode: FZ_PME_GATHER overrides the tuned one (0 by atoms per brick,
// 1 brick gather, 2 per-atom gather in brick order, 3 atom spread and atom gather)
static int pme_mode(const PmeArgs& a) {
  const char* gv = std::getenv("FZ_PME_GATHER");
  return gv ? std::max(0, std::min(3, std::atoi(gv))) : a.gather;
}

int pme_launches(const PmeArgs& a) {
  return (pme_mode(a) == 3 ? 1 : 5) + (use_plane_fft(a) ? 3 : 5) + 1;
}

void launch_pme(const PmeArgs& a_in, bool energy, cudaStream_t st) {
  PmeArgs a = a_in;
  a.gather = pme_mode(a_in);
  const int nbr = a.nb[0] * a.nb[1] * a.nb[2];
  const size_t sp = (size_t)(a.B[0] + 3) * (a.B[1] + 3) * (a.B[2] + 3) * sizeof(int);
  if (a.gather == 3) {
    cudaMemsetAsync(a.grid, 0, (size_t)a.K[0] * a.K[1] * a.K[2] * sizeof(float), st);
    launch_pdl(k_pme_spread_atoms, dim3((4 * a.n + 255) / 256), dim3(256), 0, st, a);
  } else {
    launch_pdl(k_pme_zero, dim3((nbr + 255) / 256), dim3(256), 0, st, a);
    launch_pdl(k_pme_bin, dim3((a.n + 255) / 256), dim3(256), 0, st, a);
    launch_pdl(k_pme_scan, dim3(1), dim3(1024), 0, st, a);
    launch_pdl(k_pme_scatter, dim3((a.n + 255) / 256), dim3(256), 0, st, a);
    cudaMemsetAsync(a.grid, 0, (size_t)a.K[0] * a.K[1] * a.K[2] * sizeof(float), st);
    launch_pdl(k_pme_spread, dim3(nbr), dim3(256), sp, st, a);
  }
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2], Kxh = Kx / 2 + 1;
  const FftPlan px = make_plan(Kx), py = make_plan(Ky), pz = make_plan(Kz);
  const int lx = lines_for(Kx), ly = lines_for(Ky), lz = lines_for(Kz);
  const int rows = Ky * Kz;
  // runtime-plan kernels: lines n + 1 apart; compile-time kernels: fft_ld(n) apart
  const size_t smx = (size_t)(Kx + 2 * lx * (Kx + 1)) * sizeof(float2);
  const size_t smy = (size_t)(Ky + 2 * ly * (Ky + 1)) * sizeof(float2);
  const size_t smz = (size_t)(Kz + 2 * lz * (Kz + 1)) * sizeof(float2);
  const size_t smx_t = (size_t)(Kx + 2 * lx * fft_ld(Kx)) * sizeof(float2);
  const size_t smy_t = (size_t)(Ky + 2 * ly * fft_ld(Ky)) * sizeof(float2);
  const size_t smz_t = (size_t)(Kz + 2 * lz * fft_ld(Kz)) * sizeof(float2);
  const dim3 gx((rows + lx - 1) / lx), gy(Kz * ((Kxh + ly - 1) / ly)), gz(Ky * ((Kxh + lz - 1) / lz));
  // compile-time-sized kernels where available, runtime plans otherwise
  const dim3 gx2((rows + 2 * lx - 1) / (2 * lx));  // compile-time x kernels: row pairs
  const bool plane = use_plane_fft(a);
  if (plane) {
    fft_plane(a, false, st);
  } else {
    if (!fft_x_r2c_t(a, lx, gx2, smx_t, st)) launch_pdl(k_fft_x_r2c, dim3(gx), dim3(256), smx, st, a, px, lx);
    if (!fft_y_t(a, ly, false, gy, smy_t, st)) launch_pdl(k_fft_y, dim3(gy), dim3(256), smy, st, a, py, ly, 0);
  }
  if (!fft_z_t(a, lz, energy, gz, smz_t, st)) {
    if (energy)
      launch_pdl(k_fft_z_conv<true>, dim3(gz), dim3(256), smz, st, a, pz, lz);
    else
      launch_pdl(k_fft_z_conv<false>, dim3(gz), dim3(256), smz, st, a, pz, lz);
  }
  if (plane) {
    fft_plane(a, true, st);
  } else {
    if (!fft_y_t(a, ly, true, gy, smy_t, st)) launch_pdl(k_fft_y, dim3(gy), dim3(256), smy, st, a, py, ly, 1);
    if (!fft_x_c2r_t(a, lx, gx2, smx_t, st)) launch_pdl(k_fft_x_c2r, dim3(gx), dim3(256), smx, st, a, px, lx);
  }
  const int gmode = a.gather;
  if (gmode == 1 || (gmode == 0 && (size_t)a.n <= (size_t)kGatherBrickAtoms * nbr))
    launch_pdl(k_pme_gather, dim3(nbr), dim3(256), sp, st, a);
  else
    launch_pdl(k_pme_gather_atoms, dim3((4 * a.n + 255) / 256), dim3(256), 0, st, a);
}

// ------------------------------------------------------------------ batched PME
// zeroes the int32 charge grid of each system (the memset of the single-system path)
__global__ void k_grid_zero_b(const PmeArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const PmeArgs a = args[t.x];
  const size_t kt = (size_t)a.K[0] * a.K[1] * a.K[2];
  int* g = reinterpret_cast<int*>(a.grid);
  for (size_t i = (size_t)t.y * blockDim.x + threadIdx.x; i < kt; i += (size_t)t.z * blockDim.x) g[i] = 0;
}

size_t pme_spread_smem(const PmeArgs& a) {
  return (size_t)(a.B[0] + 3) * (a.B[1] + 3) * (a.B[2] + 3) * sizeof(int);
}
int pme_z_groups(const PmeArgs& a) {
  const int nl = fft_lines_per_block(a.K[2]);
  return a.K[1] * ((a.K[0] / 2 + 1 + nl - 1) / nl);
}
bool pme_batchable(const PmeArgs& a) { return use_plane_fft(a) && a.K[2] == a.K[0]; }

void launch_pme_b(const PmeArgs* args, const BatchTables& t, const PmeSizeBatch* sizes, int nsizes,
                  size_t spread_smem, cudaStream_t st) {
  launch_pdl(k_pme_zero_b, dim3(t.n[BT_BRICKS256]), dim3(256), 0, st, args, t.tab[BT_BRICKS256]);
  launch_pdl(k_pme_bin_b, dim3(t.n[BT_ATOMS256]), dim3(256), 0, st, args, t.tab[BT_ATOMS256]);
  launch_pdl(k_pme_scan_b, dim3(t.n[BT_ONE]), dim3(1024), 0, st, args, t.tab[BT_ONE]);
  launch_pdl(k_pme_scatter_b, dim3(t.n[BT_ATOMS256]), dim3(256), 0, st, args, t.tab[BT_ATOMS256]);
  launch_pdl(k_grid_zero_b, dim3(t.n[BT_GRID256]), dim3(256), 0, st, args, t.tab[BT_GRID256]);
  launch_pdl(k_pme_spread_b, dim3(t.n[BT_BRICKS]), dim3(256), spread_smem, st, args, t.tab[BT_BRICKS]);
  for (int pass = 0; pass < 3; ++pass)
    for (int k = 0; k < nsizes; ++k) {
      const PmeSizeBatch& b = sizes[k];
      switch (b.N) {
#define FZ_C(N)                                                                                        \
  case N: {                                                                                            \
    constexpr size_t sm = plane_smem_bytes<N>();                                                       \
    static const bool attr = [] {                                                                      \
      cudaFuncSetAttribute(k_fft_xy_plane_b<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
      cudaFuncSetAttribute(k_fft_yx_plane_b<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
      return true;                                                                                     \
    }();                                                                                               \
    (void)attr;                                                                                        \
    constexpr int nl = fft_lines_per_block(N);                                                         \
    constexpr size_t smz = (size_t)(N + 2 * nl * fft_ld(N)) * sizeof(float2);                         \
    if (pass == 0) launch_pdl(k_fft_xy_plane_b<N>, dim3(b.nplane), dim3(kPlaneThreads), sm, st, args, b.plane_tab);       \
    if (pass == 1) launch_pdl(k_fft_z_conv_b<N>, dim3(b.nz), dim3(256), smz, st, args, b.z_tab);                           \
    if (pass == 2) launch_pdl(k_fft_yx_plane_b<N>, dim3(b.nplane), dim3(kPlaneThreads), sm, st, args, b.plane_tab);       \
    break;                                                                                             \
  }
        FZ_PLANE_SIZES(FZ_C)
#undef FZ_C
      }
    }
  launch_pdl(k_pme_gather_b, dim3(t.n[BT_BRICKS]), dim3(256), spread_smem, st, args, t.tab[BT_BRICKS]);
}

}  // namespace fzk
