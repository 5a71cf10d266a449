// Smooth PME, order 4: charge spreading, hand-written 3-D R2C/C2R FFT with the
// influence function fused between the forward and inverse z passes, force gather.
// Replaces ChargeSpread_small/_medium (src/pme_kernels.cu:20-239), the cuFFT C2C
// pair and BCMultiply (src/mdcuda.cu:748,780, src/cell_based_kernels.cu:1770-1826)
// and PMEForce_medium/_large (src/pme_kernels.cu:381-770).
//
// Spreading is owner-computes: the grid is cut into bricks, atoms are binned by the
// brick of their base grid point every step, and one CTA per brick accumulates the
// order-4 B-spline weights of the atoms of that brick and of the next brick in each
// dimension into shared memory with int64 fixed-point atomics (order independent, so
// the grid is bit-reproducible), then writes its brick with plain stores.  No global
// atomics, no per-grid-point lists.  B-splines are evaluated analytically (the
// reference samples a 1001-point table with a truncating index).
#include "common.cuh"
#include "kernels.h"

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

__global__ void k_pme_zero(int* cnt, int* cur, int nb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    cnt[i] = 0;
    cur[i] = 0;
  }
}

__global__ void k_pme_bin(PmeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

__global__ void k_pme_scan(PmeArgs a, int nbr) {
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

__global__ void k_pme_scatter(PmeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

// charge-grid accumulation in shared memory: int32 fixed point, 2^24 per e (values
// stay far below the +-128 e range a grid point could hold), native shared atomics
constexpr float kFixQ32 = 16777216.0f;

__global__ void __launch_bounds__(128) k_pme_spread(PmeArgs a) {
  extern __shared__ int acc[];
  const int Bx = a.B[0], By = a.B[1], Bz = a.B[2];
  const int nbx = a.nb[0], nby = a.nb[1], nbz = a.nb[2];
  const int b = blockIdx.x;
  const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const int vol = Bx * By * Bz;
  for (int k = threadIdx.x; k < vol; k += blockDim.x) acc[k] = 0;
  __syncthreads();
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  const int ox = bx * Bx, oy = by * By, oz = bz * Bz;
  const int sdx = nbx > 1 ? 2 : 1, sdy = nby > 1 ? 2 : 1, sdz = nbz > 1 ? 2 : 1;
  for (int dz = 0; dz < sdz; ++dz)
    for (int dy = 0; dy < sdy; ++dy)
      for (int dx = 0; dx < sdx; ++dx) {
        const int sb = (((bz + dz) % nbz) * nby + (by + dy) % nby) * nbx + (bx + dx) % nbx;
        const int s0 = a.brick_start[sb], s1 = a.brick_start[sb + 1];
        for (int idx = s0 + threadIdx.x; idx < s1; idx += blockDim.x) {
          const int i = a.brick_atoms[idx];
          const float4 r = a.pos4[i];
          float tx, ty, tz, wx[4], wy[4], wz[4];
          const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx);
          const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty);
          const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz);
          bsp4(tx, wx, nullptr);
          bsp4(ty, wy, nullptr);
          bsp4(tz, wz, nullptr);
          const float q = r.w;
          // local offsets of grid points k0 - j inside this brick (k0 - j - o lies in
          // (-K, K) so one conditional wrap suffices); >= B means another brick owns it
          int lxs[4], lys[4], lzs[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            int vx = kx - j - ox, vy = ky - j - oy, vz = kz - j - oz;
            vx += vx < 0 ? Kx : 0;
            vy += vy < 0 ? Ky : 0;
            vz += vz < 0 ? Kz : 0;
            lxs[j] = vx;
            lys[j] = vy;
            lzs[j] = vz;
          }
#pragma unroll
          for (int jz = 0; jz < 4; ++jz) {
            if (lzs[jz] >= Bz) continue;
#pragma unroll
            for (int jy = 0; jy < 4; ++jy) {
              if (lys[jy] >= By) continue;
              const float qzy = q * wz[jz] * wy[jy];
              int* rowp = &acc[(lzs[jz] * By + lys[jy]) * Bx];
#pragma unroll
              for (int jx = 0; jx < 4; ++jx) {
                if (lxs[jx] >= Bx) continue;
                atomicAdd(rowp + lxs[jx], __float2int_rn(qzy * wx[jx] * kFixQ32));
              }
            }
          }
        }
      }
  __syncthreads();
  for (int k = threadIdx.x; k < vol; k += blockDim.x) {
    const int lx = k % Bx, ly = (k / Bx) % By, lz = k / (Bx * By);
    a.grid[((size_t)(oz + lz) * Ky + (oy + ly)) * Kx + (ox + lx)] = (float)acc[k] * (1.0f / kFixQ32);
  }
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
__global__ void __launch_bounds__(256) k_fft_x_r2c(PmeArgs a, FftPlan pl, int nl) {
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
    A[l * ld + x] = make_float2(row < nrows ? a.grid[(size_t)row * Kx + x] : 0.f, 0.f);
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
__global__ void __launch_bounds__(256) k_fft_y(PmeArgs a, FftPlan pl, int nl, int inv) {
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
__global__ void __launch_bounds__(256) k_fft_z_conv(PmeArgs a, FftPlan pl, int nl) {
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
  double e = 0.0;
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
    if (ENERGY && mx < Kxh) {
      const double wmx = (mx == 0 || (2 * mx == Kx)) ? 1.0 : 2.0;
      e += wmx * 0.5 * (double)G * ((double)v.x * v.x + (double)v.y * v.y);
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
  if (ENERGY) energy_add(a.energy + EN_PME, e);
}

// x pass inverse: Hermitian half rows -> real potential rows
__global__ void __launch_bounds__(256) k_fft_x_c2r(PmeArgs a, FftPlan pl, int nl) {
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

// one thread per atom, atoms taken in brick order so a warp reads neighbouring grid lines
__global__ void __launch_bounds__(256) k_pme_gather(PmeArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const int i = a.brick_atoms[t];
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2];
  const float4 r = a.pos4[i];
  float tx, ty, tz, wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
  const int kx = grid_base(r.x, a.p.inv_box.x, Kx, &tx);
  const int ky = grid_base(r.y, a.p.inv_box.y, Ky, &ty);
  const int kz = grid_base(r.z, a.p.inv_box.z, Kz, &tz);
  bsp4(tx, wx, dx);
  bsp4(ty, wy, dy);
  bsp4(tz, wz, dz);
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int jz = 0; jz < 4; ++jz) {
    int z = kz - jz;
    z += z < 0 ? Kz : 0;
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
        const float phi = __ldg(row + x);
        sx = fmaf(wx[jx], phi, sx);
        sdx = fmaf(dx[jx], phi, sdx);
      }
      gx = fmaf(sdx, wy[jy] * wz[jz], gx);
      gy = fmaf(sx, dy[jy] * wz[jz], gy);
      gz = fmaf(sx, wy[jy] * dz[jz], gz);
    }
  }
  const float q = r.w;
  const int n = a.n;
  red_add(a.facc + i, to_fix(-q * gx * (float)Kx * a.p.inv_box.x));
  red_add(a.facc + n + i, to_fix(-q * gy * (float)Ky * a.p.inv_box.y));
  red_add(a.facc + 2 * n + i, to_fix(-q * gz * (float)Kz * a.p.inv_box.z));
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

static int lines_for(int n) { return n >= 256 ? 8 : (n >= 128 ? 16 : 32); }

void launch_pme(const PmeArgs& a, bool energy, cudaStream_t st) {
  const int nbr = a.nb[0] * a.nb[1] * a.nb[2];
  k_pme_zero<<<(nbr + 255) / 256, 256, 0, st>>>(a.brick_count, a.brick_cursor, nbr);
  k_pme_bin<<<(a.n + 255) / 256, 256, 0, st>>>(a);
  k_pme_scan<<<1, 1024, 0, st>>>(a, nbr);
  k_pme_scatter<<<(a.n + 255) / 256, 256, 0, st>>>(a);
  const size_t sp = (size_t)a.B[0] * a.B[1] * a.B[2] * sizeof(int);
  k_pme_spread<<<nbr, 128, sp, st>>>(a);
  const int Kx = a.K[0], Ky = a.K[1], Kz = a.K[2], Kxh = Kx / 2 + 1;
  const FftPlan px = make_plan(Kx), py = make_plan(Ky), pz = make_plan(Kz);
  const int lx = lines_for(Kx), ly = lines_for(Ky), lz = lines_for(Kz);
  const int rows = Ky * Kz;
  const size_t smx = (size_t)(Kx + 2 * lx * (Kx + 1)) * sizeof(float2);
  const size_t smy = (size_t)(Ky + 2 * ly * (Ky + 1)) * sizeof(float2);
  const size_t smz = (size_t)(Kz + 2 * lz * (Kz + 1)) * sizeof(float2);
  k_fft_x_r2c<<<(rows + lx - 1) / lx, 256, smx, st>>>(a, px, lx);
  k_fft_y<<<Kz * ((Kxh + ly - 1) / ly), 256, smy, st>>>(a, py, ly, 0);
  if (energy)
    k_fft_z_conv<true><<<Ky * ((Kxh + lz - 1) / lz), 256, smz, st>>>(a, pz, lz);
  else
    k_fft_z_conv<false><<<Ky * ((Kxh + lz - 1) / lz), 256, smz, st>>>(a, pz, lz);
  k_fft_y<<<Kz * ((Kxh + ly - 1) / ly), 256, smy, st>>>(a, py, ly, 1);
  k_fft_x_c2r<<<(rows + lx - 1) / lx, 256, smx, st>>>(a, px, lx);
  k_pme_gather<<<(a.n + 255) / 256, 256, 0, st>>>(a);
}

}  // namespace fzk
