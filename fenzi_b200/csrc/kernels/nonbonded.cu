// Real-space nonbonded pair kernel: CHARMM LJ with the switch from ron to rc plus
// erfc real-space Ewald, the functional form of nonbondforce (src/nonbonded_forces.cu:114-245).
//
// B200 design: one warp per tile (32 i-atoms of a sorted block x 32 j-atoms of the
// pair list).  i data stay in registers; j data (x, y, z, q, LJ type) and the j force
// accumulator rotate through the warp with shuffles, so each pair is evaluated once
// (Newton's third law) with no shared-memory traffic.  Forces are converted to int64
// fixed point at the end of each tile and added with RED atomics: the result does not
// depend on tile order, so forces are bit-reproducible run to run.
//
// erfc uses Abramowitz & Stegun, Handbook of Mathematical Functions (1964), eq. 7.1.26
// (|error| <= 1.5e-7), which shares its exp(-x^2) with the force term.
// The LJ switch derivative is the exact one; the reference's force expression
// (src/nonbonded_forces.cu:210-214) carries an extra Swcoeff2*invDist term.
#include "common.cuh"
#include "kernels.h"

namespace fzk {

constexpr float kAS_p = 0.3275911f;
constexpr float kAS_a1 = 0.254829592f;
constexpr float kAS_a2 = -0.284496736f;
constexpr float kAS_a3 = 1.421413741f;
constexpr float kAS_a4 = -1.453152027f;
constexpr float kAS_a5 = 1.061405429f;
constexpr float kTwoOverSqrtPi = 1.1283791670955126f;

template <bool ENERGY>
__global__ void __launch_bounds__(256, 3)
    k_nonbonded(SysParams p, const float4* __restrict__ xyzq, const int* __restrict__ typ,
                const int* __restrict__ perm, const int* __restrict__ tile_i, const uint32_t* __restrict__ tile_j,
                const int* __restrict__ tile_m, const uint32_t* __restrict__ masks, const int* __restrict__ counters,
                const float2* __restrict__ ljtab, long long* __restrict__ facc, long long* __restrict__ energy,
                int tile_cap) {
  extern __shared__ float2 lj[];
  const int nt1 = p.ntypes + 1;
  for (int k = threadIdx.x; k < nt1 * nt1; k += blockDim.x) lj[k] = ljtab[k];
  __syncthreads();
  const int ntiles = min(counters[CNT_TILES], tile_cap);
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  const float rc2 = p.rc2, ron2 = p.ron2, c3 = p.sw_c3;
  const float c2 = rc2 - 3.f * ron2;
  const float beta = p.beta;
  const float bc = beta * kTwoOverSqrtPi;
  const int n = p.n;
  double e_vdw = 0.0, e_el = 0.0;
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntiles; t += nwarps) {
    const int ti = tile_i[t];
    const bool diag = ti < 0;
    const int I = ti & 0x7fffffff;
    const int islot = I * 32 + lane;
    const float4 xi = xyzq[islot];
    const int tyi = typ[islot] * nt1;
    const float qi = xi.w * p.cc;
    const uint32_t je = tile_j[(size_t)t * 32 + lane];
    const int jslot = (int)(je & kSlotMask);
    const int code = (int)(je >> kSlotBits);
    float4 xj = xyzq[jslot];
    if (code != kNoShift) {
      const float3 s = shift_of(code, p);
      xj.x += s.x;
      xj.y += s.y;
      xj.z += s.z;
    }
    int tyj = typ[jslot];
    const int m = tile_m[t];
    uint32_t excl = m >= 0 ? masks[(size_t)m * 32 + lane] : 0u;
    if (diag) excl |= (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);  // j <= i
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float fjx = 0.f, fjy = 0.f, fjz = 0.f;
    float ev = 0.f, ee = 0.f;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const int jl = (lane + k) & 31;
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const bool ok = (r2 < rc2) && !((excl >> jl) & 1u);
      const float rinv = rsqrtf(r2);
      const float r2inv = rinv * rinv;
      // Coulomb, erfc real-space Ewald
      const float qq = qi * xj.w;
      const float br = beta * r2 * rinv;
      const float tt = __fdividef(1.f, fmaf(kAS_p, br, 1.f));
      const float ex = __expf(-br * br);
      const float poly = tt * fmaf(tt, fmaf(tt, fmaf(tt, fmaf(tt, kAS_a5, kAS_a4), kAS_a3), kAS_a2), kAS_a1);
      const float ec = qq * poly * ex * rinv;
      const float fc = fmaf(qq * bc, ex, ec) * r2inv;
      // Lennard-Jones with CHARMM switch
      const float2 ls = lj[tyi + tyj];
      const float s2 = ls.y * r2inv;
      const float s6 = s2 * s2 * s2;
      const float a = ls.x * s6;
      const float b = a * s6;
      const float elj = b - a;
      const float flj = fmaf(12.f, b, -6.f * a) * r2inv;
      const float u = rc2 - r2;
      const bool on = r2 > ron2;
      const float sw = on ? u * u * fmaf(2.f, r2, c2) * c3 : 1.f;
      const float dsw = on ? 12.f * u * (r2 - ron2) * c3 : 0.f;
      float fr = fmaf(flj, sw, fmaf(elj, dsw, fc));
      fr = ok ? fr : 0.f;
      fix = fmaf(fr, dx, fix);
      fiy = fmaf(fr, dy, fiy);
      fiz = fmaf(fr, dz, fiz);
      fjx = fmaf(-fr, dx, fjx);
      fjy = fmaf(-fr, dy, fjy);
      fjz = fmaf(-fr, dz, fjz);
      if (ENERGY) {
        ev += ok ? elj * sw : 0.f;
        ee += ok ? ec : 0.f;
      }
      // rotate j data and j force one lane down
      const int src = (lane + 1) & 31;
      xj.x = __shfl_sync(0xffffffffu, xj.x, src);
      xj.y = __shfl_sync(0xffffffffu, xj.y, src);
      xj.z = __shfl_sync(0xffffffffu, xj.z, src);
      xj.w = __shfl_sync(0xffffffffu, xj.w, src);
      tyj = __shfl_sync(0xffffffffu, tyj, src);
      fjx = __shfl_sync(0xffffffffu, fjx, src);
      fjy = __shfl_sync(0xffffffffu, fjy, src);
      fjz = __shfl_sync(0xffffffffu, fjz, src);
    }
    const int ai = perm[islot];
    if (ai >= 0) {
      red_add(facc + ai, to_fix(fix));
      red_add(facc + n + ai, to_fix(fiy));
      red_add(facc + 2 * n + ai, to_fix(fiz));
    }
    const int aj = perm[jslot];
    if (aj >= 0) {
      red_add(facc + aj, to_fix(fjx));
      red_add(facc + n + aj, to_fix(fjy));
      red_add(facc + 2 * n + aj, to_fix(fjz));
    }
    if (ENERGY) {
      e_vdw += (double)ev;
      e_el += (double)ee;
    }
  }
  if (ENERGY) {
    energy_add(energy + EN_VDW, e_vdw);
    energy_add(energy + EN_ELEC, e_el);
  }
}

void launch_nonbonded(const NonbondedArgs& a, bool energy, cudaStream_t st) {
  const int nt1 = a.p.ntypes + 1;
  const size_t smem = (size_t)nt1 * nt1 * sizeof(float2);
  if (energy)
    k_nonbonded<true><<<a.grid, 256, smem, st>>>(a.p, a.xyzq_s, a.typ_s, a.perm, a.tile_i, a.tile_j, a.tile_m,
                                                 a.masks, a.counters, a.ljtab, a.facc, a.energy, a.tile_cap);
  else
    k_nonbonded<false><<<a.grid, 256, smem, st>>>(a.p, a.xyzq_s, a.typ_s, a.perm, a.tile_i, a.tile_j, a.tile_m,
                                                  a.masks, a.counters, a.ljtab, a.facc, a.energy, a.tile_cap);
}

}  // namespace fzk
