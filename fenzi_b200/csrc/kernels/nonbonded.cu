// Real-space nonbonded pair kernel: CHARMM LJ with the switch from ron to rc plus
// erfc real-space Ewald, the functional form of nonbondforce (src/nonbonded_forces.cu:114-245).
//
// B200 design: one warp per tile (32 i-atoms of a sorted block x 32 j-atoms of the
// pair list), each pair evaluated once (Newton's third law).  i data live in
// registers; the tile's j data (x, y, z, q, LJ type, periodic image applied) are
// staged once into a doubled 64-entry shared-memory ring, so at step k lane l reads
// j = l + k with a constant-offset load and no wrap arithmetic; only the j force
// accumulator rotates through the warp (3 shuffles per pair step).  Tiles without
// excluded pairs (the large majority) run a mask-free loop.  The kernel is FP32-issue
// bound, so every pair-step instruction counts:
//   erfc(x) = t P(t) exp(-x^2), t = 1/(1 + p x)  (Abramowitz & Stegun, Handbook of
//     Mathematical Functions (1964) eq. 7.1.26, |error| <= 1.5e-7), with exp2 and the
//     constants pre-scaled so exp(-x^2) is one multiply and one MUFU.EX2;
//   the CHARMM switch (rc^2-r^2)^2 (rc^2+2r^2-3ron^2)/(rc^2-ron^2)^3 written as
//     1 - t^2 (3 - 2t) with t = sat((r^2-ron^2)/(rc^2-ron^2)) (identical polynomial),
//     its derivative exact (the reference's force at src/nonbonded_forces.cu:210-214
//     carries an extra Swcoeff2*invDist term);
// Forces go to int64 fixed point at the end of each tile (RED atomics, order
// independent): bit-reproducible run to run.
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
constexpr float kLog2e = 1.4426950408889634f;
constexpr int kWarps = 8;

// single-instruction MUFU approximations (PTX ISA: rsqrt/ex2/rcp .approx.ftz.f32)
__device__ __forceinline__ float rsqrt_a(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_a(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_a(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct PairConst {
  float rc2, beta, eb2;   // eb2 = -beta^2 log2(e)
  float p_b;              // p * beta
  float c2b;              // 2 beta / sqrt(pi)
  float sw_a, sw_b;       // t = sat(r2 * sw_a + sw_b)
  float dsw_k;            // 12 / (rc^2 - ron^2) / 6 (the LJ table in shared memory holds 6 eps4)
};

__host__ __device__ inline PairConst pair_const(const SysParams& p) {
  PairConst c;
  c.rc2 = p.rc2;
  c.beta = p.beta;
  c.eb2 = -p.beta * p.beta * kLog2e;
  c.p_b = kAS_p * p.beta;
  c.c2b = kTwoOverSqrtPi * p.beta;
  const float d = p.rc2 - p.ron2;
  c.sw_a = d > 0.f ? 1.f / d : 0.f;
  c.sw_b = d > 0.f ? -p.ron2 / d : 0.f;
  c.dsw_k = d > 0.f ? 2.f / d : 0.f;
  return c;
}

// force/r for one pair (FP32); returns 0 outside the cutoff or when masked.  ls.x is
// 6 eps4 (the shared-memory table is scaled by 6 when loaded), so with a6 = 6 eps4 s^6 and
// b6 = a6 s^6 the unswitched LJ force/r is (2 b6 - a6) / r^2 and the LJ energy
// (b6 - a6) / 6; both force parts share the 1 / r^2:
//   F/r = [(2 b6 - a6) sw + qq e^{-b^2 r^2} (erfc(br)/(r e^{-b^2 r^2}) + 2b/sqrt(pi))] / r^2
//         + (b6 - a6)/6 dsw
template <bool ENERGY>
__device__ __forceinline__ float pair_force(const PairConst& c, float r2, float qq, float2 ls, bool ok, float& ev,
                                            float& ee) {
  const float rinv = rsqrt_a(r2);
  const float r2inv = rinv * rinv;
  const float ex = ex2_a(r2 * c.eb2);                    // exp(-beta^2 r^2)
  const float tt = rcp_a(fmaf(c.p_b, r2 * rinv, 1.f));   // 1 / (1 + p beta r)
  const float poly = tt * fmaf(tt, fmaf(tt, fmaf(tt, fmaf(tt, kAS_a5, kAS_a4), kAS_a3), kAS_a2), kAS_a1);
  // erfc(beta r) = poly exp(-beta^2 r^2): F_C r / r^2 = qq exp(-beta^2 r^2) (poly / r + 2 beta/sqrt(pi)) / r^2
  const float qex = qq * ex;
  const float s2 = ls.y * r2inv;
  const float s6 = s2 * s2 * s2;
  const float a6 = ls.x * s6;
  const float b6 = a6 * s6;
  const float t = __saturatef(fmaf(r2, c.sw_a, c.sw_b));
  const float t2 = t * t;
  const float sw = fmaf(-t2, fmaf(-2.f, t, 3.f), 1.f);
  const float e6 = b6 - a6;
  const float h = fmaf(fmaf(2.f, b6, -a6), sw, qex * fmaf(poly, rinv, c.c2b));
  const float fr = fmaf(h, r2inv, e6 * ((t - t2) * c.dsw_k));
  if (ENERGY) {
    ev += ok ? e6 * sw * (1.f / 6.f) : 0.f;
    ee += ok ? qex * poly * rinv : 0.f;
  }
  return ok ? fr : 0.f;
}

// One tile of kIG i atoms x 32 j entries (xj, tyj: this lane's entry, loaded by the
// caller one tile ahead).  Lane = h * kIG + il holds i atom il of the
// group and works on segment h of the j entries (kIG of them); the tile's j data
// (image shift applied) are staged in this warp's shared ring, doubled within each
// segment, so at step k lane il reads entry h * kIG + (il + k) % kIG at a constant
// offset; the i force stays in registers, each j force accumulator rotates through
// its segment (3 width-kIG shuffles per step) and is back on the lane that loaded the
// entry after kIG steps.  excl: bit e set when entry e is excluded for this lane's i.
template <bool ENERGY>
__device__ __forceinline__ void run_tile(const PairConst& c, const SysParams& p, const float4& xi, float qi,
                                         const float2* ljrow, uint32_t je, uint32_t excl, float4 xj, int tyj,
                                         float4* jx, int* jt, const int* __restrict__ perm,
                                         long long* __restrict__ facc, int lane, int src, float& fix, float& fiy,
                                         float& fiz, float& ev, float& ee, float* vir) {
  const int jslot = (int)(je & kSlotMask);
  const int code = (int)(je >> kSlotBits);
  if (code != kNoShift) {
    const float3 s = shift_of(code, p);
    xj.x += s.x;
    xj.y += s.y;
    xj.z += s.z;
  }
  const int il = lane & (kIG - 1), seg = (lane / kIG) * 2 * kIG;
  __syncwarp();
  jx[seg + il] = xj;
  jx[seg + il + kIG] = xj;
  jt[seg + il] = tyj;
  jt[seg + il + kIG] = tyj;
  __syncwarp();
  // bit k of mrot: pair (il, entry h * kIG + (il + k) % kIG) excluded
  uint32_t mrot;
  if (kIG == 32) {
    mrot = __funnelshift_r(excl, excl, il);
  } else {
    const uint32_t segm = (1u << (kIG & 31)) - 1u;
    const uint32_t w = (excl >> ((lane / kIG) * kIG)) & segm;
    mrot = ((w >> il) | (w << ((kIG - il) & 31))) & segm;
  }
  const float4* jxl = jx + seg + il;
  const int* jtl = jt + seg + il;
  float fjx = 0.f, fjy = 0.f, fjz = 0.f;
  if (__any_sync(0xffffffffu, mrot != 0u)) {
#pragma unroll 8
    for (int k = 0; k < kIG; ++k) {
      const float4 b = jxl[k];
      const float dx = xi.x - b.x, dy = xi.y - b.y, dz = xi.z - b.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const bool ok = (r2 < c.rc2) && !((mrot >> k) & 1u);
      const float fr = pair_force<ENERGY>(c, r2, qi * b.w, ljrow[jtl[k]], ok, ev, ee);
      if (ENERGY) {
        vir[0] = fmaf(fr * dx, dx, vir[0]);
        vir[1] = fmaf(fr * dy, dy, vir[1]);
        vir[2] = fmaf(fr * dz, dz, vir[2]);
      }
      fix = fmaf(fr, dx, fix);
      fiy = fmaf(fr, dy, fiy);
      fiz = fmaf(fr, dz, fiz);
      fjx = __shfl_sync(0xffffffffu, fmaf(-fr, dx, fjx), src, kIG);
      fjy = __shfl_sync(0xffffffffu, fmaf(-fr, dy, fjy), src, kIG);
      fjz = __shfl_sync(0xffffffffu, fmaf(-fr, dz, fjz), src, kIG);
    }
  } else {
#pragma unroll 8
    for (int k = 0; k < kIG; ++k) {
      const float4 b = jxl[k];
      const float dx = xi.x - b.x, dy = xi.y - b.y, dz = xi.z - b.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const float fr = pair_force<ENERGY>(c, r2, qi * b.w, ljrow[jtl[k]], r2 < c.rc2, ev, ee);
      if (ENERGY) {
        vir[0] = fmaf(fr * dx, dx, vir[0]);
        vir[1] = fmaf(fr * dy, dy, vir[1]);
        vir[2] = fmaf(fr * dz, dz, vir[2]);
      }
      fix = fmaf(fr, dx, fix);
      fiy = fmaf(fr, dy, fiy);
      fiz = fmaf(fr, dz, fiz);
      fjx = __shfl_sync(0xffffffffu, fmaf(-fr, dx, fjx), src, kIG);
      fjy = __shfl_sync(0xffffffffu, fmaf(-fr, dy, fjy), src, kIG);
      fjz = __shfl_sync(0xffffffffu, fmaf(-fr, dz, fjz), src, kIG);
    }
  }
  const int aj = perm[jslot];
  if (aj >= 0) {
    const int n = p.n;
    red_add(facc + aj, to_fix(fjx));
    red_add(facc + n + aj, to_fix(fjy));
    red_add(facc + 2 * n + aj, to_fix(fjz));
  }
}

// Warp per i-block (blocks taken from a dynamic counter): the diagonal tile, then the
// block's inner tiles; the i force stays in registers across tiles and is flushed once.
template <bool ENERGY>
__device__ __forceinline__ void nonbonded_body(const SysParams& p, const PairConst& c, const float4* __restrict__ xyzq, const int* __restrict__ typ,
    const int* __restrict__ perm, const uint32_t* __restrict__ inner, const int* __restrict__ inner_nt,
    const int* __restrict__ inner_m, const uint32_t* __restrict__ dmask, const uint32_t* __restrict__ masks,
    int* __restrict__ counters, const int2* __restrict__ items, int chunk, const float2* __restrict__ ljtab,
    long long* __restrict__ facc, long long* __restrict__ energy, int ocap) {
  griddep_wait();
  extern __shared__ float2 lj[];
  __shared__ float4 jx_all[kWarps][64];
  __shared__ int jt_all[kWarps][64];
  const int nt1 = p.ntypes + 1;
  for (int k = threadIdx.x; k < nt1 * nt1; k += blockDim.x) lj[k] = make_float2(6.f * ljtab[k].x, ljtab[k].y);
  __syncthreads();
  const int nitems = counters[CNT_ITEMS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* jx = jx_all[warp];
  int* jt = jt_all[warp];
  const int n = p.n;
  const int il = lane & (kIG - 1);
  const int src = (il + 1) & (kIG - 1);  // segment-relative source lane of the j-force rotation
  // energy and virial sums per lane in fixed point, item by item: integer sums do not
  // depend on which items a warp happens to fetch, so energies are bit-reproducible
  long long e_vdw = 0, e_el = 0, w_acc[3] = {0, 0, 0};
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(&counters[CNT_WORK], 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= nitems) break;
    const int2 item = items[it];
    const int g = item.x;  // i-group: block I, atoms s * kIG .. s * kIG + kIG - 1
    const int I = g / kNG, s = g % kNG;
    const int ib = s * kIG + il;  // this lane's i atom, index within the block
    const int islot = I * 32 + ib;
    const float4 xi = xyzq[islot];
    const float2* ljrow = lj + typ[islot] * nt1;
    const float qi = xi.w * p.cc;
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float ev = 0.f, ee = 0.f, vir[3] = {0.f, 0.f, 0.f};
    // tile 0 of a group is the group against its own block (upper triangle j > i);
    // each tile's entry, exclusion word and j data are loaded one tile ahead
    int t = item.y;
    const int tend = min(inner_nt[g] + 1, t + chunk);
    const uint32_t* jl = inner + (size_t)g * ocap - 32;  // inner tile t-1
    const int* ml = inner_m + (size_t)g * (ocap >> 5) - 1;
    auto fetch = [&](int tt, uint32_t& je, uint32_t& ex, float4& xj, int& tyj) {
      if (tt == 0) {
        je = (uint32_t)(I * 32 + lane) | ((uint32_t)kNoShift << kSlotBits);
        ex = dmask[islot] | ((ib == 31) ? 0xffffffffu : ((2u << ib) - 1u));
      } else {
        je = jl[tt * 32 + lane];
        const int m = ml[tt];
        ex = m >= 0 ? masks[(size_t)m * kIG + il] : 0u;
      }
      xj = xyzq[je & kSlotMask];
      tyj = typ[je & kSlotMask];
    };
    uint32_t je_n, ex_n;
    float4 xj_n;
    int ty_n;
    fetch(t, je_n, ex_n, xj_n, ty_n);
    for (; t < tend; ++t) {
      const uint32_t je = je_n, ex = ex_n;
      const float4 xj = xj_n;
      const int ty = ty_n;
      if (t + 1 < tend) fetch(t + 1, je_n, ex_n, xj_n, ty_n);
      run_tile<ENERGY>(c, p, xi, qi, ljrow, je, ex, xj, ty, jx, jt, perm, facc, lane, src, fix, fiy, fiz, ev, ee,
                       vir);
    }
    // the i force of lane il is split over the 32 / kIG segments
#pragma unroll
    for (int off = kIG; off < 32; off <<= 1) {
      fix += __shfl_xor_sync(0xffffffffu, fix, off);
      fiy += __shfl_xor_sync(0xffffffffu, fiy, off);
      fiz += __shfl_xor_sync(0xffffffffu, fiz, off);
    }
    const int ai = perm[islot];
    if (lane < kIG && ai >= 0) {
      red_add(facc + ai, to_fix(fix));
      red_add(facc + n + ai, to_fix(fiy));
      red_add(facc + 2 * n + ai, to_fix(fiz));
    }
    if (ENERGY) {
      e_vdw += __double2ll_rn((double)ev * kFixE);
      e_el += __double2ll_rn((double)ee * kFixE);
      for (int d = 0; d < 3; ++d) w_acc[d] += __double2ll_rn((double)vir[d] * kFixE);
    }
  }
  if (ENERGY) {
    energy_add_fix(energy + EN_VDW, e_vdw);
    energy_add_fix(energy + EN_ELEC, e_el);
    energy_add_fix(energy + EN_VIR_X, w_acc[0]);
    energy_add_fix(energy + EN_VIR_Y, w_acc[1]);
    energy_add_fix(energy + EN_VIR_Z, w_acc[2]);
  }
}

template <bool ENERGY, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_nonbonded(SysParams p, PairConst c, const float4* __restrict__ xyzq, const int* __restrict__ typ,
                const int* __restrict__ perm, const uint32_t* __restrict__ inner, const int* __restrict__ inner_nt,
                const int* __restrict__ inner_m, const uint32_t* __restrict__ dmask,
                const uint32_t* __restrict__ masks, int* __restrict__ counters, const int2* __restrict__ items,
                int chunk, const float2* __restrict__ ljtab, long long* __restrict__ facc,
                long long* __restrict__ energy, int ocap) { griddep_wait();
  nonbonded_body<ENERGY>(p, c, xyzq, typ, perm, inner, inner_nt, inner_m, dmask, masks, counters, items, chunk, ljtab,
                         facc, energy, ocap);
}

// batched: every CTA serves one system's work queue (force variant only)
__global__ void __launch_bounds__(256, kNbBatchCtasPerSm) k_nonbonded_b(const NonbondedArgs* __restrict__ args,
                                                        const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const NonbondedArgs a = args[t.x];
  const PairConst c = pair_const(a.p);
  nonbonded_body<false>(a.p, c, a.xyzq_s, a.typ_s, a.perm, a.inner, a.inner_nt, a.inner_m, a.dmask, a.masks,
                        a.counters, a.items, a.chunk, a.ljtab, a.facc, a.energy, a.ocap);
}

void launch_nonbonded(const NonbondedArgs& a, bool energy, cudaStream_t st) {
  const int nt1 = a.p.ntypes + 1;
  const size_t smem = (size_t)nt1 * nt1 * sizeof(float2);
  const PairConst c = pair_const(a.p);
  cudaMemsetAsync(a.counters + CNT_WORK, 0, sizeof(int), st);
  // 3 CTAs per SM fit 80 registers a thread; the 4-CTA build is held to 64
  auto k = energy ? (a.minb >= 4 ? k_nonbonded<true, 4> : k_nonbonded<true, 3>)
                  : (a.minb >= 4 ? k_nonbonded<false, 4> : k_nonbonded<false, 3>);
  launch_pdl(k, dim3(a.grid), dim3(kWarps * 32), smem, st, a.p, c, a.xyzq_s, a.typ_s, a.perm, a.inner, a.inner_nt, a.inner_m, a.dmask,
                                       a.masks, a.counters, a.items, a.chunk, a.ljtab, a.facc, a.energy, a.ocap);
}

// the work counters are zeroed by the prune's last kernel every step in batched steps
void launch_nonbonded_b(const NonbondedArgs* args, const BatchTables& t, int max_ntypes, cudaStream_t st) {
  const size_t smem = (size_t)(max_ntypes + 1) * (max_ntypes + 1) * sizeof(float2);
  launch_pdl(k_nonbonded_b, dim3(t.n[BT_NB]), dim3(kWarps * 32), smem, st, args, t.tab[BT_NB]);
}

}  // namespace fzk
