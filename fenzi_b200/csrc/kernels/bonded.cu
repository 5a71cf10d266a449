// Bonded terms, Ewald exclusion correction and 1-4 pairs: the work of bondedforce
// (src/bonded_forces.cu:597-1381) with bondInteraction/angleInteraction/
// improperInteraction/torsionInteraction (:22-386), Urey-Bradley (:935-991), the
// explicit Ewald exclusion list (:783-826, src/mdcuda.cu:520-553) and the NBXMOD 5
// 1-4 pairs (:1155-1268).
//
// The reference evaluates each term once per member atom and keeps only that atom's
// force; here one thread evaluates each term once and scatters every member's force
// as int64 fixed point (RED atomics, order independent).  The exclusion correction is
// evaluated in FP64 (it cancels against the self term and the reciprocal sum).
// Dihedrals use the exact CHARMM form K(1 + cos(n phi - delta)) for any delta (the
// reference's sin(n phi - delta) update at :364-365 is right only for delta in {0, 180}).
#include "common.cuh"
#include "kernels.h"

namespace fzk {

// minimum-image difference a - b of two FP32 positions, formed in FP64 and rounded once:
// two atoms of a term split by the periodic boundary are about L apart before the image
// shift, and an FP32 difference would round at the ulp of L (up to 3.8e-6 A for
// L = 130 A), a 1e-4 relative error in the force of a stiff bond
__device__ __forceinline__ float3 image_diff(float4 a, float4 b, const SysParams& p) {
  double d[3] = {(double)a.x - (double)b.x, (double)a.y - (double)b.y, (double)a.z - (double)b.z};
  min_image_d(d, p);
  return make_float3((float)d[0], (float)d[1], (float)d[2]);
}
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ void addf(long long* facc, int n, int i, float3 f) {
  red_add(facc + i, to_fix(f.x));
  red_add(facc + n + i, to_fix(f.y));
  red_add(facc + 2 * n + i, to_fix(f.z));
}

// dihedral angle terms for atoms i,j,k,l: cos/sin phi and d(phi)/d(r) (Blondel & Karplus,
// J. Comput. Chem. 17, 1132 (1996)); returns false for a degenerate (collinear) geometry
__device__ __forceinline__ bool dihedral_geom(float4 ri, float4 rj, float4 rk, float4 rl, const SysParams& p,
                                              float* cphi, float* sphi, float3* gi, float3* gj, float3* gk,
                                              float3* gl, float3* rel) {
  const float3 F = image_diff(ri, rj, p);
  const float3 G = image_diff(rj, rk, p);
  const float3 H = image_diff(rl, rk, p);
  // positions relative to atom j: i - j = F, k - j = -G, l - j = H - G
  rel[0] = F;
  rel[1] = make_float3(-G.x, -G.y, -G.z);
  rel[2] = make_float3(H.x - G.x, H.y - G.y, H.z - G.z);
  const float3 A = cross(F, G), B = cross(H, G);
  const float A2 = dot(A, A), B2 = dot(B, B), G2 = dot(G, G);
  if (A2 < 1e-12f || B2 < 1e-12f || G2 < 1e-12f) return false;
  const float Gn = sqrtf(G2);
  const float rab = rsqrtf(A2 * B2);
  *cphi = dot(A, B) * rab;
  *sphi = dot(cross(B, A), G) * rab / Gn;
  const float FG = dot(F, G), HG = dot(H, G);
  const float ia = Gn / A2, ib = Gn / B2, fa = FG / (A2 * Gn), hb = HG / (B2 * Gn);
  *gi = make_float3(-ia * A.x, -ia * A.y, -ia * A.z);
  *gl = make_float3(ib * B.x, ib * B.y, ib * B.z);
  *gj = make_float3((ia + fa) * A.x - hb * B.x, (ia + fa) * A.y - hb * B.y, (ia + fa) * A.z - hb * B.z);
  *gk = make_float3(-ib * B.x - fa * A.x + hb * B.x, -ib * B.y - fa * A.y + hb * B.y, -ib * B.z - fa * A.z + hb * B.z);
  return true;
}

template <bool ENERGY>
__device__ __forceinline__ void bonded_body(const BondedArgs& a, int bid) {
  griddep_wait();
  const int t = bid * blockDim.x + threadIdx.x;
  const int n = a.p.n;
  const SysParams& p = a.p;
  double e[7] = {0, 0, 0, 0, 0, 0, 0};  // bond angle ub dihed impr ewexcl (vdw14, elec14 below)
  double e14v = 0, e14e = 0;
  double w[3] = {0, 0, 0};  // virial diagonal sum over atoms of r_a F_a (relative vectors)
  int r = t;
  if (r < a.nbond) {
    const int2 b = a.bond[r];
    const float2 pr = a.bond_prm[r];
    const float3 d = image_diff(a.pos4[b.x], a.pos4[b.y], p);
    const float rr = sqrtf(dot(d, d));
    const float dr = rr - pr.y;
    const float f = rr > 0.f ? -2.f * pr.x * dr / rr : 0.f;
    addf(a.facc, n, b.x, make_float3(f * d.x, f * d.y, f * d.z));
    addf(a.facc, n, b.y, make_float3(-f * d.x, -f * d.y, -f * d.z));
    if (ENERGY) {
      e[0] = (double)pr.x * dr * dr;
      w[0] = f * d.x * d.x;
      w[1] = f * d.y * d.y;
      w[2] = f * d.z * d.z;
    }
  } else if ((r -= a.nbond) < a.nangle) {
    const int4 q = a.angle[r];
    const float2 pr = a.angle_prm[r];
    const float4 rj = a.pos4[q.y];
    const float3 u = image_diff(a.pos4[q.x], rj, p);
    const float3 v = image_diff(a.pos4[q.z], rj, p);
    const float uu = dot(u, u), vv = dot(v, v), uv = dot(u, v);
    const float3 uxv = cross(u, v);
    const float ruv = rsqrtf(uu * vv);
    const float c = uv * ruv;
    const float s = sqrtf(dot(uxv, uxv)) * ruv;
    const float th = atan2f(s, c);
    const float dth = th - pr.y;
    const float dE = 2.f * pr.x * dth;
    const float sf = fmaxf(s, 1e-6f);
    const float k1 = -dE / sf;
    // dtheta/du = -(v/(|u||v|) - c u/|u|^2)/sin ; force = -dE * dtheta/du
    const float3 gu = make_float3(v.x * ruv - c * u.x / uu, v.y * ruv - c * u.y / uu, v.z * ruv - c * u.z / uu);
    const float3 gv = make_float3(u.x * ruv - c * v.x / vv, u.y * ruv - c * v.y / vv, u.z * ruv - c * v.z / vv);
    const float3 fi = make_float3(-k1 * gu.x, -k1 * gu.y, -k1 * gu.z);
    const float3 fk = make_float3(-k1 * gv.x, -k1 * gv.y, -k1 * gv.z);
    addf(a.facc, n, q.x, fi);
    addf(a.facc, n, q.z, fk);
    addf(a.facc, n, q.y, make_float3(-fi.x - fk.x, -fi.y - fk.y, -fi.z - fk.z));
    if (ENERGY) {
      e[1] = (double)pr.x * dth * dth;
      w[0] = fi.x * u.x + fk.x * v.x;
      w[1] = fi.y * u.y + fk.y * v.y;
      w[2] = fi.z * u.z + fk.z * v.z;
    }
  } else if ((r -= a.nangle) < a.nub) {
    const int2 b = a.ub[r];
    const float2 pr = a.ub_prm[r];
    const float3 d = image_diff(a.pos4[b.x], a.pos4[b.y], p);
    const float rr = sqrtf(dot(d, d));
    const float dr = rr - pr.y;
    const float f = rr > 0.f ? -2.f * pr.x * dr / rr : 0.f;
    addf(a.facc, n, b.x, make_float3(f * d.x, f * d.y, f * d.z));
    addf(a.facc, n, b.y, make_float3(-f * d.x, -f * d.y, -f * d.z));
    if (ENERGY) {
      e[2] = (double)pr.x * dr * dr;
      w[0] = f * d.x * d.x;
      w[1] = f * d.y * d.y;
      w[2] = f * d.z * d.z;
    }
  } else if ((r -= a.nub) < a.ndihe) {
    const int4 q = a.dihe[r];
    const float4 pr = a.dihe_prm[r];  // K, n, cos d, sin d
    float c, s;
    float3 gi, gj, gk, gl, rel[3];
    if (dihedral_geom(a.pos4[q.x], a.pos4[q.y], a.pos4[q.z], a.pos4[q.w], p, &c, &s, &gi, &gj, &gk, &gl, rel)) {
      const int nn = (int)pr.y;
      float cn = 1.f, sn = 0.f;
      for (int m = 0; m < nn; ++m) {
        const float c2 = cn * c - sn * s;
        sn = sn * c + cn * s;
        cn = c2;
      }
      const float cosd = fmaf(cn, pr.z, sn * pr.w);   // cos(n phi - delta)
      const float sind = fmaf(sn, pr.z, -cn * pr.w);  // sin(n phi - delta)
      const float dE = -pr.x * (float)nn * sind;      // dE/dphi
      addf(a.facc, n, q.x, make_float3(-dE * gi.x, -dE * gi.y, -dE * gi.z));
      addf(a.facc, n, q.y, make_float3(-dE * gj.x, -dE * gj.y, -dE * gj.z));
      addf(a.facc, n, q.z, make_float3(-dE * gk.x, -dE * gk.y, -dE * gk.z));
      addf(a.facc, n, q.w, make_float3(-dE * gl.x, -dE * gl.y, -dE * gl.z));
      if (ENERGY) {
        e[3] = (double)pr.x * (1.0 + (double)cosd);
        w[0] = -dE * (gi.x * rel[0].x + gk.x * rel[1].x + gl.x * rel[2].x);
        w[1] = -dE * (gi.y * rel[0].y + gk.y * rel[1].y + gl.y * rel[2].y);
        w[2] = -dE * (gi.z * rel[0].z + gk.z * rel[1].z + gl.z * rel[2].z);
      }
    }
  } else if ((r -= a.ndihe) < a.nimpr) {
    const int4 q = a.impr[r];
    const float2 pr = a.impr_prm[r];
    float c, s;
    float3 gi, gj, gk, gl, rel[3];
    if (dihedral_geom(a.pos4[q.x], a.pos4[q.y], a.pos4[q.z], a.pos4[q.w], p, &c, &s, &gi, &gj, &gk, &gl, rel)) {
      float dp = atan2f(s, c) - pr.y;
      dp -= 6.283185307179586f * rintf(dp * 0.15915494309189535f);
      const float dE = 2.f * pr.x * dp;
      addf(a.facc, n, q.x, make_float3(-dE * gi.x, -dE * gi.y, -dE * gi.z));
      addf(a.facc, n, q.y, make_float3(-dE * gj.x, -dE * gj.y, -dE * gj.z));
      addf(a.facc, n, q.z, make_float3(-dE * gk.x, -dE * gk.y, -dE * gk.z));
      addf(a.facc, n, q.w, make_float3(-dE * gl.x, -dE * gl.y, -dE * gl.z));
      if (ENERGY) {
        e[4] = (double)pr.x * dp * dp;
        w[0] = -dE * (gi.x * rel[0].x + gk.x * rel[1].x + gl.x * rel[2].x);
        w[1] = -dE * (gi.y * rel[0].y + gk.y * rel[1].y + gl.y * rel[2].y);
        w[2] = -dE * (gi.z * rel[0].z + gk.z * rel[1].z + gl.z * rel[2].z);
      }
    }
  } else if ((r -= a.nimpr) < a.nexcl) {
    // Ewald exclusion correction, FP64: E = -CC qq erf(beta r)/r
    const int2 b = a.excl[r];
    const float4 ri = a.pos4[b.x], rj = a.pos4[b.y];
    double d[3] = {(double)ri.x - rj.x, (double)ri.y - rj.y, (double)ri.z - rj.z};
    min_image_d(d, p);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double rr = sqrt(r2);
    const double beta = (double)p.beta;
    const double qq = (double)ri.w * (double)rj.w;
    const double erfv = erf(beta * rr);
    const double f = kCC * qq * (1.1283791670955126 * beta * rr * exp(-beta * beta * r2) - erfv) / (r2 * rr);
    const long long fx = to_fix_d(f * d[0]), fy = to_fix_d(f * d[1]), fz = to_fix_d(f * d[2]);
    red_add(a.facc + b.x, fx);
    red_add(a.facc + n + b.x, fy);
    red_add(a.facc + 2 * n + b.x, fz);
    red_add(a.facc + b.y, -fx);
    red_add(a.facc + n + b.y, -fy);
    red_add(a.facc + 2 * n + b.y, -fz);
    if (ENERGY) {
      e[5] = -kCC * qq * erfv / rr;
      w[0] = f * d[0] * d[0];
      w[1] = f * d[1] * d[1];
      w[2] = f * d[2] * d[2];
    }
  } else if ((r -= a.nexcl) < a.n14) {
    // 1-4: 1-4 LJ (switched) + erfc Coulomb, no cutoff test (src/bonded_forces.cu:1155-1268)
    const int2 b = a.p14[r];
    const float4 ri = a.pos4[b.x], rj = a.pos4[b.y];
    const float3 d = image_diff(ri, rj, p);
    const float r2 = dot(d, d);
    const float rr = sqrtf(r2), r2inv = 1.f / r2;
    const float2 ls = a.lj14[a.type[b.x] * (p.ntypes + 1) + a.type[b.y]];
    const float s2 = ls.y * r2inv, s6 = s2 * s2 * s2;
    const float aa = ls.x * s6, bb = aa * s6;
    const float elj = bb - aa;
    const float flj = (12.f * bb - 6.f * aa) * r2inv;
    float sw = 1.f, dsw = 0.f;
    if (r2 > p.ron2) {
      const float u = p.rc2 - r2;
      sw = u * u * (p.rc2 + 2.f * r2 - 3.f * p.ron2) * p.sw_c3;
      dsw = 12.f * u * (r2 - p.ron2) * p.sw_c3;
    }
    const float qq = p.cc * ri.w * rj.w;
    const float br = p.beta * rr;
    const float ec = qq * erfcf(br) / rr;
    const float fc = (ec + qq * 1.1283791670955126f * p.beta * __expf(-br * br)) * r2inv;
    const float fr = flj * sw + elj * dsw + fc;
    addf(a.facc, n, b.x, make_float3(fr * d.x, fr * d.y, fr * d.z));
    addf(a.facc, n, b.y, make_float3(-fr * d.x, -fr * d.y, -fr * d.z));
    if (ENERGY) {
      e14v = (double)(elj * sw);
      e14e = (double)ec;
      w[0] = fr * d.x * d.x;
      w[1] = fr * d.y * d.y;
      w[2] = fr * d.z * d.z;
    }
  }
  if (ENERGY) {
    energy_add(a.energy + EN_BOND, e[0]);
    energy_add(a.energy + EN_ANGLE, e[1]);
    energy_add(a.energy + EN_UREYB, e[2]);
    energy_add(a.energy + EN_DIHED, e[3]);
    energy_add(a.energy + EN_IMPR, e[4]);
    energy_add(a.energy + EN_EWEXCL, e[5]);
    energy_add(a.energy + EN_VDW, e14v);
    energy_add(a.energy + EN_ELEC, e14e);
    energy_add(a.energy + EN_VIR_X, w[0]);
    energy_add(a.energy + EN_VIR_Y, w[1]);
    energy_add(a.energy + EN_VIR_Z, w[2]);
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(256) k_bonded(BondedArgs a) { griddep_wait(); bonded_body<ENERGY>(a, blockIdx.x); }

__global__ void __launch_bounds__(256) k_bonded_b(const BondedArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const BondedArgs a = args[t.x];
  bonded_body<false>(a, t.y);
}

void launch_bonded(const BondedArgs& a, bool energy, cudaStream_t st) {
  const int tot = a.nbond + a.nangle + a.nub + a.ndihe + a.nimpr + a.nexcl + a.n14;
  if (tot == 0) return;
  const int g = (tot + 255) / 256;
  if (energy)
    launch_pdl(k_bonded<true>, dim3(g), dim3(256), 0, st, a);
  else
    launch_pdl(k_bonded<false>, dim3(g), dim3(256), 0, st, a);
}

int bonded_blocks(const BondedArgs& a) {
  return (a.nbond + a.nangle + a.nub + a.ndihe + a.nimpr + a.nexcl + a.n14 + 255) / 256;
}

void launch_bonded_b(const BondedArgs* args, const BatchTables& t, cudaStream_t st) {
  if (t.n[BT_BONDED] > 0) launch_pdl(k_bonded_b, dim3(t.n[BT_BONDED]), dim3(256), 0, st, args, t.tab[BT_BONDED]);
}

// ---------------------------------------------------------------- consharm restraint
constexpr double kFixCom = 16777216.0;  // mass-centre sums, 2^24 per amu A

// positions wrapped into [-L/2, L/2) (the reference's primary box), mass-weighted sums
// per segment in fixed point (order independent)
__global__ void __launch_bounds__(256) k_restraint_com(SysParams p, const float4* __restrict__ pos4,
                                                       const int* __restrict__ seg, const float* __restrict__ mass,
                                                       long long* acc) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (i < p.n) {
    const int sg = seg[i];
    if (sg >= 0) {
      const float4 r = pos4[i];
      const double m = mass[i];
      const double x = r.x - p.box.x * floorf(r.x * p.inv_box.x + 0.5f);
      const double y = r.y - p.box.y * floorf(r.y * p.inv_box.y + 0.5f);
      const double z = r.z - p.box.z * floorf(r.z * p.inv_box.z + 0.5f);
      w[3 * sg] = m * x;
      w[3 * sg + 1] = m * y;
      w[3 * sg + 2] = m * z;
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    long long v = __double2ll_rn(w[k] * kFixCom);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0) red_add(acc + k, v);
  }
}

__global__ void __launch_bounds__(256) k_restraint_force(int n, const int* __restrict__ seg,
                                                         const long long* __restrict__ acc, double inv_m0,
                                                         double inv_m1, double dx, double dy, double dz, double fc,
                                                         long long* facc) { griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || seg[i] != 1) return;
  const double s = 1.0 / kFixCom;
  const double fx = fc * (dx + acc[0] * s * inv_m0 - acc[3] * s * inv_m1);
  const double fy = fc * (dy + acc[1] * s * inv_m0 - acc[4] * s * inv_m1);
  const double fz = fc * (dz + acc[2] * s * inv_m0 - acc[5] * s * inv_m1);
  red_add(facc + i, to_fix_d(fx));
  red_add(facc + n + i, to_fix_d(fy));
  red_add(facc + 2 * n + i, to_fix_d(fz));
}

void launch_restraint(const SysParams& p, const float4* pos4, const int* seg, const float* mass, long long* acc,
                      double inv_m0, double inv_m1, const double* dist, double fc, long long* facc, cudaStream_t st) {
  const int g = (p.n + 255) / 256;
  launch_pdl(k_restraint_com, dim3(g), dim3(256), 0, st, p, pos4, seg, mass, acc);
  launch_pdl(k_restraint_force, dim3(g), dim3(256), 0, st, p.n, seg, acc, inv_m0, inv_m1, dist[0], dist[1], dist[2], fc, facc);
}

}  // namespace fzk
