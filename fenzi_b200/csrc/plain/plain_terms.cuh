// Plain path: bonded terms, 1-4 pairs and the Ewald exclusion correction, one thread
// per term with atomic force adds (the terms of bondedforce,
// src/bonded_forces.cu:22-386, 703-1365, and src/mdcuda.cu:520-553).
#pragma once
#include "plain_kernels.cuh"

namespace fzp {

template <class T> struct Terms {
  int nbond, nub, nangle, ndihe, nimpr, n14, nexcl;
  const int2* bond;  const T* bond_k;  const T* bond_r0;
  const int2* ub;    const T* ub_k;    const T* ub_r0;
  const int4* angle; const T* angle_k; const T* angle_t0;
  const int4* dihe;  const T* dihe_k;  const int* dihe_n; const T* dihe_d;
  const int4* impr;  const T* impr_k;  const T* impr_p0;
  const int2* p14;   const T* eps4_14; const T* sig2_14;
  const int2* excl;
  const int* type;
};

template <class T> struct D3 {
  T x, y, z;
};
template <class T> __device__ __forceinline__ D3<T> sub_img(const Prm<T>& p, const typename Vec<T>::v4& a,
                                                            const typename Vec<T>::v4& b) {
  D3<T> d{a.x - b.x, a.y - b.y, a.z - b.z};
  min_image(p, d.x, d.y, d.z);
  return d;
}
template <class T> __device__ __forceinline__ T dot(const D3<T>& a, const D3<T>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T> __device__ __forceinline__ D3<T> cross(const D3<T>& a, const D3<T>& b) {
  return D3<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T, class V4> __device__ __forceinline__ void fadd(V4* f, int i, T s, const D3<T>& g) {
  atomicAdd(&f[i].x, s * g.x);
  atomicAdd(&f[i].y, s * g.y);
  atomicAdd(&f[i].z, s * g.z);
}

// dihedral angle (IUPAC sign) and its gradients (Blondel and Karplus, J. Comput.
// Chem. 17, 1132 (1996))
template <class T>
__device__ __forceinline__ T dihedral(const Prm<T>& p, const typename Vec<T>::v4* pos, int4 q, D3<T>& gi, D3<T>& gj,
                                      D3<T>& gk, D3<T>& gl) {
  const D3<T> F = sub_img(p, pos[q.x], pos[q.y]);
  const D3<T> G = sub_img(p, pos[q.y], pos[q.z]);
  const D3<T> H = sub_img(p, pos[q.w], pos[q.z]);
  const D3<T> A = cross(F, G), B = cross(H, G);
  const T A2 = dot(A, A), B2 = dot(B, B), Gn = m_sqrt(dot(G, G));
  const T phi = m_atan2(dot(cross(B, A), G) / Gn, dot(A, B));
  const T FG = dot(F, G), HG = dot(H, G);
  const T a1 = Gn / A2, b1 = Gn / B2, a2 = FG / (A2 * Gn), b2 = HG / (B2 * Gn);
  gi = D3<T>{-a1 * A.x, -a1 * A.y, -a1 * A.z};
  gl = D3<T>{b1 * B.x, b1 * B.y, b1 * B.z};
  gj = D3<T>{(a1 + a2) * A.x - b2 * B.x, (a1 + a2) * A.y - b2 * B.y, (a1 + a2) * A.z - b2 * B.z};
  gk = D3<T>{-(b1 * B.x) - a2 * A.x + b2 * B.x, -(b1 * B.y) - a2 * A.y + b2 * B.y, -(b1 * B.z) - a2 * A.z + b2 * B.z};
  return phi;
}

// one thread per term over [bonds | UB | angles | dihedrals | impropers | 1-4 | excl]
template <class T>
__global__ void k_terms(Prm<T> p, Terms<T> t, const typename Vec<T>::v4* __restrict__ pos,
                        typename Vec<T>::v4* force, double* e_acc) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double e[PE_N];
#pragma unroll
  for (int s = 0; s < PE_N; ++s) e[s] = 0.0;
  const T kPi = T(3.14159265358979323846);
  if (k < t.nbond) {
    const int2 b = t.bond[k];
    const D3<T> d = sub_img(p, pos[b.x], pos[b.y]);
    const T r = m_sqrt(dot(d, d)), dr = r - t.bond_r0[k];
    e[PE_BOND] = t.bond_k[k] * dr * dr;
    const T fr = -2 * t.bond_k[k] * dr / r;
    fadd(force, b.x, fr, d);
    fadd(force, b.y, -fr, d);
  } else if ((k -= t.nbond) < t.nub) {
    const int2 b = t.ub[k];
    const D3<T> d = sub_img(p, pos[b.x], pos[b.y]);
    const T r = m_sqrt(dot(d, d)), dr = r - t.ub_r0[k];
    e[PE_UREYB] = t.ub_k[k] * dr * dr;
    const T fr = -2 * t.ub_k[k] * dr / r;
    fadd(force, b.x, fr, d);
    fadd(force, b.y, -fr, d);
  } else if ((k -= t.nub) < t.nangle) {
    const int4 a = t.angle[k];
    const D3<T> u = sub_img(p, pos[a.x], pos[a.y]), v = sub_img(p, pos[a.z], pos[a.y]);
    const T uu = dot(u, u), vv = dot(v, v), ru = m_sqrt(uu), rv = m_sqrt(vv);
    T c = dot(u, v) / (ru * rv);
    c = c > T(1) ? T(1) : (c < T(-1) ? T(-1) : c);
    const D3<T> w = cross(u, v);
    const T sn = m_sqrt(dot(w, w)) / (ru * rv);
    const T dth = m_atan2(sn, c) - t.angle_t0[k];
    e[PE_ANGLE] = t.angle_k[k] * dth * dth;
    const T dE = 2 * t.angle_k[k] * dth;
    const T s = sn > T(1e-12) ? sn : T(1e-12);
    const T iuv = T(1) / (ru * rv);
    const D3<T> gu{-(v.x * iuv - c * u.x / uu) / s, -(v.y * iuv - c * u.y / uu) / s, -(v.z * iuv - c * u.z / uu) / s};
    const D3<T> gv{-(u.x * iuv - c * v.x / vv) / s, -(u.y * iuv - c * v.y / vv) / s, -(u.z * iuv - c * v.z / vv) / s};
    fadd(force, a.x, -dE, gu);
    fadd(force, a.z, -dE, gv);
    fadd(force, a.y, dE, D3<T>{gu.x + gv.x, gu.y + gv.y, gu.z + gv.z});
  } else if ((k -= t.nangle) < t.ndihe) {
    const int4 q = t.dihe[k];
    D3<T> gi, gj, gk, gl;
    const T phi = dihedral(p, pos, q, gi, gj, gk, gl);
    const T K = t.dihe_k[k], nn = (T)t.dihe_n[k], arg = nn * phi - t.dihe_d[k];
    e[PE_DIHED] = K * (1 + m_cos(arg));
    const T dE = -K * nn * m_sin(arg);
    fadd(force, q.x, -dE, gi);
    fadd(force, q.y, -dE, gj);
    fadd(force, q.z, -dE, gk);
    fadd(force, q.w, -dE, gl);
  } else if ((k -= t.ndihe) < t.nimpr) {
    const int4 q = t.impr[k];
    D3<T> gi, gj, gk, gl;
    T dp = dihedral(p, pos, q, gi, gj, gk, gl) - t.impr_p0[k];
    dp -= 2 * kPi * m_rint(dp / (2 * kPi));
    e[PE_IMPR] = t.impr_k[k] * dp * dp;
    const T dE = 2 * t.impr_k[k] * dp;
    fadd(force, q.x, -dE, gi);
    fadd(force, q.y, -dE, gj);
    fadd(force, q.z, -dE, gk);
    fadd(force, q.w, -dE, gl);
  } else if ((k -= t.nimpr) < t.n14) {
    const int2 b = t.p14[k];
    const D3<T> d = sub_img(p, pos[b.x], pos[b.y]);
    const int ty = t.type[b.x] * p.nt + t.type[b.y];
    T ev, ee;
    const T fr = pair_force(p, dot(d, d), pos[b.x].w * pos[b.y].w, t.eps4_14[ty], t.sig2_14[ty], ev, ee);
    e[PE_VDW] = ev;
    e[PE_ELEC] = ee;
    fadd(force, b.x, fr, d);
    fadd(force, b.y, -fr, d);
  } else if ((k -= t.n14) < t.nexcl) {
    const int2 b = t.excl[k];
    const D3<T> d = sub_img(p, pos[b.x], pos[b.y]);
    const T r2 = dot(d, d), r = m_sqrt(r2), qq = pos[b.x].w * pos[b.y].w;
    const T erfv = m_erf(p.beta * r);
    e[PE_EWEXCL] = -p.cc * qq * erfv / r;
    const T fr = p.cc * qq * (T(1.1283791670955126) * p.beta * r * m_exp(-p.beta * p.beta * r2) - erfv) / (r2 * r);
    fadd(force, b.x, fr, d);
    fadd(force, b.y, -fr, d);
  }
  // warp sums of the energies that occur in this warp, one atomic add each
#pragma unroll
  for (int s = 0; s < PE_N; ++s) {
    if (!__any_sync(0xffffffffu, e[s] != 0.0)) continue;
    double v = e[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&e_acc[s], v);
  }
}

}  // namespace fzp
