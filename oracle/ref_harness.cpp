/*
 * Runs the reference's own force kernels on the host (the checker of the oracle;
 * test infrastructure only, never part of the product).
 *
 * The kernels (src/bonded_forces.cu bondedforce / bondedforce_c36, src/nonbonded_forces.cu
 * nonbondforce) and their helpers are compiled from the reference sources by
 * oracle/refbuild.py; this file lays the reference's device data out exactly as its
 * readers and InitMem do, runs one host loop iteration per GPU thread, and sums the
 * per-thread outputs the way the reference's reductions do.  Data layouts restated
 * from the reference:
 *   - per-atom transposed lists, W = atoms ("WorkgroupSize"), row 0 = count:
 *       bonds_index / ureyb_index rows 2i+1 = parameter index, 2i+2 = partner
 *       (src/prmread.cu:1775-1782); angles/dihedrals/impropers_index row i+1 = term
 *       index into *_set[Count * k + (term + 1)], k = 0 parameter index, k >= 1 atoms
 *       (src/prmread.cu:1800-1950);
 *   - parameters: bondprm = (2 K, r0) (src/prmread.cu:2328), angleprm = (K, theta0 rad)
 *     (:2358-2359), ureybprm = (K, S0) (:2376-2377), improper_prm = (K, psi0),
 *     dihedral_prm[j * MAX_DIHED_TYPE + h] = (K, n, delta rad) with
 *     dihedral_type_count[h] folds (src/prmread.cu:2390-2455), prm1_4 per type =
 *     (eps14, rmin14/2 / 2^(1/6)) (:2483-2499), nbfixprm per type pair = (4 eps_ij,
 *     sigma_ij^2) (:2549-2551, 2724-2736);
 *   - the nonbonded list nblist[k * W + i], row 0 = count, entries type << 20 | atom
 *     (src/cucomplexops.h:64-69), every pair in both atoms' lists;
 *   - switch coefficients Swcoeff1 = rc^2, Swcoeff2 = rc^2 - 3 ron^2,
 *     Swcoeff3 = 1 / (rc^2 - ron^2)^3 (src/mem.cu:556-559); boxH = half box edges.
 * Launch: BPART (bonded) and NBPART (nonbonded) threads per atom, gtid in [0, P W)
 * (src/mdcuda.cu:563-640, src/dynamics.cu), per-thread outputs summed over the P
 * threads of an atom; energies summed over atoms in double.
 */
#include "ref_shim.h"

fzref_dim3 threadIdx{0, 0, 0}, blockIdx{0, 0, 0}, blockDim{1, 1, 1}, gridDim{1, 1, 1};
fzref_real beta, betaSqr, cutoffd, Cutond, Swcoeff1d, Swcoeff2d, Swcoeff3d;
int WorkgroupSized, num_types_presentd, Angle_Countd, Dihed_Countd, Improper_Countd;
float4 boxH;
const float4* texcrd;
const int* textype;
const float2* texprm1_4;
const float2* texnbfixprm;

#if FZREF_VARIANT == 64
#include "ref_defs64.inc"
#define float double
#else
#include "ref_defs32.inc"
#endif
/* PME globals of the reference (src/globals.h:50-57, 104-106, 122-123, 136-167, 627):
 * host values of InitDeviceConstants, constant symbols of BCMultiply */
float KAPPa;
float4 Region;
int fftx, ffty, fftz;
float* M4d;
float* dM4d;
float sqr_b1d[MAXFFT_X], sqr_b2d[MAXFFT_Y], sqr_b3d[MAXFFT_Z];
float c1d[MAXFFT_X], c2d[MAXFFT_Y], c3d[MAXFFT_Z];
int FFTX, FFTY, FFTZ, TOTAL_PME_LATTICES;
float FFTXH, FFTYH, FFTZH;
float4 box;
#if FZREF_VARIANT == 64
#include "ref_pieces64.inc"
#undef float
#else
#include "ref_pieces32.inc"
#endif

namespace {

typedef fzref_real R;

struct Sys {
  int n;
  const double* pos;
  const double* q;
  const int* type;
  int ntypes;
  const double* nbfix_eps4;
  const double* nbfix_sig2;
  const double* p14_eps;
  const double* p14_sig;
  int nbond;
  const int* bond;
  const double* bond_k;
  const double* bond_r0;
  int nangle;
  const int* angle;
  const double* angle_k;
  const double* angle_t0;
  const int* angle_ub;  // per angle: index into the UB arrays or -1
  int nub;
  const double* ub_k;
  const double* ub_s0;
  int ndihe;
  const int* dihe;
  const int* dihe_nfold;
  const double* fold_k;
  const int* fold_n;
  const double* fold_d;
  int nimpr;
  const int* impr;
  const double* impr_k;
  const double* impr_p0;
  double box[3];
  double rc, ron, beta;
  const int* nb_off;  // CSR neighbour list (both directions), n + 1 offsets
  const int* nb_idx;
};

void set_common(const Sys& s, std::vector<float4>& crd, std::vector<float2>& p14, std::vector<float2>& nbf) {
  const int n = s.n;
  crd.resize(n);
  for (int i = 0; i < n; ++i)
    crd[i] = float4{(R)s.pos[3 * i], (R)s.pos[3 * i + 1], (R)s.pos[3 * i + 2], (R)s.q[i]};
  p14.resize(s.ntypes);
  for (int t = 0; t < s.ntypes; ++t) p14[t] = float2{(R)s.p14_eps[t], (R)s.p14_sig[t]};
  nbf.resize((size_t)s.ntypes * s.ntypes);
  for (int k = 0; k < s.ntypes * s.ntypes; ++k) nbf[k] = float2{(R)s.nbfix_eps4[k], (R)s.nbfix_sig2[k]};
  texcrd = crd.data();
  textype = s.type;
  texprm1_4 = p14.data();
  texnbfixprm = nbf.data();
  WorkgroupSized = n;
  num_types_presentd = s.ntypes;
  beta = (R)s.beta;
  betaSqr = beta * beta;
  cutoffd = (R)s.rc;
  Cutond = (R)s.ron;
  const R rc = (R)s.rc, ron = (R)s.ron;
  Swcoeff1d = rc * rc;
  Swcoeff2d = rc * rc - 3 * ron * ron;
  R c3 = (R)1 / (rc * rc - ron * ron);
  Swcoeff3d = c3 * c3 * c3;
  boxH = float4{(R)(0.5 * s.box[0]), (R)(0.5 * s.box[1]), (R)(0.5 * s.box[2]), (R)0};
}

// per-atom transposed list: rows[r * n + atom], row 0 = count
struct PerAtom {
  int n, rows;
  std::vector<int> a;
  PerAtom(int n_, const std::vector<std::vector<int>>& lists, int per) : n(n_) {
    size_t mx = 0;
    for (const auto& l : lists) mx = std::max(mx, l.size() / per);
    rows = 1 + (int)mx * per;
    a.assign((size_t)rows * n, 0);
    for (int i = 0; i < n; ++i) {
      a[i] = (int)(lists[i].size() / per);
      for (size_t k = 0; k < lists[i].size(); ++k) a[(k + 1) * n + i] = lists[i][k];
    }
  }
};

}  // namespace

extern "C" {

/* Bonded terms of the reference (bondedforce, or bondedforce_c36 when c36 != 0) on
 * the host.  f[3n] receives the per-atom force (overwritten); e[8] the energies
 * bond, angle, Urey-Bradley, dihedral, improper, Ewald exclusion, 1-4 vdW, 1-4 elec. */
int fzr_bonded(const Sys* sp, int c36, double* f, double* e) {
  const Sys& s = *sp;
  const int n = s.n;
  std::vector<float4> crd;
  std::vector<float2> p14, nbf;
  set_common(s, crd, p14, nbf);
  // bonds: one parameter set per bond (h = bond index)
  std::vector<float2> bondprm(std::max(1, s.nbond));
  std::vector<std::vector<int>> bl(n);
  for (int b = 0; b < s.nbond; ++b) {
    const int x = s.bond[2 * b], y = s.bond[2 * b + 1];
    bondprm[b] = float2{(R)(2.0 * s.bond_k[b]), (R)s.bond_r0[b]};
    bl[x].push_back(b);
    bl[x].push_back(y);
    bl[y].push_back(b);
    bl[y].push_back(x);
  }
  PerAtom bonds(n, bl, 2);
  // angles (+ Urey-Bradley on the 1-3 atoms of an angle)
  std::vector<float2> angleprm(std::max(1, s.nangle)), ureybprm(std::max(1, s.nub));
  std::vector<int> angles_set(4 * (size_t)std::max(1, s.nangle) + 1, 0);
  std::vector<std::vector<int>> al(n), ul(n);
  for (int a = 0; a < s.nangle; ++a) {
    angleprm[a] = float2{(R)s.angle_k[a], (R)s.angle_t0[a]};
    angles_set[(size_t)s.nangle * 0 + a + 1] = a;
    for (int k = 0; k < 3; ++k) {
      const int at = s.angle[3 * a + k];
      angles_set[(size_t)s.nangle * (k + 1) + a + 1] = at;
      al[at].push_back(a);
    }
    const int u = s.angle_ub ? s.angle_ub[a] : -1;
    if (u >= 0) {
      ureybprm[u] = float2{(R)s.ub_k[u], (R)s.ub_s0[u]};
      const int x = s.angle[3 * a], z = s.angle[3 * a + 2];
      ul[x].push_back(u);
      ul[x].push_back(z);
      ul[z].push_back(u);
      ul[z].push_back(x);
    }
  }
  PerAtom angles(n, al, 1), ureyb(n, ul, 2);
  // dihedrals: parameter sets deduplicated into h < MAX_DIHED_TYPE
  std::vector<dihedralParameter> dprm(MAX_DIHED_TYPE * MAXDPRM);
  std::vector<unsigned char> dcount(MAX_DIHED_TYPE, 0);
  std::vector<std::vector<double>> sets;
  std::vector<int> dihedrals_set(5 * (size_t)std::max(1, s.ndihe) + 1, 0);
  std::vector<std::vector<int>> dl(n);
  for (int d = 0, fo = 0; d < s.ndihe; ++d) {
    const int nf = s.dihe_nfold[d];
    if (nf < 1 || nf > MAXDPRM) return -1;
    std::vector<double> key;
    for (int j = 0; j < nf; ++j) {
      key.push_back(s.fold_k[fo + j]);
      key.push_back((double)s.fold_n[fo + j]);
      key.push_back(s.fold_d[fo + j]);
    }
    int h = -1;
    for (size_t k = 0; k < sets.size(); ++k)
      if (sets[k] == key) h = (int)k;
    if (h < 0) {
      h = (int)sets.size();
      if (h >= MAX_DIHED_TYPE) return -2;
      sets.push_back(key);
      dcount[h] = (unsigned char)nf;
      for (int j = 0; j < nf; ++j) {
        dihedralParameter& P = dprm[j * MAX_DIHED_TYPE + h];
        P.x = (R)s.fold_k[fo + j];
        P.n = (short)s.fold_n[fo + j];
        P.d = (R)s.fold_d[fo + j];
      }
    }
    fo += nf;
    dihedrals_set[(size_t)s.ndihe * 0 + d + 1] = h;
    for (int k = 0; k < 4; ++k) {
      const int at = s.dihe[4 * d + k];
      dihedrals_set[(size_t)s.ndihe * (k + 1) + d + 1] = at;
      dl[at].push_back(d);
    }
  }
  PerAtom dihedrals(n, dl, 1);
  std::vector<float2> iprm(std::max(1, s.nimpr));
  std::vector<int> impropers_set(5 * (size_t)std::max(1, s.nimpr) + 1, 0);
  std::vector<std::vector<int>> il(n);
  for (int d = 0; d < s.nimpr; ++d) {
    iprm[d] = float2{(R)s.impr_k[d], (R)s.impr_p0[d]};
    impropers_set[(size_t)s.nimpr * 0 + d + 1] = d;
    for (int k = 0; k < 4; ++k) {
      const int at = s.impr[4 * d + k];
      impropers_set[(size_t)s.nimpr * (k + 1) + d + 1] = at;
      il[at].push_back(d);
    }
  }
  PerAtom impropers(n, il, 1);
  Angle_Countd = s.nangle;
  Dihed_Countd = s.ndihe;
  Improper_Countd = s.nimpr;

  const int P = BPART, T = P * n;
  std::vector<float4> fb(T);
  std::vector<fzref_real> ebnd(T), eang(T), eub(T), edih(T), evdw(T), eel(T), eimp(T), eex(T);
  std::vector<int> ewlist(1, 0);
  gridDim = fzref_dim3{1, 1, 1};
  blockIdx = fzref_dim3{0, 0, 0};
  blockDim = fzref_dim3{(unsigned)T, 1, 1};
  for (int g = 0; g < T; ++g) {
    threadIdx = fzref_dim3{(unsigned)g, 0, 0};
    if (c36)
      bondedforce_c36(fb.data(), bonds.a.data(), bondprm.data(), ebnd.data(), angles.a.data(), angles_set.data(),
                      angleprm.data(), eang.data(), ureyb.a.data(), ureybprm.data(), eub.data(), dihedrals.a.data(),
                      dihedrals_set.data(), dprm.data(), dcount.data(), edih.data(), evdw.data(), eel.data(),
                      impropers.a.data(), impropers_set.data(), iprm.data(), eimp.data(), ewlist.data(), eex.data());
    else
      bondedforce(fb.data(), bonds.a.data(), bondprm.data(), ebnd.data(), angles.a.data(), angles_set.data(),
                  angleprm.data(), eang.data(), ureyb.a.data(), ureybprm.data(), eub.data(), dihedrals.a.data(),
                  dihedrals_set.data(), dprm.data(), dcount.data(), edih.data(), evdw.data(), eel.data(),
                  impropers.a.data(), impropers_set.data(), iprm.data(), eimp.data(), ewlist.data(), eex.data());
  }
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    for (int p = 0; p < P; ++p) {
      fx += (double)fb[p * n + i].x;
      fy += (double)fb[p * n + i].y;
      fz += (double)fb[p * n + i].z;
    }
    f[3 * i] = fx;
    f[3 * i + 1] = fy;
    f[3 * i + 2] = fz;
  }
  const std::vector<fzref_real>* ev[8] = {&ebnd, &eang, &eub, &edih, &eimp, &eex, &evdw, &eel};
  for (int k = 0; k < 8; ++k) {
    double t = 0;
    for (int g = 0; g < T; ++g) t += (double)(*ev[k])[g];
    e[k] = t;
  }
  return 0;
}

/* The reference's nonbonded kernel (nonbondforce) on the host over the given full
 * neighbour list.  f[3n] receives the per-atom force; e[2] = vdW, elec energies. */
int fzr_nonbond(const Sys* sp, double* f, double* e) {
  const Sys& s = *sp;
  const int n = s.n;
  if (n >= (1 << 20) || s.ntypes >= (1 << 11)) return -1;
  std::vector<float4> crd;
  std::vector<float2> p14, nbf;
  set_common(s, crd, p14, nbf);
  int mx = 0;
  for (int i = 0; i < n; ++i) mx = std::max(mx, s.nb_off[i + 1] - s.nb_off[i]);
  std::vector<unsigned int> nbl((size_t)(mx + 1) * n, 0u);
  for (int i = 0; i < n; ++i) {
    const int c = s.nb_off[i + 1] - s.nb_off[i];
    nbl[i] = (unsigned)c;
    for (int k = 0; k < c; ++k) {
      const int j = s.nb_idx[s.nb_off[i] + k];
      nbl[(size_t)(k + 1) * n + i] = ((unsigned)s.type[j] << 20) | (unsigned)j;
    }
  }
  const int P = NBPART, T = P * n;
  std::vector<float4> fn(T);
  std::vector<fzref_real> evdw(T, 0), eel(T, 0);
  gridDim = fzref_dim3{1, 1, 1};
  blockIdx = fzref_dim3{0, 0, 0};
  blockDim = fzref_dim3{(unsigned)T, 1, 1};
  for (int g = 0; g < T; ++g) {
    threadIdx = fzref_dim3{(unsigned)g, 0, 0};
    nonbondforce(fn.data(), nbl.data(), evdw.data(), eel.data());
  }
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0;
    for (int p = 0; p < P; ++p) {
      fx += (double)fn[p * n + i].x;
      fy += (double)fn[p * n + i].y;
      fz += (double)fn[p * n + i].z;
    }
    f[3 * i] = fx;
    f[3 * i + 1] = fy;
    f[3 * i + 2] = fz;
  }
  double tv = 0, te = 0;
  for (int g = 0; g < T; ++g) {
    tv += (double)evdw[g];
    te += (double)eel[g];
  }
  e[0] = tv;
  e[1] = te;
  return 0;
}

/* The reference's PME influence function: InitDeviceConstants (moduli |b(m)|^2 and
 * exp(-pi^2 m^2 / kappa^2) per dimension) and BCMultiply applied to a grid of ones,
 * so G[(mz * Ky + my) * Kx + mx] = |b|^2 C(m) / (|m|^2 pi K^3) (0 at m = 0). */
int fzr_pme_influence(const int* K, const double* L, double kappa, double* G) {
  if (K[0] > MAXFFT_X || K[1] > MAXFFT_Y || K[2] > MAXFFT_Z) return -1;
  fftx = K[0];
  ffty = K[1];
  fftz = K[2];
  Region = float4{(R)L[0], (R)L[1], (R)L[2], (R)0};
  KAPPa = (R)kappa;
  std::vector<R> m4(NUM_SPLINE_SAMPLES + 1), dm4(NUM_SPLINE_SAMPLES + 1);
  M4d = m4.data();
  dM4d = dm4.data();
  InitDeviceConstants();
  FFTX = K[0];
  FFTY = K[1];
  FFTZ = K[2];
  FFTXH = (R)(K[0] / 2);
  FFTYH = (R)(K[1] / 2);
  FFTZH = (R)(K[2] / 2);
  TOTAL_PME_LATTICES = K[0] * K[1] * K[2];
  box = Region;
  const int T = TOTAL_PME_LATTICES;
  std::vector<cufftComplex> Q(T, cufftComplex{(R)1, (R)0});
  gridDim = fzref_dim3{1, 1, 1};
  blockIdx = fzref_dim3{0, 0, 0};
  blockDim = fzref_dim3{(unsigned)T, 1, 1};
  for (int g = 0; g < T; ++g) {
    threadIdx = fzref_dim3{(unsigned)g, 0, 0};
    BCMultiply(Q.data());
  }
  for (int g = 0; g < T; ++g) G[g] = (double)Q[g].x;
  return 0;
}

}  // extern "C"
