/*
 * FP64 CPU oracle for the FEN ZI molecular-dynamics step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker used by tests/,
 * __graft_entry__.smoke() and the cpu_baseline / reference leg of bench.py.
 * The product library (fenzi_b200/libfenzi_b200.so) never links, loads or
 * calls it, and nothing in the product falls back to it.
 *
 * It restates, in double precision, the functional forms of the reference
 * (TauferLab/fen-zi, SVN "10.24"):
 *   - nonbonded LJ with the CHARMM switch + erfc real-space Ewald
 *       src/nonbonded_forces.cu:114-245, NBFIX/combining src/prmread.cu:2458-2570,2724-2736,
 *       switch coefficients src/mem.cu:556-566
 *   - Ewald exclusion correction for 1-2/1-3 pairs   src/mdcuda.cu:520-553
 *   - 1-4 pairs (1-4 LJ + erfc Coulomb, e14fac = 1)   src/bonded_forces.cu:1155-1268
 *   - bonds / angles / Urey-Bradley / dihedrals / impropers
 *       src/bonded_forces.cu:22-386, 935-991
 *   - exclusion generation (1-2, 1-3 -> Ewald list; + 1-4 -> excluded)
 *       src/prmread.cu:2928-3062 (GenExcl_minimal_new)
 *   - smooth PME, order 4 (Essmann et al., J. Chem. Phys. 103, 8577 (1995)),
 *       influence function src/cell_based_kernels.cu:1770-1903, gather src/pme_kernels.cu:381-573
 *   - self energy  src/prmread.cu:1621,1734
 *   - velocity Verlet in AKMA units src/mdcuda.cu:27-92,354-478, src/dynamics.cu:623-820
 *   - SHAKE / RATTLE (Newton + Gauss elimination per cluster) src/shake.cu:20-615
 *   - kinetic energy / temperature src/evalprops.cu:172-242
 * plus a direct (non-mesh) Ewald reciprocal sum, which the reference does not have,
 * used as the truth for the PME error.
 *
 * Pinned to the reference's own arithmetic: the reference ships no golden outputs and
 * its CUDA build does not compile with CUDA 12.9, but its force kernels compile for the
 * host from its sources (oracle/refbuild.py, oracle/ref_harness.cpp).  Their outputs
 * (tests/golden/ref_terms.npz, made by tests/golden/make_ref_golden.py) agree with this
 * oracle to 1e-12 wherever the formulas coincide, and differ exactly by the documented
 * departures elsewhere (tests/test_ref_pin.py).  Mathematical identities are checked
 * too (F = -dE/dr by finite differences, PME vs direct Ewald, FFT vs numpy).
 */
#ifndef FENZI_ORACLE_H
#define FENZI_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* AKMA unit constants, src/defs.in.h:156-158 */
#define ORC_CC 332.0716
#define ORC_RC 0.001987
#define ORC_TU 20.4548

/* energy slots (same order as the product's fz_energies) */
enum {
  ORC_E_BOND = 0, ORC_E_ANGLE, ORC_E_UREYB, ORC_E_DIHED, ORC_E_IMPR,
  ORC_E_VDW, ORC_E_ELEC, ORC_E_PME, ORC_E_EWEXCL, ORC_E_EWSELF, ORC_NE
};

/* term selection bits for orc_forces */
enum {
  ORC_T_NB = 1, ORC_T_EXCL = 2, ORC_T_P14 = 4, ORC_T_PME = 8,
  ORC_T_BOND = 16, ORC_T_ANGLE = 32, ORC_T_UREYB = 64, ORC_T_DIHED = 128,
  ORC_T_IMPR = 256, ORC_T_SELF = 512,
  ORC_T_ALL = 1023
};

typedef struct orc_system {
  int n;
  const double* q;        /* [n] e */
  const double* mass;     /* [n] amu */
  const int* type;        /* [n] LJ type index */
  int ntypes;
  const double* eps4;     /* [nt*nt] 4*eps_ij (NBFIX already applied) */
  const double* sig2;     /* [nt*nt] sigma_ij^2 */
  const double* eps4_14;  /* [nt*nt] 1-4 variants */
  const double* sig2_14;
  int nbond;  const int* bond;  const double* bond_k;  const double* bond_r0;   /* E = k (r-r0)^2 */
  int nangle; const int* angle; const double* angle_k; const double* angle_t0;  /* rad, E = k (t-t0)^2 */
  int nub;    const int* ub;    const double* ub_k;    const double* ub_r0;     /* atoms 1,3 */
  int ndihe;  const int* dihe;  const double* dihe_k;  const int* dihe_n; const double* dihe_d; /* one row per fold */
  int nimpr;  const int* impr;  const double* impr_k;  const double* impr_p0;
  int ncons;  const int* cons;  const double* cons_d;  /* SHAKE constraints (pairs + length) */
  double box[3];
  double rc, ron, beta;
  int K[3];
  int nthreads;
} orc_system;

void* orc_create(const orc_system* s);
void  orc_destroy(void* h);

/* forces are ADDED to f[3n]; e[ORC_NE] is overwritten */
int orc_forces(void* h, const double* pos, double* f, double* e, int terms);
/* direct reciprocal Ewald sum over |m_i| <= kmax (sphere |m~| <= kmax/min(L)) */
int orc_ewald_recip(void* h, const double* pos, int kmax, double* f, double* e);
/* PME influence function C(m) = |b(m)|^2 exp(-pi^2 |m|^2 / beta^2) / |m|^2 on the grid
 * G[(mz K1 + my) K0 + mx] (0 at m = 0), the factor of the reciprocal sum up to CC/(pi V) */
int orc_pme_influence(const int* K, const double* L, double beta, double* G);
/* in-place 3-D complex DFT, x fastest; sign -1 forward, +1 inverse (unnormalised) */
int orc_fft3d(int nx, int ny, int nz, double* data, int sign);

/* number of excluded (1-2/1-3) pairs, 1-4 pairs, clusters, constraints */
int orc_counts(void* h, int* out4);
/* number of unique non-excluded pairs with r < rcut (roofline pair count) */
long long orc_count_pairs(void* h, const double* pos, double rcut);

/* SHAKE of positions: pos_ref = r(t), pos = unconstrained r(t+dt) (in/out), vel in/out */
int orc_shake(void* h, const double* pos_ref, double* pos, double* vel, double dt_ps, double tol, int maxit);
/* RATTLE of velocities at constrained positions pos */
int orc_rattle(void* h, const double* pos, double* vel);
double orc_kinetic(void* h, const double* vel);

/* velocity Verlet + SHAKE/RATTLE, nsteps; pos/vel in/out; f: forces at the end (out, may be NULL);
 * epot/ekin: per-step traces (length nsteps, may be NULL) */
int orc_md(void* h, double* pos, double* vel, int nsteps, double dt_ps, double tol,
           double* f, double* epot, double* ekin);

/* energy minimisation (the reference's MinimizeStep loop: conjugate gradient, then
 * steepest descent, undoing moves that raise the energy; src/dynamics.cu:491-620,
 * src/mdcuda.cu:126-351, src/fenzi.cu:397-418); pos in/out, per counted step the
 * potential energy and the method (1 CG, 2 SD) of its move (may be NULL); returns the
 * number of counted steps */
int orc_minimize(void* h, double* pos, int max_steps, double cgfac, double sdfac, double cgrate, double sdrate,
                 double* energies, int* methods);
/* Maxwell-Boltzmann velocity reassignment (counter-based RNG shared with the GPU),
 * COM momentum removal, RATTLE projection.  src/init.cu:19-211 */
void orc_reassign_velocities(void* h, const double* pos, double T, uint64_t seed, uint32_t counter, double* vel);
/* the raw counter-based normal deviates used above: out[3n] */
void orc_normals(int n, uint64_t seed, uint32_t counter, double* out);

/* virial diagonal W_aa = -L_a dU/dL_a (central differences, relative step hrel) of the
 * selected terms at the oracle's box: atoms scaled (group = 0, the atomic virial) or the
 * mass centres of the integration units (SHAKE clusters and free atoms) scaled with the
 * units moved rigidly (group = 1, the group virial) */
int orc_virial_fd(void* h, const double* pos, double hrel, int terms, int group, double* vir3);
/* instantaneous constraint virial for positions, velocities and forces f[3n] */
int orc_constraint_virial(void* h, const double* pos, const double* vel, const double* f, double* vir3);
/* pressure (atm) of the unit centres: (2 KE_centres + W_group) / (3 V) */
double orc_group_pressure(void* h, const double* pos, const double* vel, double hrel);
/* Andersen barostat steps with the integration units as scaling groups (the product's
 * splitting: piston half kick, centre-of-mass friction, rigid unit scaling,
 * kick/drift/SHAKE, group pressure from the half-step velocities, piston half kick,
 * kick, friction, RATTLE).  box3 and lstate = {L', L''} in/out; traces of L (x edge)
 * and P (atm) per step (may be NULL). */
int orc_npt(void* h, double* pos, double* vel, double* box3, double* lstate, int nsteps, double dt_ps, double tol,
            double pref_atm, double pmass, double hrel, double* Ltrace, double* Ptrace);

#ifdef __cplusplus
}
#endif
#endif
