// Launch interfaces of the sm_100a kernels (host side of each .cu file).
#pragma once
#include "common.cuh"

namespace fzk {

constexpr int kColCap = 4096;  // atoms per column sorted in shared memory
constexpr int kWarpsPerCta = 8;  // warps of a pair-kernel CTA
constexpr int kNbBatchCtasPerSm = 4;  // CTAs per SM the batched pair kernel is built and launched for
enum : int {
  CNT_TILES = 0, CNT_MASKS, CNT_SLOTS, CNT_REBUILDS, CNT_PRUNES, CNT_WORK, CNT_ITEMS, CNT_COUNT = 8
};
// kernels each launcher issues (the step's launch count)
constexpr int kRebuildBuildLaunches = 6;  // launch_rebuild_build
constexpr int kRebuildPruneLaunches = 3;  // launch_rebuild_prune

// Batched launches: one kernel launch covers many systems.  A block table holds one
// int4 per launched block: (index into the launch's argument array, the block's index
// in that system's own grid, that grid's size, 0).  Tables are built on the host from
// the systems' sizes, one per per-system grid shape.
enum : int {
  BT_ONE = 0,     // one block per system
  BT_ATOMS256,    // (n + 255) / 256
  BT_COLUMNS,     // x-y columns of the neighbour sort
  BT_SLOTS256,    // (sorted slots + 255) / 256
  BT_BLOCKS8,     // (32-slot blocks + 7) / 8
  BT_NB,          // pair-kernel CTAs
  BT_BONDED,      // bonded-term blocks
  BT_BRICKS256,   // (PME bricks + 255) / 256
  BT_BRICKS,      // one block per PME brick
  BT_GRID256,     // (K^3 + 255) / 256
  BT_COUNT
};
struct BatchTables {
  const int4* tab[BT_COUNT];
  int n[BT_COUNT];
};

struct RebuildArgs {
  SysParams p;
  int* flag;
  int* counters;
  int* status;
  float4* pos4;
  float4* pos_build;
  const int* type;
  int *col_of, *col_count, *col_cursor, *col_start, *col_tmp;
  int *perm, *inv_perm;
  float4* xyzq_s;
  int* typ_s;
  float4 *bb_lo, *bb_hi;
  const int *excl_off, *excl_idx;
  int *xn, *xs;  // per slot: count and slots (stride xmax) of its excluded partners
  int xmax;
  int2* xrange;   // per slot: lowest and highest 32-slot block holding one of its partners
  uint32_t* masks;
  int mask_cap, all_images;
  int* blk_col;   // block -> column
  int dcx, dcy;   // column offsets searched for neighbour blocks
  // per-i-block pair lists: outer (rlist, at rebuild) and inner (rc + delta, at prune)
  uint32_t* outer;
  int* outer_n;
  uint32_t* inner;
  int* inner_nt;
  int* inner_m;
  uint32_t* dmask;
  int ocap;
  int* flag_prune;
  float rp2;
  float4* pos_prune;
  int2* items;   // pair-kernel work items (i-block, first tile)
  int chunk;     // tiles per work item
  int prune_split;  // 1: prune with a CTA per i-block (small systems), same lists
  int outer_split;  // 1: outer-list build with a CTA per i-block, same lists
};
// whether the CTA-per-block prune's shared memory (kNG x ocap entries) fits
bool prune_split_fits(int ocap);
void launch_rebuild(const RebuildArgs& a, cudaStream_t st);
// the two halves of launch_rebuild: the outer-list build (flag) and the prune (flag_prune)
void launch_rebuild_build(const RebuildArgs& a, cudaStream_t st);
void launch_rebuild_prune(const RebuildArgs& a, cudaStream_t st);
void launch_rebuild_build_b(const RebuildArgs* args, const BatchTables& t, cudaStream_t st);
void launch_rebuild_prune_b(const RebuildArgs* args, const BatchTables& t, cudaStream_t st);
// one-thread kernel: graph conditional value = (*flag != 0)
// IF-node value = (*flag || (flag2 && *flag2))
void launch_set_condition(cudaGraphConditionalHandle h, const int* flag, const int* flag2, cudaStream_t st);

struct NonbondedArgs {
  SysParams p;
  const float4* xyzq_s;
  const int* typ_s;
  const int* perm;
  const uint32_t* inner;
  const int* inner_nt;
  const int* inner_m;
  const uint32_t* dmask;
  const uint32_t* masks;
  int* counters;        // CNT_ITEMS (work items), CNT_WORK (dynamic item counter, zeroed per launch)
  const int2* items;
  int chunk;
  const float2* ljtab;  // (ntypes+1)^2 (4 eps, sigma^2)
  long long* facc;      // 3 x n fixed point
  long long* energy;    // energy slots
  int ocap;
  int grid;
  int minb;  // CTAs per SM the kernel is built for (3 or 4)
};
void launch_nonbonded(const NonbondedArgs& a, bool energy, cudaStream_t st);
void launch_nonbonded_b(const NonbondedArgs* args, const BatchTables& t, int max_ntypes, cudaStream_t st);

struct PmeArgs {
  SysParams p;
  const float4* pos4;
  int n;
  int K[3];
  int B[3];     // brick edge per dimension
  int nb[3];    // bricks per dimension
  int* brick_of;     // [n]
  int* brick_count;  // [nbricks]
  int* brick_cursor;
  int* brick_start;  // [nbricks+1]
  int* brick_atoms;  // [n]
  float* grid;       // real grid Kz*Ky*Kx: int32 fixed-point charges, then the float potential
  float2* cgrid;     // complex half grid Kz*Ky*(Kx/2+1)
  const float2* tw[3];     // twiddles per dimension (forward, e^{-2 pi i m/K})
  const float* gfac[3];    // per-dim b^2 exp(-pi^2 f^2/beta^2)
  const float* f2[3];      // per-dim f^2 = (m'/L)^2
  float gscale;            // CC / (pi V)
  long long* facc;
  long long* energy;
  int* status;
  int gather;  // gather kernel: 1 one CTA per brick, 2 one thread per atom, 0 by atoms per brick
};
void launch_pme(const PmeArgs& a, bool energy, cudaStream_t st);
// batched PME: the systems of one grid size share the FFT launches
struct PmeSizeBatch {
  int N;                  // Kx = Ky (plane kernels), Kz compiled
  const int4* plane_tab;  // (system, z plane, Kz)
  int nplane;
  const int4* z_tab;      // (system, z-pass group, groups)
  int nz;
};
bool pme_batchable(const PmeArgs& a);
size_t pme_spread_smem(const PmeArgs& a);
int pme_z_groups(const PmeArgs& a);
void launch_pme_b(const PmeArgs* args, const BatchTables& t, const PmeSizeBatch* sizes, int nsizes,
                  size_t spread_smem, cudaStream_t st);
int pme_launches(const PmeArgs& a);

struct BondedArgs {
  SysParams p;
  const float4* pos4;
  int nbond, nangle, nub, ndihe, nimpr, nexcl, n14;
  const int2* bond;   const float2* bond_prm;   // k, r0
  const int4* angle;  const float2* angle_prm;  // k, t0
  const int2* ub;     const float2* ub_prm;
  const int4* dihe;   const float4* dihe_prm;   // k, n, cos d, sin d
  const int4* impr;   const float2* impr_prm;   // k, psi0
  const int2* excl;
  const int2* p14;
  const int* type;
  const float2* lj14;  // (ntypes+1)^2
  long long* facc;
  long long* energy;
};
void launch_bonded(const BondedArgs& a, bool energy, cudaStream_t st);
int bonded_blocks(const BondedArgs& a);
void launch_bonded_b(const BondedArgs* args, const BatchTables& t, cudaStream_t st);

struct IntegrateArgs {
  SysParams p;
  int nunits;
  const int4* unit_atoms;   // -1 padded
  const int* unit_meta;     // na | nc<<4 | pairs<<8 (local a,b 2 bits each)
  const float4* unit_d;     // constraint lengths
  float4* pos4;
  float4* vel4;             // xyz velocity, w = 1/m
  long long* facc;
  float4* xyzq_s;
  const int* inv_perm;
  const float4* pos_build;
  const float4* pos_prune;
  int* flag;
  int* flag_prune;
  float prune_half2;        // (delta/2)^2
  int* status;
  long long* energy;
  double dtu;               // dt * TU
  double box_d[3], inv_box_d[3];
  double shake_tol;
  int shake_maxit;
  int settle;  // every (3 atoms, 3 constraints) unit is a SETTLE triangle, apex first
  int u_begin, u_end;        // unit range of one launch (set by the launchers)
  int ncls;                  // unit classes: units [cls_begin[c], cls_begin[c+1]) have
  int cls_na[8], cls_nc[8];  //   cls_na[c] atoms and cls_nc[c] constraints
  int cls_begin[9];
  float4* min_prev_f;        // minimiser: previous force and search direction per atom
  float4* min_dir;
  int min_method;            //   1 conjugate gradient, 2 steepest descent
  float min_fac;             //   step factor (A per kcal/mol/A)
  double lam;    // barostat step: centre-of-mass scale of every unit (1 = none)
  double vfric;  // barostat step: centre-of-mass velocity scale of the half kicks (1 = none)
};
// kick (F/2) + drift + SHAKE, zeroes the force accumulator, scatters sorted positions
// the units of one class (atoms, constraints, SETTLE) across the systems of a batch:
// args holds one IntegrateArgs per (system, class) with u_begin/u_end of that class
struct ClassBatch {
  int na, nc, settle;
  const IntegrateArgs* args;
  const int4* tab;
  int nblocks;
};
void launch_kick_drift_b(const ClassBatch& c, cudaStream_t st);
void launch_kick_rattle_b(const ClassBatch& c, cudaStream_t st);
void launch_close_kick_drift_b(const ClassBatch& c, cudaStream_t st);
void launch_kick_drift(const IntegrateArgs& a, cudaStream_t st);
// the previous step's closing kick + RATTLE and this step's kick + drift + SHAKE in one
// pass (constant volume; bit-identical to launch_kick_rattle then launch_kick_drift)
void launch_close_kick_drift(const IntegrateArgs& a, cudaStream_t st);
// the same for a barostat step (rigid unit scaling by lam, centre-of-mass velocity
// scale vfric)
void launch_kick_drift_npt(const IntegrateArgs& a, cudaStream_t st);
// barostat step: unit centre-of-mass kinetic energy and intra-unit virial correction
void launch_unit_virial(const IntegrateArgs& a, cudaStream_t st);
// one minimiser move of every unit (forces zeroed, constraints re-imposed, list flags)
void launch_min_step(const IntegrateArgs& a, cudaStream_t st);
// adds the instantaneous constraint virial of the current positions/velocities/forces
void launch_constraint_virial(const IntegrateArgs& a, cudaStream_t st);
// kick (F/2) + RATTLE (+ kinetic energy)
void launch_kick_rattle(const IntegrateArgs& a, bool kinetic, bool kick, cudaStream_t st);
void launch_kinetic(const IntegrateArgs& a, cudaStream_t st);
// Maxwell-Boltzmann draw (counter-based), momentum removal, RATTLE projection
void launch_reassign(const IntegrateArgs& a, double T, uint64_t seed, uint32_t counter, double inv_mtot,
                     long long* psum, cudaStream_t st);

// consharm restraint (src/mdcuda.cu:481-516, src/cell_based_kernels.cu:715-877): every
// atom of segment 1 gets fc (dist + R0 - R1), R the segments' mass centres
void launch_restraint(const SysParams& p, const float4* pos4, const int* seg, const float* mass, long long* acc,
                      double inv_m0, double inv_m1, const double* dist, double fc, long long* facc, cudaStream_t st);

double measure_fp32_peak(int device);

}  // namespace fzk
