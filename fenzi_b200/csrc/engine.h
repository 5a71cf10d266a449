// Device engine of one system: its HBM state, kernel argument builders and the step
// pieces queued on its stream.  Shared by the single-system C ABI (engine.cu) and the
// batched ensemble / serving loop (batch.cu).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host/host.h"
#include "kernels/kernels.h"

namespace fz {

#define FZ_CUDA(call)                                                                                  \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return fail(FZ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct Engine {
  int dev = 0;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  fzk::SysParams p{};
  int n = 0, nunits = 0, ncol = 0, nslots = 0, mask_cap = 0, all_images = 0;
  int ocap = 0;            // per-block pair-list capacity (multiple of 32)
  float rp2 = 0.f, prune_half2 = 0.f;
  int nb_grid = 0, nb_per_sm = 3, n_sm = 148;
  int dcx = 1, dcy = 1;
  int* blk_col = nullptr;
  std::vector<void*> allocs;
  // atoms
  float4 *pos4 = nullptr, *vel4 = nullptr, *pos_build = nullptr;
  long long *facc = nullptr, *energy = nullptr, *psum = nullptr;
  int* type = nullptr;
  // sorted slots / neighbour tiles
  float4 *xyzq_s = nullptr, *bb_lo = nullptr, *bb_hi = nullptr;
  int *typ_s = nullptr, *perm = nullptr, *inv_perm = nullptr, *col_of = nullptr, *col_count = nullptr,
      *col_cursor = nullptr, *col_start = nullptr, *col_tmp = nullptr;
  uint32_t *outer = nullptr, *inner = nullptr, *masks = nullptr, *dmask = nullptr;
  int *outer_n = nullptr, *inner_nt = nullptr, *inner_m = nullptr, *flag_prune = nullptr;
  float4* pos_prune = nullptr;
  int2* items = nullptr;
  int chunk = 16;
  int tiles = 0;  // pair tiles of the first pruned list (sizes the work items)
  int *excl_off = nullptr, *excl_idx = nullptr;
  int *xn = nullptr, *xs = nullptr, xmax = 1;  // per-slot excluded-partner slots
  int2* xrange = nullptr;                          // per slot: partner block range
  int *flag = nullptr, *counters = nullptr, *status = nullptr;
  float2 *ljtab = nullptr, *lj14 = nullptr;
  // bonded
  int nbond = 0, nangle = 0, nub = 0, ndihe = 0, nimpr = 0, nexcl = 0, n14 = 0;
  int2 *bond = nullptr, *ub = nullptr, *excl = nullptr, *p14 = nullptr;
  int4 *angle = nullptr, *dihe = nullptr, *impr = nullptr;
  float2 *bond_prm = nullptr, *angle_prm = nullptr, *ub_prm = nullptr, *impr_prm = nullptr;
  float4* dihe_prm = nullptr;
  int nfixed = 0;  // atoms of fixed (consfix) segments
  // consharm restraint: segment of every atom (0, 1, -1), masses, fixed-point mass
  // centre sums (x0 y0 z0 x1 y1 z1), inverse segment masses, target offset, constant
  bool restraint = false;
  int* rs_seg = nullptr;
  float* rs_mass = nullptr;
  long long* rs_acc = nullptr;
  double rs_inv_m[2] = {0, 0}, rs_dist[3] = {0, 0, 0}, rs_fc = 0;
  // minimiser state (allocated on first use): previous force, search direction,
  // positions before the last move
  float4 *min_prev_f = nullptr, *min_dir = nullptr, *min_pos = nullptr;
  // integration units, grouped in classes of equal (atoms, constraints)
  int ncls = 0, cls_na[8] = {}, cls_nc[8] = {}, cls_begin[9] = {};
  int4* unit_atoms = nullptr;
  int* unit_meta = nullptr;
  float4* unit_d = nullptr;
  // PME
  int K[3] = {0, 0, 0}, B[3] = {0, 0, 0}, nbk[3] = {0, 0, 0};
  int gather_mode = 0;  // PME gather kernel (PmeArgs::gather)
  bool tuned = false;   // launch shapes picked by the autotuner
  int *brick_of = nullptr, *brick_count = nullptr, *brick_cursor = nullptr, *brick_start = nullptr,
      *brick_atoms = nullptr;
  float* grid = nullptr;
  float2* cgrid = nullptr;
  float2* tw[3] = {nullptr, nullptr, nullptr};
  float *gfac[3] = {nullptr, nullptr, nullptr}, *f2[3] = {nullptr, nullptr, nullptr};
  float gscale = 0.f;
  // run state
  bool forces_valid = false;
  long long step = 0;
  double self_energy = 0, inv_mtot = 0, dtu = 0, shake_tol = 1e-10;
  int settle = 0;  // (3,3) units solved by SETTLE (all are symmetric triangles)
  double box_d[3] = {0, 0, 0};
  int ncons = 0;
  int temp_reset_every = 0;
  double temperature = 300.0;
  unsigned long long seed = 0;
  long long launches = 0;
  // per-stage timing
  bool timing = false;
  cudaEvent_t ev[12] = {};
  double stage_ms[5] = {0, 0, 0, 0, 0};
  long long timed_steps = 0;
  // CUDA graph of one MD step (kick/drift/SHAKE, neighbour maintenance, forces,
  // kick/RATTLE); captured on first use, replayed with one launch per step
  cudaGraph_t step_graph = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  // graph of `chunk_steps` consecutive steps (one launch per chunk): replayed for the
  // runs of steps with no velocity reassignment inside; 0 or 1 disables (FZ_GRAPH_CHUNK)
  cudaGraph_t chunk_graph = nullptr;
  cudaGraphExec_t chunk_exec = nullptr;
  int chunk_steps = 100;
  // chunk graphs fuse each step's closing kick + RATTLE into the next step's opening
  // kick + drift pass (FZ_FUSE_CLOSE=0 keeps the two passes apart)
  bool fuse_close = true;
  // prune with one CTA per i-block (systems with few blocks; identical lists)
  int prune_split = 0;
  int outer_split = 0;
  bool use_graph = true;
  // With cond_graph (env FZ_GRAPH_COND=1) the rebuild and prune kernels of captured
  // steps are the bodies of two conditional IF nodes set from the device flags, else
  // flag-checking kernels launched every step; st_cap captures the bodies.
  bool cond_graph = false;
  cudaStream_t st_cap = nullptr;
  cudaError_t capture_error = cudaSuccess;
  long long seen_rb_launch = 0, seen_pr_launch = 0;  // device counters already accounted
  bool graph_since_check = false;                     // captured steps ran since check()
  // PME runs on a second stream concurrently with the pair and bonded kernels
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // pinned staging
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  // Andersen barostat (isotropic; the box keeps its aspect ratios).  L is the x edge;
  // the piston obeys L'' = (P - Pref) / (3 M L^2) - 2 L'^2 / L, P = (2 KE + W) / (3 V)
  // (src/cell_based_kernels.cu:569-579).
  bool npt = false;
  double pmass = 1e-5, pref_atm = 1.0;
  double ratio[3] = {1.0, 1.0, 1.0};
  double Ldot = 0.0, Lacc = 0.0;
  double L_build = 0.0, L_prune = 0.0;  // box x edge at the last list build / prune
  long long seen_rebuilds = 0, seen_prunes = 0;
  double last_pressure = 0.0;
  double plist = 0.0, cutoff = 0.0, col_a = 0.0;
  float skin_half2_nve = 0.f, prune_half2_nve = 0.f;
  double prune_delta = 0.0;
  float* pme_tab_host = nullptr;  // pinned: gfac|f2 per dimension
  int ncx = 1, ncy = 1;

  template <class T>
  fz_status alloc(T** ptr, size_t count) {
    *ptr = nullptr;
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) return fail(FZ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    e = cudaMemsetAsync(p, 0, count * sizeof(T), st);
    if (e != cudaSuccess) return fail(FZ_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    *ptr = static_cast<T*>(p);
    return FZ_OK;
  }
  template <class T>
  fz_status upload(T** ptr, const std::vector<T>& v) {
    fz_status s = alloc(ptr, v.size());
    if (s) return s;
    if (!v.empty()) FZ_CUDA(cudaMemcpyAsync(*ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return FZ_OK;
  }
  void release(void* ptr) {
    for (auto& a : allocs)
      if (a == ptr) {
        cudaFree(a);
        a = allocs.back();
        allocs.pop_back();
        return;
      }
  }
  fz_status staging(size_t bytes) {
    if (pinned_bytes >= bytes) return FZ_OK;
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    FZ_CUDA(cudaMallocHost(&pinned, bytes));
    pinned_bytes = bytes;
    return FZ_OK;
  }
  ~Engine() {
    if (st) cudaStreamSynchronize(st);
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (step_graph) cudaGraphDestroy(step_graph);
    if (chunk_exec) cudaGraphExecDestroy(chunk_exec);
    if (chunk_graph) cudaGraphDestroy(chunk_graph);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st2) cudaStreamDestroy(st2);
    if (st_cap) cudaStreamDestroy(st_cap);
    for (auto& x : ev)
      if (x) cudaEventDestroy(x);
    for (void* p : allocs) cudaFree(p);
    if (pinned) cudaFreeHost(pinned);
    if (pme_tab_host) cudaFreeHost(pme_tab_host);
    if (own_stream && st) cudaStreamDestroy(st);
  }

  fzk::RebuildArgs rebuild_args() const {
    fzk::RebuildArgs a{};
    a.p = p;
    a.flag = flag;
    a.counters = counters;
    a.status = status;
    a.pos4 = pos4;
    a.pos_build = pos_build;
    a.type = type;
    a.col_of = col_of;
    a.col_count = col_count;
    a.col_cursor = col_cursor;
    a.col_start = col_start;
    a.col_tmp = col_tmp;
    a.perm = perm;
    a.inv_perm = inv_perm;
    a.xyzq_s = xyzq_s;
    a.typ_s = typ_s;
    a.bb_lo = bb_lo;
    a.bb_hi = bb_hi;
    a.excl_off = excl_off;
    a.excl_idx = excl_idx;
    a.xn = xn;
    a.xs = xs;
    a.xrange = xrange;
    a.xmax = xmax;
    a.masks = masks;
    a.mask_cap = mask_cap;
    a.all_images = all_images;
    a.outer = outer;
    a.outer_n = outer_n;
    a.inner = inner;
    a.inner_nt = inner_nt;
    a.inner_m = inner_m;
    a.dmask = dmask;
    a.ocap = ocap;
    a.flag_prune = flag_prune;
    a.rp2 = rp2;
    a.pos_prune = pos_prune;
    a.items = items;
    a.chunk = chunk;
    a.prune_split = prune_split;
    a.outer_split = outer_split;
    a.blk_col = blk_col;
    a.dcx = dcx;
    a.dcy = dcy;
    return a;
  }
  fzk::NonbondedArgs nb_args() const {
    fzk::NonbondedArgs a{};
    a.p = p;
    a.xyzq_s = xyzq_s;
    a.typ_s = typ_s;
    a.perm = perm;
    a.inner = inner;
    a.inner_nt = inner_nt;
    a.inner_m = inner_m;
    a.dmask = dmask;
    a.masks = masks;
    a.counters = counters;
    a.ljtab = ljtab;
    a.facc = facc;
    a.energy = energy;
    a.ocap = ocap;
    a.items = items;
    a.chunk = chunk;
    a.grid = nb_grid;
    // FZ_NB_GRID_PER_SM: fewer CTAs than the build's occupancy, leaving room on every SM
    // for the PME kernels of the second stream (a measurement knob)
    if (const char* v = std::getenv("FZ_NB_GRID_PER_SM")) a.grid = n_sm * std::max(1, std::min(8, std::atoi(v)));
    a.minb = nb_per_sm;
    return a;
  }
  fzk::PmeArgs pme_args() const {
    fzk::PmeArgs a{};
    a.p = p;
    a.pos4 = pos4;
    a.n = n;
    for (int d = 0; d < 3; ++d) {
      a.K[d] = K[d];
      a.B[d] = B[d];
      a.nb[d] = nbk[d];
      a.tw[d] = tw[d];
      a.gfac[d] = gfac[d];
      a.f2[d] = f2[d];
    }
    a.brick_of = brick_of;
    a.brick_count = brick_count;
    a.brick_cursor = brick_cursor;
    a.brick_start = brick_start;
    a.brick_atoms = brick_atoms;
    a.grid = grid;
    a.cgrid = cgrid;
    a.gscale = gscale;
    a.facc = facc;
    a.energy = energy;
    a.status = status;
    a.gather = gather_mode;
    return a;
  }
  fzk::BondedArgs bonded_args() const {
    fzk::BondedArgs a{};
    a.p = p;
    a.pos4 = pos4;
    a.nbond = nbond;
    a.nangle = nangle;
    a.nub = nub;
    a.ndihe = ndihe;
    a.nimpr = nimpr;
    a.nexcl = nexcl;
    a.n14 = n14;
    a.bond = bond;
    a.bond_prm = bond_prm;
    a.angle = angle;
    a.angle_prm = angle_prm;
    a.ub = ub;
    a.ub_prm = ub_prm;
    a.dihe = dihe;
    a.dihe_prm = dihe_prm;
    a.impr = impr;
    a.impr_prm = impr_prm;
    a.excl = excl;
    a.p14 = p14;
    a.type = type;
    a.lj14 = lj14;
    a.facc = facc;
    a.energy = energy;
    return a;
  }
  fzk::IntegrateArgs int_args() const {
    fzk::IntegrateArgs a{};
    a.p = p;
    a.nunits = nunits;
    a.unit_atoms = unit_atoms;
    a.unit_meta = unit_meta;
    a.unit_d = unit_d;
    a.pos4 = pos4;
    a.vel4 = vel4;
    a.facc = facc;
    a.xyzq_s = xyzq_s;
    a.inv_perm = inv_perm;
    a.pos_build = pos_build;
    a.pos_prune = pos_prune;
    a.flag = flag;
    a.flag_prune = flag_prune;
    a.prune_half2 = prune_half2;
    a.status = status;
    a.energy = energy;
    a.dtu = dtu;
    for (int d = 0; d < 3; ++d) {
      a.box_d[d] = box_d[d];
      a.inv_box_d[d] = 1.0 / box_d[d];
    }
    a.shake_tol = shake_tol;
    a.shake_maxit = 500;
    a.settle = settle;
    a.lam = 1.0;
    a.vfric = 1.0;
    a.u_begin = 0;
    a.u_end = nunits;
    a.ncls = ncls;
    for (int c = 0; c < 8; ++c) {
      a.cls_na[c] = cls_na[c];
      a.cls_nc[c] = cls_nc[c];
    }
    for (int c = 0; c < 9; ++c) a.cls_begin[c] = cls_begin[c];
    return a;
  }

  // ---------------------------------------------------------------- step pieces
  void mark(int k) {
    if (timing) cudaEventRecord(ev[k], st);
  }
  void forces(bool energies, int terms = FZ_TERM_ALL) {
    mark(1);
    fzk::launch_rebuild(rebuild_args(), st);
    launches += fzk::kRebuildBuildLaunches + fzk::kRebuildPruneLaunches;
    mark(2);
    if (terms & FZ_TERM_NONBONDED) {
      fzk::launch_nonbonded(nb_args(), energies, st);
      launches += 1;
    }
    mark(3);
    if (terms & (FZ_TERM_BONDED | FZ_TERM_BONDED_PARTS)) {
      fzk::BondedArgs a = bonded_args();
      if (!(terms & FZ_TERM_BONDED)) {
        // selected parts only: the kernel's flattened term range skips empty classes
        if (!(terms & FZ_TERM_BONDS)) a.nbond = 0;
        if (!(terms & FZ_TERM_ANGLES)) a.nangle = 0;
        if (!(terms & FZ_TERM_UREYB)) a.nub = 0;
        if (!(terms & FZ_TERM_DIHEDRALS)) a.ndihe = 0;
        if (!(terms & FZ_TERM_IMPROPERS)) a.nimpr = 0;
        if (!(terms & FZ_TERM_PAIRS14)) a.n14 = 0;
        if (!(terms & FZ_TERM_EXCLUSIONS)) a.nexcl = 0;
      }
      fzk::launch_bonded(a, energies, st);
      launches += bonded_launches();
    }
    if ((terms & FZ_TERM_BONDED) && restraint) {
      restraint_forces(st);
      launches += 2;
    }
    mark(4);
    if (terms & FZ_TERM_PME) {
      fzk::launch_pme(pme_args(), energies, st);
      launches += fzk::pme_launches(pme_args());
    }
    mark(5);
  }
  // accumulates the events of one timed step: 0 start, 1..5 forces, 6 end
  void collect_step() {
    cudaEventSynchronize(ev[6]);
    float ms = 0.f;
    auto el = [&](int a, int b) {
      cudaEventElapsedTime(&ms, ev[a], ev[b]);
      return (double)ms;
    };
    stage_ms[0] += el(1, 2);
    stage_ms[1] += el(2, 3);
    stage_ms[2] += el(3, 4);
    stage_ms[3] += el(4, 5);
    stage_ms[4] += el(0, 1) + el(5, 6);
    timed_steps++;
  }
  // consharm: mass centres of the two segments, then the pull on segment 1's atoms
  void restraint_forces(cudaStream_t s) {
    cudaMemsetAsync(rs_acc, 0, 8 * sizeof(long long), s);
    fzk::launch_restraint(p, pos4, rs_seg, rs_mass, rs_acc, rs_inv_m[0], rs_inv_m[1], rs_dist, rs_fc, facc, s);
  }
  // Adds to the capture on st an IF node that runs body(stream) when *dflag != 0 (or
  // *dflag2 != 0 when given).
  template <class F>
  void conditional(const int* dflag, const int* dflag2, F body) {
    cudaStreamCaptureStatus cs;
    unsigned long long id;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
    if (e != cudaSuccess) {
      capture_error = e;
      return;
    }
    fzk::launch_set_condition(h, dflag, dflag2, st);
    e = cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, nd, &np);
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(st_cap, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      capture_error = e;
      return;
    }
    body(st_cap);
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(st_cap, &out);
    if (e != cudaSuccess) capture_error = e;
  }
  // neighbour maintenance: conditional nodes inside a capture, else flag-checking kernels
  bool capturing_conditional() {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cond_graph && st_cap && cudaStreamIsCapturing(st, &cs) == cudaSuccess &&
           cs == cudaStreamCaptureStatusActive;
  }
  // list rebuild when due (it wraps the positions, so it precedes every reader)
  void rebuild_build_step() {
    const fzk::RebuildArgs ra = rebuild_args();
    if (capturing_conditional()) conditional(flag, nullptr, [&](cudaStream_t s) { fzk::launch_rebuild_build(ra, s); });
    else fzk::launch_rebuild_build(ra, st);
  }
  // inner-list prune when due (reads the sorted positions, writes only list data)
  void prune_step() {
    const fzk::RebuildArgs ra = rebuild_args();
    // a rebuild this step (flag still raised) always ends in a prune
    if (capturing_conditional())
      conditional(flag_prune, flag, [&](cudaStream_t s) { fzk::launch_rebuild_prune(ra, s); });
    else fzk::launch_rebuild_prune(ra, st);
  }
  void rebuild_step() {
    rebuild_build_step();
    prune_step();
  }
  // kernels one captured step launches besides the conditional bodies
  long long graph_step_launches() const {
    return 2 * ncls + (cond_graph ? 2 : fzk::kRebuildBuildLaunches + fzk::kRebuildPruneLaunches) + 1 +
           bonded_launches() + fzk::pme_launches(pme_args()) + (restraint ? 2 : 0);
  }
  int bonded_launches() const { return (nbond + nangle + nub + ndihe + nimpr + nexcl + n14 > 0) ? 1 : 0; }
  // launches of the conditional bodies (per rebuild and per prune) since the last
  // call, from the device counters; called after a synchronisation
  void account_conditional(const int* cnt) {
    if (cond_graph && graph_since_check)
      launches += fzk::kRebuildBuildLaunches * (cnt[fzk::CNT_REBUILDS] - seen_rb_launch) +
                  fzk::kRebuildPruneLaunches * (cnt[fzk::CNT_PRUNES] - seen_pr_launch);
    graph_since_check = false;
    seen_rb_launch = cnt[fzk::CNT_REBUILDS];
    seen_pr_launch = cnt[fzk::CNT_PRUNES];
  }
  // forces with PME on st2, overlapping the pair and bonded kernels on st
  // (PME needs only the positions, so it starts before the prune and overlaps it too)
  void forces_overlapped() {
    rebuild_build_step();
    cudaEventRecord(ev_fork, st);
    cudaStreamWaitEvent(st2, ev_fork, 0);
    fzk::launch_pme(pme_args(), false, st2);
    prune_step();
    fzk::launch_nonbonded(nb_args(), false, st);
    fzk::launch_bonded(bonded_args(), false, st);
    if (restraint) restraint_forces(st);
    cudaEventRecord(ev_join, st2);
    cudaStreamWaitEvent(st, ev_join, 0);
  }
  // One integrator pass over all unit classes; with a second stream the first class
  // (free atoms) runs beside the others: classes touch disjoint atoms.
  template <class L>
  void integrate_classes(const fzk::IntegrateArgs& ia, L launch) {
    if (!st2 || ia.ncls < 2) {
      launch(ia, st);
      return;
    }
    fzk::IntegrateArgs first = ia, rest = ia;
    first.ncls = 1;
    rest.ncls = ia.ncls - 1;
    for (int c = 0; c < rest.ncls; ++c) {
      rest.cls_na[c] = ia.cls_na[c + 1];
      rest.cls_nc[c] = ia.cls_nc[c + 1];
      rest.cls_begin[c] = ia.cls_begin[c + 1];
    }
    rest.cls_begin[rest.ncls] = ia.cls_begin[ia.ncls];
    cudaEventRecord(ev_fork, st);
    cudaStreamWaitEvent(st2, ev_fork, 0);
    launch(first, st2);
    launch(rest, st);
    cudaEventRecord(ev_join, st2);
    cudaStreamWaitEvent(st, ev_join, 0);
  }
  // One MD step.  open: the step starts with its own kick + drift pass (else the
  // previous step left its closing kick + RATTLE to this step's first pass); close: the
  // step ends with the kick + RATTLE pass (else the next step's first pass does it).
  void step_body(bool open = true, bool close = true) {
    const fzk::IntegrateArgs ia = int_args();
    if (open)
      integrate_classes(ia, [](const fzk::IntegrateArgs& a, cudaStream_t s) { fzk::launch_kick_drift(a, s); });
    else
      integrate_classes(ia, [](const fzk::IntegrateArgs& a, cudaStream_t s) { fzk::launch_close_kick_drift(a, s); });
    if (st2)
      forces_overlapped();
    else
      forces(false);
    if (close)
      integrate_classes(ia, [](const fzk::IntegrateArgs& a, cudaStream_t s) {
        fzk::launch_kick_rattle(a, false, true, s);
      });
  }
  fz_status graph_step() {
    if (!step_exec) {
      capture_error = cudaSuccess;
      FZ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const long long l0 = launches;
      step_body();
      launches = l0;
      cudaGraph_t g = nullptr;
      FZ_CUDA(cudaStreamEndCapture(st, &g));
      step_graph = g;
      if (capture_error != cudaSuccess)
        return fail(FZ_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(capture_error));
      FZ_CUDA(cudaGraphInstantiate(&step_exec, step_graph, 0));
    }
    FZ_CUDA(cudaGraphLaunch(step_exec, st));
    launches += graph_step_launches();
    graph_since_check = true;
    return FZ_OK;
  }
  // chunk_steps steps in one graph launch (captured on first use)
  fz_status graph_chunk() {
    if (!chunk_exec) {
      capture_error = cudaSuccess;
      FZ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const long long l0 = launches;
      // inside the chunk each step's closing pass joins the next step's opening one
      for (int k = 0; k < chunk_steps; ++k) step_body(k == 0 || !fuse_close, k == chunk_steps - 1 || !fuse_close);
      launches = l0;
      cudaGraph_t g = nullptr;
      FZ_CUDA(cudaStreamEndCapture(st, &g));
      chunk_graph = g;
      if (capture_error != cudaSuccess)
        return fail(FZ_ERR_CUDA, std::string("chunk capture: ") + cudaGetErrorString(capture_error));
      FZ_CUDA(cudaGraphInstantiate(&chunk_exec, chunk_graph, 0));
    }
    FZ_CUDA(cudaGraphLaunch(chunk_exec, st));
    launches += (long long)chunk_steps * graph_step_launches() - (fuse_close ? (long long)(chunk_steps - 1) * ncls : 0);
    graph_since_check = true;
    return FZ_OK;
  }
  void drop_graph() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (step_graph) cudaGraphDestroy(step_graph);
    if (chunk_exec) cudaGraphExecDestroy(chunk_exec);
    if (chunk_graph) cudaGraphDestroy(chunk_graph);
    step_exec = nullptr;
    step_graph = nullptr;
    chunk_exec = nullptr;
    chunk_graph = nullptr;
  }
  fz_status check() {
    int h = 0;
    int cnt[fzk::CNT_COUNT];
    FZ_CUDA(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    FZ_CUDA(cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    FZ_CUDA(cudaStreamSynchronize(st));
    FZ_CUDA(cudaGetLastError());
    account_conditional(cnt);
    if (h) {
      std::string m = "device status:";
      if (h & fzk::ST_TILE_OVERFLOW) m += " pair-tile capacity exceeded;";
      if (h & fzk::ST_MASK_OVERFLOW) m += " exclusion-mask capacity exceeded;";
      if (h & fzk::ST_SLOT_OVERFLOW) m += " sorted-slot capacity exceeded;";
      if (h & fzk::ST_COLUMN_OVERFLOW) m += " column occupancy exceeded;";
      if (h & fzk::ST_SHAKE_NOCONV) m += " SHAKE did not converge within its iteration cap;";
      if (h & fzk::ST_BAD_COORD) m += " non-finite or runaway coordinates;";
      const int code = (h & fzk::ST_SHAKE_NOCONV) ? FZ_ERR_SHAKE : FZ_ERR_CAPACITY;
      return fail(code, m);
    }
    return FZ_OK;
  }
};

// moves an engine to the box with x edge L (aspect ratios kept): kernel parameters,
// column reach and PME influence tables (engine.cu)
fz_status set_box(Engine* e, double L);

}  // namespace fz
