// Device engine: owns a system's HBM state and queues the MD step on one stream.
// Replaces InitMem / InitDeviceConstants (src/mem.cu:49-727,
// src/cell_based_kernels.cu:1831-1947), ComputeAccelGPU (src/mdcuda.cu:557-849),
// SingleStep (src/dynamics.cu:623-820), InitVelocity (src/init.cu:19-211) and the
// D2H side of EvalProps (src/evalprops.cu:17-308).
//
// HBM layout (all in original atom order unless noted):
//   pos4  float4[n]   x, y, z, q          vel4 float4[n]  vx, vy, vz, 1/m
//   facc  int64[3n]   force accumulator, fixed point 2^32, SoA x|y|z
//   xyzq_s float4[S], typ_s int[S], perm int[S]   sorted slots (S = n + 32*columns + 32)
//   outer/inner uint32[blocks x ocap]            per-block pair lists (kernels/neighbor.cu):
//                                                outer at rlist (rebuild), inner at rc + 0.3 (prune)
//   grid float[K^3], cgrid float2[Kz*Ky*(Kx/2+1)] PME
// A step is ~20 launches and no host synchronisation; fz_step checks the sticky
// device status word once per call.
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
  int nb_grid = 0;
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
  int *excl_off = nullptr, *excl_idx = nullptr;
  int *flag = nullptr, *counters = nullptr, *status = nullptr;
  float2 *ljtab = nullptr, *lj14 = nullptr;
  // bonded
  int nbond = 0, nangle = 0, nub = 0, ndihe = 0, nimpr = 0, nexcl = 0, n14 = 0;
  int2 *bond = nullptr, *ub = nullptr, *excl = nullptr, *p14 = nullptr;
  int4 *angle = nullptr, *dihe = nullptr, *impr = nullptr;
  float2 *bond_prm = nullptr, *angle_prm = nullptr, *ub_prm = nullptr, *impr_prm = nullptr;
  float4* dihe_prm = nullptr;
  // integration units
  int4* unit_atoms = nullptr;
  int* unit_meta = nullptr;
  float4* unit_d = nullptr;
  // PME
  int K[3] = {0, 0, 0}, B[3] = {0, 0, 0}, nbk[3] = {0, 0, 0};
  int *brick_of = nullptr, *brick_count = nullptr, *brick_cursor = nullptr, *brick_start = nullptr,
      *brick_atoms = nullptr;
  float* grid = nullptr;
  int* qgrid = nullptr;
  float2* cgrid = nullptr;
  float2* tw[3] = {nullptr, nullptr, nullptr};
  float *gfac[3] = {nullptr, nullptr, nullptr}, *f2[3] = {nullptr, nullptr, nullptr};
  float gscale = 0.f;
  // run state
  bool forces_valid = false;
  long long step = 0;
  double self_energy = 0, inv_mtot = 0, dtu = 0, shake_tol = 1e-10;
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
  bool use_graph = true;
  // PME runs on a second stream concurrently with the pair and bonded kernels
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // pinned staging
  void* pinned = nullptr;
  size_t pinned_bytes = 0;

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
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st2) cudaStreamDestroy(st2);
    for (auto& x : ev)
      if (x) cudaEventDestroy(x);
    for (void* p : allocs) cudaFree(p);
    if (pinned) cudaFreeHost(pinned);
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
    a.qgrid = qgrid;
    a.cgrid = cgrid;
    a.gscale = gscale;
    a.facc = facc;
    a.energy = energy;
    a.status = status;
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
    return a;
  }

  // ---------------------------------------------------------------- step pieces
  void mark(int k) {
    if (timing) cudaEventRecord(ev[k], st);
  }
  void forces(bool energies, int terms = FZ_TERM_ALL) {
    mark(1);
    fzk::launch_rebuild(rebuild_args(), st);
    launches += 11;
    mark(2);
    if (terms & FZ_TERM_NONBONDED) {
      fzk::launch_nonbonded(nb_args(), energies, st);
      launches += 1;
    }
    mark(3);
    if (terms & FZ_TERM_BONDED) {
      fzk::launch_bonded(bonded_args(), energies, st);
      launches += (nbond + nangle + nub + ndihe + nimpr + nexcl + n14 > 0) ? 1 : 0;
    }
    mark(4);
    if (terms & FZ_TERM_PME) {
      fzk::launch_pme(pme_args(), energies, st);
      launches += 11;
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
  // forces with PME on st2, overlapping the pair and bonded kernels on st
  void forces_overlapped() {
    fzk::launch_rebuild(rebuild_args(), st);
    cudaEventRecord(ev_fork, st);
    cudaStreamWaitEvent(st2, ev_fork, 0);
    fzk::launch_pme(pme_args(), false, st2);
    fzk::launch_nonbonded(nb_args(), false, st);
    fzk::launch_bonded(bonded_args(), false, st);
    cudaEventRecord(ev_join, st2);
    cudaStreamWaitEvent(st, ev_join, 0);
  }
  void step_body() {
    const fzk::IntegrateArgs ia = int_args();
    fzk::launch_kick_drift(ia, st);
    if (st2)
      forces_overlapped();
    else
      forces(false);
    fzk::launch_kick_rattle(ia, false, true, st);
  }
  fz_status graph_step() {
    if (!step_exec) {
      FZ_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const long long l0 = launches;
      step_body();
      launches = l0;
      cudaGraph_t g = nullptr;
      FZ_CUDA(cudaStreamEndCapture(st, &g));
      step_graph = g;
      FZ_CUDA(cudaGraphInstantiate(&step_exec, step_graph, 0));
    }
    FZ_CUDA(cudaGraphLaunch(step_exec, st));
    launches += 2 + 11 + 1 + ((nbond + nangle + nub + ndihe + nimpr + nexcl + n14 > 0) ? 1 : 0) + 11;
    return FZ_OK;
  }
  void drop_graph() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (step_graph) cudaGraphDestroy(step_graph);
    step_exec = nullptr;
    step_graph = nullptr;
  }
  fz_status check() {
    int h = 0;
    FZ_CUDA(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    FZ_CUDA(cudaStreamSynchronize(st));
    FZ_CUDA(cudaGetLastError());
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

void destroy_engine(Engine* e) { delete e; }

static int brick_edge(int K) {
  // largest divisor of K in [4, 16] that still gives >= 256 bricks (one CTA each);
  // else the smallest divisor >= 4 (brick edge >= 3 keeps the stencil halo one brick deep)
  int best = 0;
  for (int d = 4; d <= 16; ++d)
    if (K % d == 0 && (K / d) * (K / d) * (K / d) >= 256) best = d;
  if (best) return best;
  for (int d = 4; d <= K; ++d)
    if (K % d == 0) return d;
  return K;
}

static bool fft_size_ok(int n) {
  if (n < 2 || n > 1024) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

static double bmod2(int m, int K) {
  const double M4v[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
  double re = 0, im = 0;
  for (int k = 0; k < 3; ++k) {
    const double a = 2.0 * M_PI * (double)m * k / K;
    re += M4v[k] * std::cos(a);
    im += M4v[k] * std::sin(a);
  }
  return 1.0 / (re * re + im * im);
}

static fz_status build_engine(fz_system* s, int device, void* stream) {
  const Topology& t = s->top;
  const fz_config& c = s->cfg;
  Engine* e = new Engine();
  s->eng = e;
  e->dev = device;
  FZ_CUDA(cudaSetDevice(device));
  if (stream) {
    e->st = (cudaStream_t)stream;
  } else {
    FZ_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
    e->own_stream = true;
  }
  FZ_CUDA(cudaStreamCreateWithFlags(&e->st2, cudaStreamNonBlocking));
  FZ_CUDA(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
  FZ_CUDA(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
  const int n = t.n;
  e->n = n;
  const int nt = (int)t.type_names.size();
  // ---- parameters
  fzk::SysParams& p = e->p;
  p.box = make_float3((float)c.box[0], (float)c.box[1], (float)c.box[2]);
  for (int d = 0; d < 3; ++d) e->box_d[d] = c.box[d];
  p.inv_box = make_float3((float)(1.0 / c.box[0]), (float)(1.0 / c.box[1]), (float)(1.0 / c.box[2]));
  const double rc = c.cutoff, ron = std::min(c.cuton, c.cutoff);
  p.rc2 = (float)(rc * rc);
  p.ron2 = (float)(ron * ron);
  p.sw_c3 = rc > ron ? (float)(1.0 / std::pow(rc * rc - ron * ron, 3)) : 0.f;
  p.beta = (float)c.kappa;
  p.cc = (float)kCC;
  const double plist = std::max(c.pairlistdist, c.cutoff);
  p.skin_half2 = (float)std::pow(0.5 * (plist - c.cutoff), 2);
  p.rlist = (float)plist;
  p.n = n;
  p.ntypes = nt;
  const double lmin = std::min(c.box[0], std::min(c.box[1], c.box[2]));
  if (rc >= 0.5 * lmin) return fail(FZ_ERR_ARG, "cutoff must be below half the smallest box edge");
  const double V = c.box[0] * c.box[1] * c.box[2];
  const double rho = n / V;
  const double a = std::cbrt(32.0 / rho);
  int ncx = std::max(1, (int)std::floor(c.box[0] / a)), ncy = std::max(1, (int)std::floor(c.box[1] / a));
  while ((double)n / (ncx * ncy) > fzk::kColCap / 2 && (ncx < 4096 && ncy < 4096)) {
    ncx *= 2;
    ncy *= 2;
  }
  p.ncol[0] = ncx;
  p.ncol[1] = ncy;
  e->ncol = ncx * ncy;
  const double colw = std::max(c.box[0] / ncx, c.box[1] / ncy);
  e->all_images = (0.5 * lmin < plist + 3.0 * std::max(colw, a)) ? 1 : 0;
  // column offsets whose x-y rectangles can lie within the pair-list radius
  e->dcx = std::min(ncx, (int)std::ceil(plist / (c.box[0] / ncx)));
  e->dcy = std::min(ncy, (int)std::ceil(plist / (c.box[1] / ncy)));
  e->nslots = ((n + 32 * e->ncol + 64 + 31) / 32) * 32;
  p.nslots = e->nslots;
  for (int d = 0; d < 3; ++d) {
    e->K[d] = c.pme_grid[d];
    if (!fft_size_ok(e->K[d])) return fail(FZ_ERR_ARG, "PME grid sizes must be 2^a 3^b 5^c in [2, 1024]");
    e->B[d] = brick_edge(e->K[d]);
    e->nbk[d] = e->K[d] / e->B[d];
    p.K[d] = e->K[d];
  }
  // per-block list capacity: atoms within rlist of a block box (Minkowski volume of a
  // box ~1.4 a), with room for blocks that see all their neighbours at higher index
  const double ab = 1.4 * a, R = plist;
  const double vm = ab * ab * ab + 6 * ab * ab * R + 3 * M_PI * ab * R * R + 4.0 / 3.0 * M_PI * R * R * R;
  e->ocap = (int)std::ceil(std::max(256.0, 1.25 * rho * vm) / 32.0) * 32;
  e->mask_cap = (e->nslots / 32) * (e->ocap / 32);
  {
    const double delta = std::min(0.3, plist - c.cutoff);
    e->rp2 = (float)((c.cutoff + delta) * (c.cutoff + delta));
    e->prune_half2 = (float)(0.25 * delta * delta);
  }
  e->dtu = c.timestep_ps * kTU;
  e->shake_tol = c.shake_tol > 0 ? c.shake_tol : 1e-10;
  e->temp_reset_every = c.temp_reset_every;
  e->temperature = c.temperature;
  e->seed = (unsigned long long)c.seed;
  e->self_energy = t.self_energy;
  e->ncons = (int)t.cons_d.size();
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  // pair kernel CTAs per SM (3 = register-limited maximum); PME overlaps it on a second stream
  {
    const char* v = std::getenv("FZ_NB_CTAS_PER_SM");
    const int per = v ? std::max(1, std::min(3, std::atoi(v))) : 3;
    e->nb_grid = dev_sms * per;
  }
  // ---- atom arrays
  std::vector<float4> pos4(n), vel4(n);
  double mt = 0;
  for (int i = 0; i < n; ++i) {
    pos4[i] = make_float4((float)t.pos[3 * i], (float)t.pos[3 * i + 1], (float)t.pos[3 * i + 2], (float)t.q[i]);
    vel4[i] = make_float4(0.f, 0.f, 0.f, t.mass[i] > 0 ? (float)(1.0 / t.mass[i]) : 0.f);
    mt += t.mass[i];
  }
  e->inv_mtot = mt > 0 ? 1.0 / mt : 0.0;
  fz_status r;
  if ((r = e->upload(&e->pos4, pos4)) || (r = e->upload(&e->vel4, vel4)) || (r = e->alloc(&e->pos_build, n)) ||
      (r = e->alloc(&e->facc, 3 * (size_t)n)) || (r = e->alloc(&e->energy, fzk::EN_COUNT)) ||
      (r = e->alloc(&e->psum, 4)) || (r = e->upload(&e->type, t.type)))
    return r;
  // ---- sorted slots, columns, tiles
  const int nslots = e->nslots, nblk = nslots / 32;
  if ((r = e->alloc(&e->xyzq_s, nslots)) || (r = e->alloc(&e->typ_s, nslots)) || (r = e->alloc(&e->perm, nslots)) ||
      (r = e->alloc(&e->inv_perm, n)) || (r = e->alloc(&e->col_of, n)) || (r = e->alloc(&e->col_count, e->ncol)) ||
      (r = e->alloc(&e->col_cursor, e->ncol)) || (r = e->alloc(&e->col_start, e->ncol + 1)) ||
      (r = e->alloc(&e->col_tmp, nslots)) || (r = e->alloc(&e->bb_lo, nblk)) || (r = e->alloc(&e->blk_col, nblk)) || (r = e->alloc(&e->bb_hi, nblk)) ||
      (r = e->alloc(&e->outer, (size_t)nblk * e->ocap)) || (r = e->alloc(&e->inner, (size_t)nblk * e->ocap)) ||
      (r = e->alloc(&e->outer_n, nblk)) || (r = e->alloc(&e->inner_nt, nblk)) ||
      (r = e->alloc(&e->inner_m, (size_t)nblk * (e->ocap / 32))) || (r = e->alloc(&e->dmask, (size_t)nblk * 32)) ||
      (r = e->alloc(&e->masks, (size_t)e->mask_cap * 32)) || (r = e->alloc(&e->pos_prune, n)) ||
      (r = e->alloc(&e->flag_prune, 1)) || (r = e->alloc(&e->items, (size_t)nblk * (e->ocap / 32 + 1))) ||
      (r = e->alloc(&e->flag, 1)) || (r = e->alloc(&e->counters, fzk::CNT_COUNT)) || (r = e->alloc(&e->status, 1)))
    return r;
  {
    // the permanent dummy slot (last) used to pad partial tiles: far away, q = 0, padding type
    std::vector<float4> dummy(32);
    std::vector<int> dt(32, nt), dp(32, -1);
    for (int k = 0; k < 32; ++k) dummy[k] = make_float4(1.0e6f + (float)(nslots - 32 + k), 1.0e6f, 1.0e6f, 0.f);
    FZ_CUDA(cudaMemcpyAsync(e->xyzq_s + nslots - 32, dummy.data(), 32 * sizeof(float4), cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaMemcpyAsync(e->typ_s + nslots - 32, dt.data(), 32 * sizeof(int), cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaMemcpyAsync(e->perm + nslots - 32, dp.data(), 32 * sizeof(int), cudaMemcpyHostToDevice, e->st));
  }
  if ((r = e->upload(&e->excl_off, t.excl_off)) || (r = e->upload(&e->excl_idx, t.excl_idx))) return r;
  // LJ tables with a zero padding type at index nt
  {
    const int nt1 = nt + 1;
    std::vector<float2> lj((size_t)nt1 * nt1, make_float2(0.f, 0.f)), l14 = lj;
    for (int i = 0; i < nt; ++i)
      for (int j = 0; j < nt; ++j) {
        lj[(size_t)i * nt1 + j] = make_float2((float)t.eps4[(size_t)i * nt + j], (float)t.sig2[(size_t)i * nt + j]);
        l14[(size_t)i * nt1 + j] =
            make_float2((float)t.eps4_14[(size_t)i * nt + j], (float)t.sig2_14[(size_t)i * nt + j]);
      }
    if ((size_t)nt1 * nt1 * sizeof(float2) > 200 * 1024) return fail(FZ_ERR_ARG, "too many LJ types");
    if ((r = e->upload(&e->ljtab, lj)) || (r = e->upload(&e->lj14, l14))) return r;
  }
  // ---- bonded arrays
  {
    std::vector<int2> b, u, x, q14;
    std::vector<int4> an, dh, im;
    std::vector<float2> bp, ap, up, ip;
    std::vector<float4> dp;
    for (size_t k = 0; k < t.bond_k.size(); ++k) {
      b.push_back(make_int2(t.bond[2 * k], t.bond[2 * k + 1]));
      bp.push_back(make_float2((float)t.bond_k[k], (float)t.bond_r0[k]));
    }
    for (size_t k = 0; k < t.angle_k.size(); ++k) {
      an.push_back(make_int4(t.angle[3 * k], t.angle[3 * k + 1], t.angle[3 * k + 2], 0));
      ap.push_back(make_float2((float)t.angle_k[k], (float)t.angle_t0[k]));
    }
    for (size_t k = 0; k < t.ub_k.size(); ++k) {
      u.push_back(make_int2(t.ub[2 * k], t.ub[2 * k + 1]));
      up.push_back(make_float2((float)t.ub_k[k], (float)t.ub_r0[k]));
    }
    for (size_t k = 0; k < t.dihe_k.size(); ++k) {
      dh.push_back(make_int4(t.dihe[4 * k], t.dihe[4 * k + 1], t.dihe[4 * k + 2], t.dihe[4 * k + 3]));
      dp.push_back(make_float4((float)t.dihe_k[k], (float)t.dihe_n[k], (float)std::cos(t.dihe_d[k]),
                               (float)std::sin(t.dihe_d[k])));
    }
    for (size_t k = 0; k < t.impr_k.size(); ++k) {
      im.push_back(make_int4(t.impr[4 * k], t.impr[4 * k + 1], t.impr[4 * k + 2], t.impr[4 * k + 3]));
      ip.push_back(make_float2((float)t.impr_k[k], (float)t.impr_p0[k]));
    }
    for (size_t k = 0; k < t.excl_pairs.size() / 2; ++k) x.push_back(make_int2(t.excl_pairs[2 * k], t.excl_pairs[2 * k + 1]));
    for (size_t k = 0; k < t.p14_pairs.size() / 2; ++k) q14.push_back(make_int2(t.p14_pairs[2 * k], t.p14_pairs[2 * k + 1]));
    e->nbond = (int)b.size();
    e->nangle = (int)an.size();
    e->nub = (int)u.size();
    e->ndihe = (int)dh.size();
    e->nimpr = (int)im.size();
    e->nexcl = (int)x.size();
    e->n14 = (int)q14.size();
    if ((r = e->upload(&e->bond, b)) || (r = e->upload(&e->bond_prm, bp)) || (r = e->upload(&e->angle, an)) ||
        (r = e->upload(&e->angle_prm, ap)) || (r = e->upload(&e->ub, u)) || (r = e->upload(&e->ub_prm, up)) ||
        (r = e->upload(&e->dihe, dh)) || (r = e->upload(&e->dihe_prm, dp)) || (r = e->upload(&e->impr, im)) ||
        (r = e->upload(&e->impr_prm, ip)) || (r = e->upload(&e->excl, x)) || (r = e->upload(&e->p14, q14)))
      return r;
  }
  // ---- integration units: free atoms first, then clusters (by size)
  {
    std::vector<int> in_cl(n, 0);
    for (const auto& cl : t.clusters)
      for (int k = 0; k < cl.na; ++k) in_cl[cl.atom[k]] = 1;
    std::vector<int4> ua;
    std::vector<int> um;
    std::vector<float4> ud;
    for (int i = 0; i < n; ++i)
      if (!in_cl[i]) {
        ua.push_back(make_int4(i, -1, -1, -1));
        um.push_back(1);
        ud.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
      }
    for (int na = 2; na <= 4; ++na)
      for (const auto& cl : t.clusters) {
        if (cl.na != na) continue;
        ua.push_back(make_int4(cl.atom[0], cl.atom[1], cl.atom[2], cl.atom[3]));
        int meta = cl.na | (cl.nc << 4);
        for (int k = 0; k < cl.nc; ++k) meta |= (cl.ca[k] << (8 + 4 * k)) | (cl.cb[k] << (10 + 4 * k));
        um.push_back(meta);
        ud.push_back(make_float4((float)cl.d[0], (float)cl.d[1], (float)cl.d[2], 0.f));
      }
    e->nunits = (int)ua.size();
    if ((r = e->upload(&e->unit_atoms, ua)) || (r = e->upload(&e->unit_meta, um)) || (r = e->upload(&e->unit_d, ud)))
      return r;
  }
  // ---- PME
  {
    const int Kx = e->K[0], Ky = e->K[1], Kz = e->K[2];
    const int nbr = e->nbk[0] * e->nbk[1] * e->nbk[2];
    if ((r = e->alloc(&e->brick_of, n)) || (r = e->alloc(&e->brick_count, nbr)) ||
        (r = e->alloc(&e->brick_cursor, nbr)) || (r = e->alloc(&e->brick_start, nbr + 1)) ||
        (r = e->alloc(&e->brick_atoms, n)) || (r = e->alloc(&e->grid, (size_t)Kx * Ky * Kz)) ||
        (r = e->alloc(&e->qgrid, (size_t)Kx * Ky * Kz)) ||
        (r = e->alloc(&e->cgrid, (size_t)Kz * Ky * (Kx / 2 + 1))))
      return r;
    const double b2 = c.kappa * c.kappa;
    for (int d = 0; d < 3; ++d) {
      const int Kd = e->K[d];
      std::vector<float2> tw(Kd);
      std::vector<float> g(Kd), ff(Kd);
      for (int m = 0; m < Kd; ++m) {
        const double ang = -2.0 * M_PI * m / Kd;
        tw[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        const double f = (m <= Kd / 2 ? m : m - Kd) / c.box[d];
        ff[m] = (float)(f * f);
        g[m] = (float)(bmod2(m, Kd) * std::exp(-M_PI * M_PI * f * f / b2));
      }
      if ((r = e->upload(&e->tw[d], tw)) || (r = e->upload(&e->gfac[d], g)) || (r = e->upload(&e->f2[d], ff))) return r;
    }
    e->gscale = (float)(kCC / (M_PI * V));
  }
  // first neighbour build
  const int one = 1;
  FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
  fzk::launch_rebuild(e->rebuild_args(), e->st);
  int cnt[fzk::CNT_COUNT];
  FZ_CUDA(cudaMemcpyAsync(cnt, e->counters, sizeof(cnt), cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  FZ_CUDA(cudaGetLastError());
  // grow the per-block lists if the measured neighbourhood did not fit (status bit)
  int st_h = 0;
  FZ_CUDA(cudaMemcpy(&st_h, e->status, sizeof(int), cudaMemcpyDeviceToHost));
  for (int tries = 0; (st_h & (fzk::ST_TILE_OVERFLOW | fzk::ST_MASK_OVERFLOW)) && tries < 4; ++tries) {
    FZ_CUDA(cudaStreamSynchronize(e->st));
    e->release(e->outer);
    e->release(e->inner);
    e->release(e->inner_m);
    e->release(e->masks);
    e->ocap *= 2;
    e->mask_cap = nblk * (e->ocap / 32);
    e->release(e->items);
    if ((r = e->alloc(&e->items, (size_t)nblk * (e->ocap / 32 + 1))) ||
        (r = e->alloc(&e->outer, (size_t)nblk * e->ocap)) || (r = e->alloc(&e->inner, (size_t)nblk * e->ocap)) ||
        (r = e->alloc(&e->inner_m, (size_t)nblk * (e->ocap / 32))) || (r = e->alloc(&e->masks, (size_t)e->mask_cap * 32)))
      return r;
    const int zero = 0;
    FZ_CUDA(cudaMemcpyAsync(e->status, &zero, sizeof(int), cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
    fzk::launch_rebuild(e->rebuild_args(), e->st);
    FZ_CUDA(cudaMemcpyAsync(&st_h, e->status, sizeof(int), cudaMemcpyDeviceToHost, e->st));
    FZ_CUDA(cudaStreamSynchronize(e->st));
  }
  // tiles per pair-kernel work item: enough items to keep ~24 warps per SM busy
  {
    int cnt2[fzk::CNT_COUNT];
    FZ_CUDA(cudaMemcpyAsync(cnt2, e->counters, sizeof(cnt2), cudaMemcpyDeviceToHost, e->st));
    FZ_CUDA(cudaStreamSynchronize(e->st));
    const int want = std::max(1, std::min(16, cnt2[fzk::CNT_TILES] / (dev_sms * 24)));
    if (want != e->chunk) {
      e->chunk = want;
      FZ_CUDA(cudaMemcpyAsync(e->flag_prune, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
      fzk::launch_rebuild(e->rebuild_args(), e->st);
    }
  }
  FZ_CUDA(cudaStreamSynchronize(e->st));
  return e->check();
}

}  // namespace fz

using namespace fz;

// ====================================================================== C ABI (device)
static fz_status need_engine(fz_system* s) {
  if (!s) return fail(FZ_ERR_ARG, "null system");
  if (!s->eng) return fail(FZ_ERR_STATE, "fz_upload has not been called");
  cudaSetDevice(s->eng->dev);
  return FZ_OK;
}

extern "C" fz_status fz_upload(fz_system* s, int device, void* stream) {
  if (!s) return fail(FZ_ERR_ARG, "null system");
  if (s->eng) {
    destroy_engine(s->eng);
    s->eng = nullptr;
  }
  const fz_status r = build_engine(s, device, stream);
  if (r != FZ_OK) {
    destroy_engine(s->eng);
    s->eng = nullptr;
  }
  return r;
}

extern "C" fz_status fz_compute_forces_terms(fz_system* s, int terms, int energies) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
  if (energies) FZ_CUDA(cudaMemsetAsync(e->energy, 0, fzk::EN_COUNT * sizeof(long long), e->st));
  e->forces(energies != 0, terms & FZ_TERM_ALL);
  // a partial evaluation is not the state's force: the next step recomputes
  e->forces_valid = (terms & FZ_TERM_ALL) == FZ_TERM_ALL;
  return e->check();
}

extern "C" fz_status fz_compute_forces(fz_system* s, int energies) {
  return fz_compute_forces_terms(s, FZ_TERM_ALL, energies);
}

extern "C" fz_status fz_step(fz_system* s, int nsteps) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (nsteps < 0) return fail(FZ_ERR_ARG, "nsteps < 0");
  Engine* e = s->eng;
  if (!e->forces_valid) {
    FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
    e->forces(false);
    e->forces_valid = true;
  }
  const fzk::IntegrateArgs ia = e->int_args();
  for (int k = 0; k < nsteps; ++k) {
    if (e->use_graph && !e->timing) {
      if ((r = e->graph_step())) return r;
    } else {
      e->mark(0);
      fzk::launch_kick_drift(ia, e->st);
      e->forces(false);
      fzk::launch_kick_rattle(ia, false, true, e->st);
      e->mark(6);
      if (e->timing) e->collect_step();
      e->launches += 2;
    }
    e->step++;
    if (e->temp_reset_every > 0 && e->step % e->temp_reset_every == 0) {
      fzk::launch_reassign(ia, e->temperature, e->seed, (uint32_t)(e->step / e->temp_reset_every), e->inv_mtot,
                           e->psum, e->st);
      e->launches += 4;
    }
  }
  return e->check();
}

extern "C" fz_status fz_reassign_velocities(fz_system* s, double T, uint64_t seed, uint32_t counter) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  fzk::launch_reassign(e->int_args(), T, seed, counter, e->inv_mtot, e->psum, e->st);
  return e->check();
}

extern "C" fz_status fz_eval_props(fz_system* s, fz_energies* out) {
  fz_status r;
  if (!out) return fail(FZ_ERR_ARG, "null output");
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
  FZ_CUDA(cudaMemsetAsync(e->energy, 0, fzk::EN_COUNT * sizeof(long long), e->st));
  e->forces(true);
  e->forces_valid = true;
  fzk::launch_kinetic(e->int_args(), e->st);
  long long en[fzk::EN_COUNT];
  FZ_CUDA(cudaMemcpyAsync(en, e->energy, sizeof(en), cudaMemcpyDeviceToHost, e->st));
  if ((r = e->check())) return r;
  const double s_ = 1.0 / fzk::kFixE;
  std::memset(out, 0, sizeof(*out));
  out->bond = en[fzk::EN_BOND] * s_;
  out->angle = en[fzk::EN_ANGLE] * s_;
  out->ureyb = en[fzk::EN_UREYB] * s_;
  out->dihed = en[fzk::EN_DIHED] * s_;
  out->impr = en[fzk::EN_IMPR] * s_;
  out->vdw = en[fzk::EN_VDW] * s_;
  out->elec = en[fzk::EN_ELEC] * s_;
  out->pme = en[fzk::EN_PME] * s_;
  out->ewexcl = en[fzk::EN_EWEXCL] * s_;
  out->ewself = e->self_energy;
  out->potential = out->bond + out->angle + out->ureyb + out->dihed + out->impr + out->vdw + out->elec + out->pme +
                   out->ewexcl + out->ewself;
  out->kinetic = en[fzk::EN_KIN] * s_;
  const double dof = 3.0 * e->n - 6.0 - e->ncons;  // src/evalprops.cu:225
  out->temperature = dof > 0 ? 2.0 * out->kinetic / (kRC * dof) : 0.0;
  out->step = e->step;
  return FZ_OK;
}

static fz_status get_f4(fz_system* s, const float4* src, double* out) {
  Engine* e = s->eng;
  fz_status r;
  if ((r = e->staging(sizeof(float4) * e->n))) return r;
  FZ_CUDA(cudaMemcpyAsync(e->pinned, src, sizeof(float4) * e->n, cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  const float4* h = (const float4*)e->pinned;
  for (int i = 0; i < e->n; ++i) {
    out[3 * i] = h[i].x;
    out[3 * i + 1] = h[i].y;
    out[3 * i + 2] = h[i].z;
  }
  return FZ_OK;
}

static fz_status set_f4(fz_system* s, float4* dst, const double* in, bool keep_w) {
  Engine* e = s->eng;
  fz_status r;
  if ((r = e->staging(sizeof(float4) * e->n))) return r;
  FZ_CUDA(cudaMemcpyAsync(e->pinned, dst, sizeof(float4) * e->n, cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  float4* h = (float4*)e->pinned;
  for (int i = 0; i < e->n; ++i) {
    const float w = h[i].w;
    h[i] = make_float4((float)in[3 * i], (float)in[3 * i + 1], (float)in[3 * i + 2], keep_w ? w : 0.f);
  }
  FZ_CUDA(cudaMemcpyAsync(dst, e->pinned, sizeof(float4) * e->n, cudaMemcpyHostToDevice, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  return FZ_OK;
}

extern "C" fz_status fz_get_positions(fz_system* s, double* out) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out) return fail(FZ_ERR_ARG, "null output");
  return get_f4(s, s->eng->pos4, out);
}

extern "C" fz_status fz_set_positions(fz_system* s, const double* in) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!in) return fail(FZ_ERR_ARG, "null input");
  if ((r = set_f4(s, s->eng->pos4, in, true))) return r;
  const int one = 1;
  FZ_CUDA(cudaMemcpyAsync(s->eng->flag, &one, sizeof(int), cudaMemcpyHostToDevice, s->eng->st));
  s->eng->forces_valid = false;
  return FZ_OK;
}

extern "C" fz_status fz_get_velocities(fz_system* s, double* out) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out) return fail(FZ_ERR_ARG, "null output");
  return get_f4(s, s->eng->vel4, out);
}

extern "C" fz_status fz_set_velocities(fz_system* s, const double* in) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!in) return fail(FZ_ERR_ARG, "null input");
  return set_f4(s, s->eng->vel4, in, true);
}

extern "C" fz_status fz_get_forces_fixed(fz_system* s, long long* out) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out) return fail(FZ_ERR_ARG, "null output");
  Engine* e = s->eng;
  FZ_CUDA(cudaMemcpyAsync(out, e->facc, 3 * sizeof(long long) * e->n, cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  return FZ_OK;
}

extern "C" fz_status fz_get_forces(fz_system* s, double* out) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out) return fail(FZ_ERR_ARG, "null output");
  Engine* e = s->eng;
  std::vector<long long> f(3 * (size_t)e->n);
  if ((r = fz_get_forces_fixed(s, f.data()))) return r;
  for (int i = 0; i < e->n; ++i)
    for (int c = 0; c < 3; ++c) out[3 * i + c] = (double)f[(size_t)c * e->n + i] / fzk::kFixFd;
  return FZ_OK;
}

extern "C" fz_status fz_set_state_f32(fz_system* s, const float* pos, const float* vel) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  // xyz per atom into the float4 arrays (q and 1/m kept): strided device copies
  if (pos) {
    FZ_CUDA(cudaMemcpy2DAsync(e->pos4, sizeof(float4), pos, 3 * sizeof(float), 3 * sizeof(float), e->n,
                              cudaMemcpyHostToDevice, e->st));
    const int one = 1;
    FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
    e->forces_valid = false;
  }
  if (vel)
    FZ_CUDA(cudaMemcpy2DAsync(e->vel4, sizeof(float4), vel, 3 * sizeof(float), 3 * sizeof(float), e->n,
                              cudaMemcpyHostToDevice, e->st));
  return FZ_OK;
}

extern "C" fz_status fz_get_state_f32(fz_system* s, float* pos, float* vel) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  if (pos)
    FZ_CUDA(cudaMemcpy2DAsync(pos, 3 * sizeof(float), e->pos4, sizeof(float4), 3 * sizeof(float), e->n,
                              cudaMemcpyDeviceToHost, e->st));
  if (vel)
    FZ_CUDA(cudaMemcpy2DAsync(vel, 3 * sizeof(float), e->vel4, sizeof(float4), 3 * sizeof(float), e->n,
                              cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  return FZ_OK;
}

extern "C" fz_status fz_get_counters(fz_system* s, long long* out4) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  int cnt[fzk::CNT_COUNT];
  FZ_CUDA(cudaMemcpyAsync(cnt, e->counters, sizeof(cnt), cudaMemcpyDeviceToHost, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  out4[0] = e->launches;
  out4[1] = cnt[fzk::CNT_REBUILDS];
  out4[2] = cnt[fzk::CNT_TILES];
  out4[3] = cnt[fzk::CNT_PRUNES];
  return FZ_OK;
}

extern "C" fz_status fz_set_stage_timing(fz_system* s, int enable) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  if (enable && !e->ev[0])
    for (auto& x : e->ev) FZ_CUDA(cudaEventCreate(&x));
  e->timing = enable != 0;
  for (double& x : e->stage_ms) x = 0;
  e->timed_steps = 0;
  return FZ_OK;
}

extern "C" fz_status fz_get_stage_times(fz_system* s, double* out6) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out6) return fail(FZ_ERR_ARG, "null output");
  for (int k = 0; k < 5; ++k) out6[k] = s->eng->stage_ms[k];
  out6[5] = (double)s->eng->timed_steps;
  return FZ_OK;
}

extern "C" fz_status fz_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return fail(FZ_ERR_ARG, "null output");
  *tflops = fzk::measure_fp32_peak(device);
  FZ_CUDA(cudaGetLastError());
  return *tflops > 0 ? FZ_OK : fail(FZ_ERR_CUDA, "FMA benchmark failed");
}

extern "C" fz_status fz_sync(fz_system* s) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  return s->eng->check();
}

extern "C" void* fz_stream(fz_system* s) { return (s && s->eng) ? (void*)s->eng->st : nullptr; }
