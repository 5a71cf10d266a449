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
#include "engine.h"

#include <algorithm>
#include <array>
#include <map>
#include <mutex>

namespace fz {

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

// PME brick shapes the autotuner tries: the default edge, then for each target t the
// largest divisor of K in [4, t] per dimension (cubic grids give cubic bricks)
static std::vector<std::array<int, 3>> brick_candidates(const int K[3]) {
  std::vector<std::array<int, 3>> out;
  out.push_back({brick_edge(K[0]), brick_edge(K[1]), brick_edge(K[2])});
  for (int t : {4, 6, 8, 12, 16}) {
    std::array<int, 3> b;
    for (int d = 0; d < 3; ++d) {
      int best = 0;
      for (int q = 4; q <= t; ++q)
        if (K[d] % q == 0) best = q;
      b[d] = best ? best : brick_edge(K[d]);
    }
    if (std::find(out.begin(), out.end(), b) == out.end()) out.push_back(b);
  }
  return out;
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

// ---------------------------------------------------------------- autotuner
// Picks launch shapes that leave every result bit-identical, so a timing-dependent
// choice never changes a force: pair-kernel CTAs per SM (the pair kernel's grid; each
// work item's forces are summed and flushed alike whichever warp takes it), the PME
// brick edge (the block shape of the charge spread and of the gather: grid charges
// are integer sums) and the gather kernel (per brick or per atom, the same sums in
// the same order).  The tiles per work item are not tuned: an item's i force is
// summed in FP32 before its fixed-point flush, so that size is a fixed rule of the
// tile count.  Each candidate is timed on the device with CUDA events (the best of 3
// trials of 3 launches, after 2 warm-up launches), one knob at a time from the
// defaults; a candidate replaces the current choice only when at least 1 % faster.
// Choices are cached per shape (grid, atom count in eighth-octave buckets, pair tiles
// in quarter-octave buckets), so batch members and served jobs of one shape tune once
// per process.  FZ_AUTOTUNE=0 keeps the defaults; FZ_NB_CTAS_PER_SM, FZ_PME_BRICK and
// FZ_PME_GATHER fix their knob.
namespace {
struct TunedShape {
  int per_sm, B[3], gather;
};
std::mutex g_tune_mu;
std::map<std::array<long long, 5>, TunedShape> g_tune_cache;

template <class F>
float time_launches(cudaStream_t st, F&& launch) {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch();
  launch();
  float best = 3e38f;
  for (int t = 0; t < 3; ++t) {
    cudaEventRecord(a, st);
    for (int k = 0; k < 3; ++k) launch();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}
}  // namespace

static void set_per_sm(Engine* e, int per) {
  e->nb_per_sm = per;
  e->nb_grid = e->n_sm * per;
}

static void set_bricks(Engine* e, const std::array<int, 3>& b) {
  for (int d = 0; d < 3; ++d) {
    e->B[d] = b[d];
    e->nbk[d] = e->K[d] / b[d];
  }
}

static fz_status autotune(Engine* e) {
  if (const char* v = std::getenv("FZ_AUTOTUNE"))
    if (std::atoi(v) == 0) return FZ_OK;
  // a shape fixed by the environment is not tuned, and such runs bypass the cache
  const bool fix_per_sm = std::getenv("FZ_NB_CTAS_PER_SM") != nullptr;
  const bool fix_brick = std::getenv("FZ_PME_BRICK") != nullptr;
  const bool fix_gather = std::getenv("FZ_PME_GATHER") != nullptr;
  const bool cached = !(fix_per_sm || fix_brick || fix_gather);
  const std::array<long long, 5> key = {e->K[0], e->K[1], e->K[2], (long long)std::floor(8.0 * std::log2((double)e->n)),
                                        (long long)std::floor(4.0 * std::log2(1.0 + e->tiles))};
  if (cached) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      const TunedShape& t = it->second;
      set_per_sm(e, t.per_sm);
      set_bricks(e, {t.B[0], t.B[1], t.B[2]});
      e->gather_mode = t.gather;
      e->tuned = true;
      return FZ_OK;
    }
  }
  // pair-kernel CTAs per SM
  if (!fix_per_sm) {
    const int p0 = e->nb_per_sm;
    float best = time_launches(e->st, [&] { fzk::launch_nonbonded(e->nb_args(), false, e->st); });
    int pick = p0;
    for (int per : {4, 3, 2}) {
      if (per == p0) continue;
      set_per_sm(e, per);
      const float t = time_launches(e->st, [&] { fzk::launch_nonbonded(e->nb_args(), false, e->st); });
      if (t < 0.99f * best) {
        best = t;
        pick = per;
      }
    }
    set_per_sm(e, pick);
  }
  // PME brick edge x gather kernel
  if (!(fix_brick && fix_gather)) {
    std::vector<std::array<int, 3>> cands = brick_candidates(e->K);
    if (fix_brick) cands = {{e->B[0], e->B[1], e->B[2]}};
    // gather modes tried per brick shape (the environment's alone when it fixes one);
    // mode 3 (no brick lists) does not depend on the brick shape: tried once
    const std::vector<int> gmodes = fix_gather ? std::vector<int>{e->gather_mode} : std::vector<int>{0, 1, 2, 3};
    std::array<int, 3> bpick = cands[0];
    int gpick = gmodes[0];
    float best = 3e38f;
    for (size_t ib = 0; ib < cands.size(); ++ib)
      for (int g : gmodes) {
        if (g == 3 && ib > 0) continue;
        set_bricks(e, cands[ib]);
        e->gather_mode = g;
        const float t = time_launches(e->st, [&] { fzk::launch_pme(e->pme_args(), false, e->st); });
        if (t < 0.99f * best) {
          best = t;
          bpick = cands[ib];
          gpick = g;
        }
      }
    set_bricks(e, bpick);
    e->gather_mode = gpick;
  }
  // the timed launches added forces: the first step starts from a zeroed accumulator
  FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
  FZ_CUDA(cudaStreamSynchronize(e->st));
  FZ_CUDA(cudaGetLastError());
  e->tuned = true;
  if (cached) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = TunedShape{e->nb_per_sm, {e->B[0], e->B[1], e->B[2]}, e->gather_mode};
  }
  return e->check();
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
  FZ_CUDA(cudaStreamCreateWithFlags(&e->st_cap, cudaStreamNonBlocking));
  {
    // conditional IF nodes for the neighbour kernels inside captured steps: measured
    // ~12 us per step slower on B200 at 230,400 atoms than the flag-checking kernels
    // they replace, so they are off unless FZ_GRAPH_COND=1
    const char* v = std::getenv("FZ_GRAPH_COND");
    e->cond_graph = v && std::atoi(v) == 1;
    if (const char* c = std::getenv("FZ_GRAPH_CHUNK")) e->chunk_steps = std::max(0, std::min(1000, std::atoi(c)));
    if (const char* c = std::getenv("FZ_FUSE_CLOSE")) e->fuse_close = std::atoi(c) != 0;
  }
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
  // column cross-section: a x a with a^3 holding `col_atoms` atoms (32: one sorted
  // block is a near-cube; smaller values make narrower, taller blocks).  16: a block
  // is two near-cubes stacked in z, so each 16-atom i-group is a compact cube and
  // fewer pairs of its tiles fall outside the cutoff.  Measured (us per step, 1,000
  // steps): 230,400 atoms 421 (32) / 413-418 (16); 17,280 atoms 85.9 / 83.7; 256
  // boxes 1.655 / 1.608 ms.
  double col_atoms = 16.0;
  if (const char* v = std::getenv("FZ_COL_ATOMS")) col_atoms = std::min(64.0, std::max(8.0, std::atof(v)));
  const double a = std::cbrt(col_atoms / rho);
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
  e->ncx = ncx;
  e->ncy = ncy;
  e->col_a = a;
  e->plist = plist;
  e->cutoff = rc;
  for (int d = 0; d < 3; ++d) e->ratio[d] = c.box[d] / c.box[0];
  e->L_build = e->L_prune = c.box[0];
  e->pmass = c.pmass;
  e->pref_atm = c.pref;
  e->nslots = ((n + 32 * e->ncol + 64 + 31) / 32) * 32;
  p.nslots = e->nslots;
  if (e->nslots >= (1 << 26)) return fail(FZ_ERR_CAPACITY, "system too large: sorted slots exceed 2^26");
  for (int d = 0; d < 3; ++d) {
    e->K[d] = c.pme_grid[d];
    if (!fft_size_ok(e->K[d])) return fail(FZ_ERR_ARG, "PME grid sizes must be 2^a 3^b 5^c in [2, 1024]");
    e->B[d] = brick_edge(e->K[d]);
    // FZ_PME_BRICK=t: the largest divisor of K in [4, min(t, 16)] (the spread and gather
    // hold a (B+3)^3 region in shared memory sized for bricks of at most 16)
    if (const char* v = std::getenv("FZ_PME_BRICK"))
      for (int q = 4; q <= std::min(std::atoi(v), 16); ++q)
        if (e->K[d] % q == 0) e->B[d] = q;
    e->nbk[d] = e->K[d] / e->B[d];
    p.K[d] = e->K[d];
  }
  if (const char* v = std::getenv("FZ_PME_GATHER")) e->gather_mode = std::max(0, std::min(3, std::atoi(v)));
  // per-block list capacity: atoms within rlist of a block box (Minkowski volume of a
  // box 1.4 a wide and 1.4 h tall, h the mean height of 32 atoms in a column), with
  // room for blocks that see all their neighbours at higher index
  const double ab = 1.4 * a, hb = 1.4 * 32.0 / (rho * a * a), R = plist;
  const double vm = ab * ab * hb + 2 * R * (ab * ab + 2 * ab * hb) + M_PI * R * R * (2 * ab + hb) +
                    4.0 / 3.0 * M_PI * R * R * R;
  e->ocap = (int)std::ceil(std::max(256.0, 1.25 * rho * vm) / 32.0) * 32;
  e->mask_cap = (e->nslots / 32) * fzk::kNG * (e->ocap / 32);
  {
    // inner-list buffer: a larger delta prunes less often but leaves more pairs.
    // Measured (us per step, 1,000 steps, skin 1 A): 230,400 atoms 441 (0.3 A), 425
    // (0.5), 432 (0.6), 443 (0.8); 9,000 atoms 67.5, 65.5, 65.6, 66.2
    double want = 0.5;
    if (const char* v = std::getenv("FZ_PRUNE_DELTA")) want = std::max(0.05, std::atof(v));
    const double delta = std::min(want, plist - c.cutoff);
    e->rp2 = (float)((c.cutoff + delta) * (c.cutoff + delta));
    e->prune_half2 = (float)(0.25 * delta * delta);
    e->prune_delta = delta;
    e->prune_half2_nve = e->prune_half2;
    e->skin_half2_nve = p.skin_half2;
  }
  e->dtu = c.timestep_ps * kTU;
  e->shake_tol = c.shake_tol > 0 ? c.shake_tol : 1e-10;
  e->temp_reset_every = c.temp_reset_every;
  e->temperature = c.temperature;
  e->seed = (unsigned long long)c.seed;
  e->self_energy = t.self_energy;
  e->ncons = (int)t.cons_d.size();
  // fixed segments (consfix) and the two restraint segments (consharm), by PSF segment
  // name, case-insensitive as the reference compares them (src/prmread.cu:365-380)
  std::vector<char> fixed(n, 0);
  std::vector<int> rseg(n, -1);
  for (int i = 0; i < n; ++i) {
    const std::string& sg = t.seg_names.size() == (size_t)n ? t.seg_names[i] : std::string();
    for (int j = 0; j < c.consfix_nseg; ++j)
      if (!cicompare(sg, c.consfix_seg[j])) fixed[i] = 1;
    if (c.consharm) {
      if (!cicompare(sg, c.consharm_seg[0])) rseg[i] = 0;
      else if (!cicompare(sg, c.consharm_seg[1])) rseg[i] = 1;
    }
  }
  e->nfixed = 0;
  for (int i = 0; i < n; ++i) e->nfixed += fixed[i];
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
  // pair kernel CTAs per SM: 4 (64-register build, default: 0.614 vs 0.624 ms/step at
  // 230,400 atoms) or 3 (80-register build), env FZ_NB_CTAS_PER_SM; PME overlaps it on
  // a second stream
  {
    const char* v = std::getenv("FZ_NB_CTAS_PER_SM");
    const int per = v ? std::max(1, std::min(4, std::atoi(v))) : 4;
    e->nb_grid = dev_sms * per;
    e->nb_per_sm = per;
    e->n_sm = dev_sms;
  }
  // ---- atom arrays
  std::vector<float4> pos4(n), vel4(n);
  double mt = 0;
  for (int i = 0; i < n; ++i) {
    pos4[i] = make_float4((float)t.pos[3 * i], (float)t.pos[3 * i + 1], (float)t.pos[3 * i + 2], (float)t.q[i]);
    // a fixed atom has inverse mass 0: no kick, drift or minimiser move reaches it
    vel4[i] = make_float4(0.f, 0.f, 0.f, (t.mass[i] > 0 && !fixed[i]) ? (float)(1.0 / t.mass[i]) : 0.f);
    mt += t.mass[i];
  }
  e->inv_mtot = mt > 0 ? 1.0 / mt : 0.0;
  fz_status r;
  if ((r = e->upload(&e->pos4, pos4)) || (r = e->upload(&e->vel4, vel4)) || (r = e->alloc(&e->pos_build, n)) ||
      (r = e->alloc(&e->facc, 3 * (size_t)n)) || (r = e->alloc(&e->energy, fzk::EN_COUNT)) ||
      (r = e->alloc(&e->psum, 4)) || (r = e->upload(&e->type, t.type)))
    return r;
  if (c.consharm) {
    double m0 = 0, m1 = 0;
    for (int i = 0; i < n; ++i) {
      if (rseg[i] == 0) m0 += t.mass[i];
      if (rseg[i] == 1) m1 += t.mass[i];
    }
    if (!(m0 > 0 && m1 > 0)) return fail(FZ_ERR_ARG, "consharm: a restraint segment has no atoms");
    e->restraint = true;
    e->rs_inv_m[0] = 1.0 / m0;
    e->rs_inv_m[1] = 1.0 / m1;
    for (int d = 0; d < 3; ++d) e->rs_dist[d] = c.consharm_dist[d];
    e->rs_fc = c.consharm_fc;
    std::vector<float> ms(n);
    for (int i = 0; i < n; ++i) ms[i] = (float)t.mass[i];
    if ((r = e->upload(&e->rs_seg, rseg)) || (r = e->upload(&e->rs_mass, ms)) || (r = e->alloc(&e->rs_acc, 8)))
      return r;
  }
  // ---- sorted slots, columns, tiles
  const int nslots = e->nslots, nblk = nslots / 32, ngrp = nblk * fzk::kNG;
  if ((r = e->alloc(&e->xyzq_s, nslots)) || (r = e->alloc(&e->typ_s, nslots)) || (r = e->alloc(&e->perm, nslots)) ||
      (r = e->alloc(&e->inv_perm, n)) || (r = e->alloc(&e->col_of, n)) || (r = e->alloc(&e->col_count, e->ncol)) ||
      (r = e->alloc(&e->col_cursor, e->ncol)) || (r = e->alloc(&e->col_start, e->ncol + 1)) ||
      (r = e->alloc(&e->col_tmp, nslots)) || (r = e->alloc(&e->bb_lo, nblk)) || (r = e->alloc(&e->blk_col, nblk)) || (r = e->alloc(&e->bb_hi, nblk)) ||
      (r = e->alloc(&e->outer, (size_t)nblk * e->ocap)) || (r = e->alloc(&e->inner, (size_t)ngrp * e->ocap)) ||
      (r = e->alloc(&e->outer_n, nblk)) || (r = e->alloc(&e->inner_nt, ngrp)) ||
      (r = e->alloc(&e->inner_m, (size_t)ngrp * (e->ocap / 32))) || (r = e->alloc(&e->dmask, (size_t)nblk * 32)) ||
      (r = e->alloc(&e->masks, (size_t)e->mask_cap * fzk::kIG)) || (r = e->alloc(&e->pos_prune, n)) ||
      (r = e->alloc(&e->flag_prune, 1)) || (r = e->alloc(&e->items, (size_t)ngrp * (e->ocap / 32 + 1))) ||
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
  for (int i = 0; i < n; ++i) e->xmax = std::max(e->xmax, t.excl_off[i + 1] - t.excl_off[i]);
  if ((r = e->alloc(&e->xn, nslots)) || (r = e->alloc(&e->xs, (size_t)nslots * e->xmax)) ||
      (r = e->alloc(&e->xrange, nslots)))
    return r;
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
    // clusters whose atoms are all fixed need no constraint solve: free units
    std::vector<int> in_cl(n, 0);
    for (const auto& cl : t.clusters) {
      bool all_fixed = true;
      for (int k = 0; k < cl.na; ++k) all_fixed = all_fixed && fixed[cl.atom[k]];
      if (!all_fixed)
        for (int k = 0; k < cl.na; ++k) in_cl[cl.atom[k]] = 1;
    }
    std::vector<int4> ua;
    std::vector<int> um;
    std::vector<float4> ud;
    // grouped by class (atoms, constraints): each class is one integrator launch with
    // its loops fixed at compile time
    e->ncls = 0;
    auto open_class = [&](int na, int nc) {
      if (e->ncls > 0 && e->cls_na[e->ncls - 1] == na && e->cls_nc[e->ncls - 1] == nc) return;
      e->cls_na[e->ncls] = na;
      e->cls_nc[e->ncls] = nc;
      e->cls_begin[e->ncls] = (int)ua.size();
      e->ncls++;
    };
    for (int i = 0; i < n; ++i)
      if (!in_cl[i]) {
        open_class(1, 0);
        ua.push_back(make_int4(i, -1, -1, -1));
        um.push_back(1);
        ud.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
      }
    // SETTLE applies to (3 atoms, 3 constraints) clusters that are symmetric triangles:
    // an apex bonded to two base atoms of equal mass at equal lengths; those are stored
    // apex first with constraints (0,1), (0,2), (1,2)
    auto as_triangle = [&](const Cluster& cl, Cluster& out) {
      if (cl.na != 3 || cl.nc != 3) return false;
      for (int base = 0; base < 3; ++base) {  // constraint `base` joins the two base atoms
        const int b = cl.ca[base], c = cl.cb[base], ap = 3 - b - c;
        if (ap < 0 || ap > 2 || b == c) continue;
        double dab = -1, dac = -1;
        for (int k = 0; k < 3; ++k) {
          if ((cl.ca[k] == ap && cl.cb[k] == b) || (cl.ca[k] == b && cl.cb[k] == ap)) dab = cl.d[k];
          if ((cl.ca[k] == ap && cl.cb[k] == c) || (cl.ca[k] == c && cl.cb[k] == ap)) dac = cl.d[k];
        }
        const double mb = t.mass[cl.atom[b]], mc = t.mass[cl.atom[c]];
        if (dab <= 0 || dac <= 0 || (float)dab != (float)dac || mb != mc || mb <= 0 || t.mass[cl.atom[ap]] <= 0)
          continue;
        if (fixed[cl.atom[ap]] || fixed[cl.atom[b]] || fixed[cl.atom[c]]) return false;
        out = cl;
        out.atom[0] = cl.atom[ap];
        out.atom[1] = cl.atom[b];
        out.atom[2] = cl.atom[c];
        out.ca[0] = 0; out.cb[0] = 1; out.d[0] = dab;
        out.ca[1] = 0; out.cb[1] = 2; out.d[1] = dac;
        out.ca[2] = 1; out.cb[2] = 2; out.d[2] = cl.d[base];
        return true;
      }
      return false;
    };
    {
      int n33 = 0, ntri = 0;
      Cluster tmp;
      for (const auto& cl : t.clusters)
        if (cl.na == 3 && cl.nc == 3 && in_cl[cl.atom[0]]) {
          ++n33;
          ntri += as_triangle(cl, tmp) ? 1 : 0;
        }
      e->settle = (n33 > 0 && ntri == n33) ? 1 : 0;
      if (const char* v = std::getenv("FZ_SETTLE")) e->settle = e->settle && std::atoi(v) != 0;
    }
    for (int na = 2; na <= 4; ++na)
      for (int nc = 1; nc <= 3; ++nc)
        for (const auto& cl0 : t.clusters) {
          if (cl0.na != na || cl0.nc != nc || !in_cl[cl0.atom[0]]) continue;
          Cluster cl = cl0;
          if (e->settle && na == 3 && nc == 3) as_triangle(cl0, cl);
          open_class(na, nc);
          ua.push_back(make_int4(cl.atom[0], cl.atom[1], cl.atom[2], cl.atom[3]));
          int meta = cl.na | (cl.nc << 4);
          for (int k = 0; k < cl.nc; ++k) meta |= (cl.ca[k] << (8 + 4 * k)) | (cl.cb[k] << (10 + 4 * k));
          um.push_back(meta);
          ud.push_back(make_float4((float)cl.d[0], (float)cl.d[1], (float)cl.d[2], 0.f));
        }
    e->nunits = (int)ua.size();
    e->cls_begin[e->ncls] = e->nunits;
    if ((r = e->upload(&e->unit_atoms, ua)) || (r = e->upload(&e->unit_meta, um)) || (r = e->upload(&e->unit_d, ud)))
      return r;
  }
  // ---- PME
  {
    const int Kx = e->K[0], Ky = e->K[1], Kz = e->K[2];
    // brick lists sized for the candidate brick shape with the most bricks
    int nbr = e->nbk[0] * e->nbk[1] * e->nbk[2];
    for (const auto& b : brick_candidates(e->K)) nbr = std::max(nbr, (Kx / b[0]) * (Ky / b[1]) * (Kz / b[2]));
    if ((r = e->alloc(&e->brick_of, n)) || (r = e->alloc(&e->brick_count, nbr)) ||
        (r = e->alloc(&e->brick_cursor, nbr)) || (r = e->alloc(&e->brick_start, nbr + 1)) ||
        (r = e->alloc(&e->brick_atoms, n)) || (r = e->alloc(&e->grid, (size_t)Kx * Ky * Kz)) ||
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
    e->mask_cap = ngrp * (e->ocap / 32);
    e->release(e->items);
    if ((r = e->alloc(&e->items, (size_t)ngrp * (e->ocap / 32 + 1))) ||
        (r = e->alloc(&e->outer, (size_t)nblk * e->ocap)) || (r = e->alloc(&e->inner, (size_t)ngrp * e->ocap)) ||
        (r = e->alloc(&e->inner_m, (size_t)ngrp * (e->ocap / 32))) ||
        (r = e->alloc(&e->masks, (size_t)e->mask_cap * fzk::kIG)))
      return r;
    const int zero = 0;
    FZ_CUDA(cudaMemcpyAsync(e->status, &zero, sizeof(int), cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
    fzk::launch_rebuild(e->rebuild_args(), e->st);
    FZ_CUDA(cudaMemcpyAsync(&st_h, e->status, sizeof(int), cudaMemcpyDeviceToHost, e->st));
    FZ_CUDA(cudaStreamSynchronize(e->st));
  }
  // the outer-list build and the prune: a warp per i-block fills the GPU above ~16
  // blocks per SM; below, one CTA of 8 warps per block (the same lists, so the same
  // forces; 9,000 atoms 60.9 -> 54.9 us per step with the split build); FZ_PRUNE_SPLIT=0/1
  // forces it
  {
    e->prune_split = (nblk < 16 * e->n_sm && fzk::prune_split_fits(e->ocap)) ? 1 : 0;
    if (const char* v = std::getenv("FZ_PRUNE_SPLIT"))
      e->prune_split = (std::atoi(v) != 0 && fzk::prune_split_fits(e->ocap)) ? 1 : 0;
    e->outer_split = e->prune_split;
    if (const char* v = std::getenv("FZ_OUTER_SPLIT")) e->outer_split = std::atoi(v) != 0 ? 1 : 0;
  }
  // tiles per pair-kernel work item: ~8 items per pair-kernel warp, 3 to 6 tiles, so
  // the warps run out of work together (the last items are short).  Measured (us per
  // step, 1,000 steps): 230,400 atoms 426 (3 tiles), 423 (4), 422 (6), 424 (8); 17,280
  // atoms 88.4 (2), 86.4 (3), 86.0 (4), 86.6 (6); 9,000 atoms 65.9 (2), 62.1 (3), 65.0
  // (4), 73.9 (6).  The item size changes the order of the i-force sums, so it is a
  // fixed rule, not a shape the autotuner times.
  {
    int cnt2[fzk::CNT_COUNT];
    FZ_CUDA(cudaMemcpyAsync(cnt2, e->counters, sizeof(cnt2), cudaMemcpyDeviceToHost, e->st));
    FZ_CUDA(cudaStreamSynchronize(e->st));
    e->tiles = cnt2[fzk::CNT_TILES];
    int want = std::max(3, std::min(6, e->tiles / (e->n_sm * 4 * fzk::kWarpsPerCta * 8)));
    if (const char* v = std::getenv("FZ_CHUNK_TILES")) want = std::max(1, std::min(64, std::atoi(v)));
    if (want != e->chunk) {
      e->chunk = want;
      FZ_CUDA(cudaMemcpyAsync(e->flag_prune, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
      fzk::launch_rebuild(e->rebuild_args(), e->st);
    }
  }
  if ((r = autotune(e))) return r;
  FZ_CUDA(cudaStreamSynchronize(e->st));
  if ((r = e->check())) return r;
  // FZ_LIST_CAP=c (a test hook for the capacity path): from the next rebuild on, each
  // block's pair list keeps at most c entries (a multiple of 32, within what is
  // allocated; the lists are rebuilt at the new stride before any kernel reads them),
  // so an overflow during dynamics is reported by fz_step as FZ_ERR_CAPACITY instead
  // of being grown here
  if (const char* v = std::getenv("FZ_LIST_CAP")) {
    const int cap = std::max(32, std::min(e->ocap, (std::atoi(v) / 32) * 32));
    e->ocap = cap;
    e->mask_cap = ngrp * (cap / 32);
    e->drop_graph();
    FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaStreamSynchronize(e->st));
  }
  return FZ_OK;
}

// ---------------------------------------------------------------- barostat
constexpr double kPatm = 68558.64100846418;     // kcal/mol/A^3 -> atm (src/cell_based_kernels.cu:584)

// Moves the engine to a new box (x edge L, aspect ratios kept): parameters passed by
// value to the kernels, the column search reach, and the PME influence tables.
fz_status set_box(Engine* e, double L) {
  fzk::SysParams& p = e->p;
  for (int d = 0; d < 3; ++d) e->box_d[d] = L * e->ratio[d];
  const double lmin = std::min(e->box_d[0], std::min(e->box_d[1], e->box_d[2]));
  if (e->cutoff >= 0.5 * lmin) return fail(FZ_ERR_STATE, "barostat: box shrank below twice the cutoff");
  p.box = make_float3((float)e->box_d[0], (float)e->box_d[1], (float)e->box_d[2]);
  p.inv_box = make_float3((float)(1.0 / e->box_d[0]), (float)(1.0 / e->box_d[1]), (float)(1.0 / e->box_d[2]));
  const double V = e->box_d[0] * e->box_d[1] * e->box_d[2];
  e->gscale = (float)(kCC / (M_PI * V));
  e->dcx = std::min(e->ncx, (int)std::ceil(e->plist / (e->box_d[0] / e->ncx)));
  e->dcy = std::min(e->ncy, (int)std::ceil(e->plist / (e->box_d[1] / e->ncy)));
  const double colw = std::max(e->box_d[0] / e->ncx, e->box_d[1] / e->ncy);
  e->all_images = (0.5 * lmin < e->plist + 3.0 * std::max(colw, e->col_a)) ? 1 : 0;
  const int ktot = e->K[0] + e->K[1] + e->K[2];
  if (!e->pme_tab_host) FZ_CUDA(cudaMallocHost(&e->pme_tab_host, sizeof(float) * 2 * ktot));
  // the previous step's table copies have completed: barostat steps synchronise each step
  const double b2 = (double)p.beta * (double)p.beta;
  float* h = e->pme_tab_host;
  for (int d = 0; d < 3; ++d) {
    const int Kd = e->K[d];
    float* g = h;
    float* ff = h + Kd;
    for (int m = 0; m < Kd; ++m) {
      const double f = (m <= Kd / 2 ? m : m - Kd) / e->box_d[d];
      ff[m] = (float)(f * f);
      g[m] = (float)(bmod2(m, Kd) * std::exp(-M_PI * M_PI * f * f / b2));
    }
    FZ_CUDA(cudaMemcpyAsync(e->gfac[d], g, sizeof(float) * Kd, cudaMemcpyHostToDevice, e->st));
    FZ_CUDA(cudaMemcpyAsync(e->f2[d], ff, sizeof(float) * Kd, cudaMemcpyHostToDevice, e->st));
    h += 2 * Kd;
  }
  return FZ_OK;
}

// host copy of the energy slots and the cumulative list counters (synchronises)
static fz_status read_slots(Engine* e, long long* en, int* cnt) {
  FZ_CUDA(cudaMemcpyAsync(en, e->energy, sizeof(long long) * fzk::EN_COUNT, cudaMemcpyDeviceToHost, e->st));
  if (cnt) FZ_CUDA(cudaMemcpyAsync(cnt, e->counters, sizeof(int) * fzk::CNT_COUNT, cudaMemcpyDeviceToHost, e->st));
  return e->check();
}

static double volume(const Engine* e) { return e->box_d[0] * e->box_d[1] * e->box_d[2]; }

// piston acceleration for the instantaneous pressure P (kcal/mol/A^3)
static double piston_accel(const Engine* e, double P) {
  const double L = e->box_d[0];
  return (P - e->pref_atm * kPU) / (3.0 * e->pmass * L * L) - 2.0 * e->Ldot * e->Ldot / L;
}

// Forces + energies + virial of the current state and its instantaneous pressure
// (kcal/mol/A^3).  Atomic form (fz_eval_props): all kinetic energy, the force virial and
// the instantaneous constraint virial.  Group form (barostat): the kinetic energy of the
// unit centres and the virial of the unit centres.
static fz_status state_pressure(Engine* e, long long* en, double* P, bool group) {
  FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
  FZ_CUDA(cudaMemsetAsync(e->energy, 0, fzk::EN_COUNT * sizeof(long long), e->st));
  e->forces(true);
  e->forces_valid = true;
  const fzk::IntegrateArgs ia = e->int_args();
  fzk::launch_kinetic(ia, e->st);
  if (group)
    fzk::launch_unit_virial(ia, e->st);
  else if (e->ncons)
    fzk::launch_constraint_virial(ia, e->st);
  fz_status r;
  if ((r = read_slots(e, en, nullptr))) return r;
  const double s = 1.0 / fzk::kFixE;
  const double W = (en[fzk::EN_VIR_X] + en[fzk::EN_VIR_Y] + en[fzk::EN_VIR_Z]) * s;
  const double K = (group ? en[fzk::EN_KIN_HALF] : en[fzk::EN_KIN]) * s;
  *P = (2.0 * K + W) / (3.0 * volume(e));
  return FZ_OK;
}

// One barostat step: piston half kick, box drift with rigid scaling of every
// integration unit's mass centre, kick/drift/SHAKE, forces at the new box, pressure of
// the unit centres from the half-step velocities (the reference's ScanVirial placement,
// src/dynamics.cu:773-776), piston half kick, kick/RATTLE.  Peculiar centre-of-mass
// velocities feel the friction exp(-L'/L dt/2) in each half kick (Andersen, J. Chem.
// Phys. 72, 2384 (1980), with the units as scaling groups; constraint forces act
// inside a unit and do not enter the group virial).
static fz_status npt_step(Engine* e) {
  const double dt = e->dtu;
  const double L = e->box_d[0];
  e->Ldot += 0.5 * dt * e->Lacc;
  const double Ln = L + dt * e->Ldot;
  if (!(Ln > 0.0) || !std::isfinite(Ln)) return fail(FZ_ERR_STATE, "barostat: box length diverged");
  fz_status r;
  if ((r = set_box(e, Ln))) return r;
  // list validity: periodic image shifts move with the box, by up to sqrt(3) dL
  const double rmax = std::max(e->ratio[0], std::max(e->ratio[1], e->ratio[2]));
  const double mb = 0.05 * (e->plist - e->cutoff), mp = 0.1 * e->prune_delta;
  const int one = 1;
  if (std::sqrt(3.0) * std::fabs(Ln - e->L_build) * rmax > 2.0 * mb)
    FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
  else if (std::sqrt(3.0) * std::fabs(Ln - e->L_prune) * rmax > 2.0 * mp)
    FZ_CUDA(cudaMemcpyAsync(e->flag_prune, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
  FZ_CUDA(cudaMemsetAsync(e->energy, 0, fzk::EN_COUNT * sizeof(long long), e->st));
  fzk::IntegrateArgs ia = e->int_args();
  ia.lam = Ln / L;
  ia.vfric = std::exp(-0.5 * dt * e->Ldot / L);
  fzk::launch_kick_drift_npt(ia, e->st);
  e->forces(true);
  fzk::launch_unit_virial(ia, e->st);
  long long en[fzk::EN_COUNT];
  int cnt[fzk::CNT_COUNT];
  if ((r = read_slots(e, en, cnt))) return r;
  if (cnt[fzk::CNT_REBUILDS] != e->seen_rebuilds) {
    e->seen_rebuilds = cnt[fzk::CNT_REBUILDS];
    e->L_build = e->L_prune = Ln;
  }
  if (cnt[fzk::CNT_PRUNES] != e->seen_prunes) {
    e->seen_prunes = cnt[fzk::CNT_PRUNES];
    e->L_prune = Ln;
  }
  const double s = 1.0 / fzk::kFixE;
  const double W = (en[fzk::EN_VIR_X] + en[fzk::EN_VIR_Y] + en[fzk::EN_VIR_Z]) * s;
  const double P = (2.0 * en[fzk::EN_KIN_HALF] * s + W) / (3.0 * volume(e));
  e->last_pressure = P * kPatm;
  e->Lacc = piston_accel(e, P);
  e->Ldot += 0.5 * dt * e->Lacc;
  ia = e->int_args();
  ia.vfric = std::exp(-0.5 * dt * e->Ldot / Ln);
  fzk::launch_kick_rattle(ia, false, true, e->st);
  e->launches += 3 * e->ncls;  // kick/drift, unit virial, kick/RATTLE (forces() counts its own)
  return FZ_OK;
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
  e->forces(energies != 0, terms & (FZ_TERM_ALL | FZ_TERM_BONDED_PARTS));
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
    // a whole chunk in one graph launch when no velocity reassignment falls inside it
    if (!e->npt && e->use_graph && !e->timing && e->chunk_steps > 1 && nsteps - k >= e->chunk_steps &&
        (e->temp_reset_every <= 0 ||
         e->temp_reset_every - e->step % e->temp_reset_every >= e->chunk_steps)) {
      if ((r = e->graph_chunk())) return r;
      e->step += e->chunk_steps;
      k += e->chunk_steps - 1;
      if (e->temp_reset_every > 0 && e->step % e->temp_reset_every == 0) {
        fzk::launch_reassign(ia, e->temperature, e->seed, (uint32_t)(e->step / e->temp_reset_every), e->inv_mtot,
                             e->psum, e->st);
        e->launches += 3 + e->ncls;
      }
      continue;
    }
    if (e->npt) {
      if ((r = npt_step(e))) return r;
    } else if (e->use_graph && !e->timing) {
      if ((r = e->graph_step())) return r;
    } else {
      e->mark(0);
      fzk::launch_kick_drift(ia, e->st);
      e->forces(false);
      fzk::launch_kick_rattle(ia, false, true, e->st);
      e->mark(6);
      if (e->timing) e->collect_step();
      e->launches += 2 * e->ncls;
    }
    e->step++;
    if (e->temp_reset_every > 0 && e->step % e->temp_reset_every == 0) {
      fzk::launch_reassign(e->npt ? e->int_args() : ia, e->temperature, e->seed, (uint32_t)(e->step / e->temp_reset_every), e->inv_mtot,
                           e->psum, e->st);
      e->launches += 3 + e->ncls;
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
  long long en[fzk::EN_COUNT];
  double P = 0.0;
  if ((r = state_pressure(e, en, &P, false))) return r;
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
  // src/evalprops.cu:225 (with consfix: the atoms outside fixed segments, :223)
  const double dof = 3.0 * (e->n - e->nfixed) - 6.0 - e->ncons;
  out->temperature = dof > 0 ? 2.0 * out->kinetic / (kRC * dof) : 0.0;
  out->virial[0] = en[fzk::EN_VIR_X] * s_;
  out->virial[1] = en[fzk::EN_VIR_Y] * s_;
  out->virial[2] = en[fzk::EN_VIR_Z] * s_;
  out->pressure_atm = P * kPatm;
  out->step = e->step;
  for (int d = 0; d < 3; ++d) out->box[d] = e->box_d[d];
  out->volume = volume(e);
  out->conserved = out->potential + out->kinetic;
  if (e->npt) {
    const double rho = e->ratio[1] * e->ratio[2], L = e->box_d[0];
    const double vdot = 3.0 * L * L * e->Ldot;
    out->conserved += e->pref_atm * kPU * out->volume + 0.5 * e->pmass * rho * vdot * vdot;
  }
  return FZ_OK;
}

// MinimizeStep loop of the reference's main (src/dynamics.cu:491-620,
// src/fenzi.cu:397-418): conjugate-gradient moves until the energy rises, then
// steepest descent until it rises again; a move that raises the energy is undone and
// retried with the next method; every 100 steps the step factor is multiplied by
// 100 x its rate (conjgradrate / steepdesrate).
extern "C" fz_status fz_minimize(fz_system* s, int max_steps, int* steps_done, double* energy_out) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (max_steps < 0) return fail(FZ_ERR_ARG, "fz_minimize: max_steps < 0");
  Engine* e = s->eng;
  const fz_config& c = s->cfg;
  if (!e->min_pos) {
    if ((r = e->alloc(&e->min_prev_f, e->n)) || (r = e->alloc(&e->min_dir, e->n)) || (r = e->alloc(&e->min_pos, e->n)))
      return r;
  } else {
    FZ_CUDA(cudaMemsetAsync(e->min_prev_f, 0, sizeof(float4) * e->n, e->st));
    FZ_CUDA(cudaMemsetAsync(e->min_dir, 0, sizeof(float4) * e->n, e->st));
  }
  e->drop_graph();
  auto energy = [&](double* out) -> fz_status {
    FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
    FZ_CUDA(cudaMemsetAsync(e->energy, 0, fzk::EN_COUNT * sizeof(long long), e->st));
    e->forces(true);
    e->forces_valid = true;
    long long en[fzk::EN_COUNT];
    fz_status rr = read_slots(e, en, nullptr);
    if (rr) return rr;
    double u = e->self_energy;
    for (int k = fzk::EN_BOND; k <= fzk::EN_EWEXCL; ++k) u += en[k] / fzk::kFixE;
    *out = u;
    return FZ_OK;
  };
  int method = 1;
  double fac[3] = {0.0, c.conjgradfac, c.steepdesfac};
  const double rate[3] = {0.0, c.conjgradrate, c.steepdesrate};
  double prev = 0.0, cur = 0.0;
  if ((r = energy(&cur))) return r;
  // the reference's MinimizeStep keeps its previous energy in a static that starts at 0
  // and never undoes a move while it is 0, so the first move is always kept; an undone
  // move is not counted (stepCount - 1, src/dynamics.cu:598-618)
  bool first = true;
  int step = 0;
  for (; step < max_steps && method != 0; ++step) {
    FZ_CUDA(cudaMemcpyAsync(e->min_pos, e->pos4, sizeof(float4) * e->n, cudaMemcpyDeviceToDevice, e->st));
    fzk::IntegrateArgs ia = e->int_args();
    ia.min_prev_f = e->min_prev_f;
    ia.min_dir = e->min_dir;
    ia.min_method = method;
    ia.min_fac = (float)fac[method];
    fzk::launch_min_step(ia, e->st);
    prev = cur;
    if ((r = energy(&cur))) return r;
    if (cur > prev && !first) {  // undo the move, switch method
      FZ_CUDA(cudaMemcpyAsync(e->pos4, e->min_pos, sizeof(float4) * e->n, cudaMemcpyDeviceToDevice, e->st));
      const int one = 1;
      FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
      if ((r = energy(&cur))) return r;
      method = method == 1 ? 2 : 0;
      --step;
    }
    first = false;
    if (step > 0 && step % 100 == 0 && method != 0) fac[method] *= rate[method] * 100.0;
  }
  FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
  e->forces(false);
  e->forces_valid = true;
  if ((r = e->check())) return r;
  if (steps_done) *steps_done = step;
  if (energy_out) *energy_out = cur;
  return FZ_OK;
}

extern "C" fz_status fz_set_barostat(fz_system* s, int enable, double pref_atm, double pmass) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  Engine* e = s->eng;
  if (enable && !(pmass > 0.0)) return fail(FZ_ERR_ARG, "fz_set_barostat: piston mass must be positive");
  e->drop_graph();
  if (!enable) {
    e->npt = false;
    e->p.skin_half2 = e->skin_half2_nve;
    e->prune_half2 = e->prune_half2_nve;
    e->Ldot = e->Lacc = 0.0;
    return FZ_OK;
  }
  e->pref_atm = pref_atm;
  e->pmass = pmass;
  // tighter displacement triggers leave room for the image shifts of a moving box
  const double skin = e->plist - e->cutoff;
  e->p.skin_half2 = (float)std::pow(0.5 * skin - 0.05 * skin, 2);
  e->prune_half2 = (float)std::pow(0.5 * e->prune_delta - 0.1 * e->prune_delta, 2);
  const int one = 1;
  FZ_CUDA(cudaMemcpyAsync(e->flag, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
  long long en[fzk::EN_COUNT];
  double P = 0.0;
  if ((r = state_pressure(e, en, &P, true))) return r;
  int cnt[fzk::CNT_COUNT];
  if ((r = read_slots(e, en, cnt))) return r;
  e->seen_rebuilds = cnt[fzk::CNT_REBUILDS];
  e->seen_prunes = cnt[fzk::CNT_PRUNES];
  e->L_build = e->L_prune = e->box_d[0];
  if (!e->npt) e->Ldot = 0.0;
  e->npt = true;
  e->last_pressure = P * kPatm;
  e->Lacc = piston_accel(e, P);
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

extern "C" fz_status fz_get_virial(fz_system* s, double* out3) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out3) return fail(FZ_ERR_ARG, "null output");
  Engine* e = s->eng;
  long long en[fzk::EN_COUNT];
  if ((r = read_slots(e, en, nullptr))) return r;
  for (int d = 0; d < 3; ++d) out3[d] = en[fzk::EN_VIR_X + d] / fzk::kFixE;
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
  out4[2] = (long long)cnt[fzk::CNT_TILES] * fzk::kIG * 32;
  out4[3] = cnt[fzk::CNT_PRUNES];
  return FZ_OK;
}

extern "C" fz_status fz_get_launch_shapes(fz_system* s, int* out7) {
  fz_status r;
  if ((r = need_engine(s))) return r;
  if (!out7) return fail(FZ_ERR_ARG, "null output");
  const Engine* e = s->eng;
  out7[0] = e->chunk;
  out7[1] = e->nb_per_sm;
  for (int d = 0; d < 3; ++d) out7[2 + d] = e->B[d];
  out7[5] = e->gather_mode;
  out7[6] = e->tuned ? 1 : 0;
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
