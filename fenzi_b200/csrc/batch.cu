// Batched ensemble and serving loop.
//
// fz_batch: many independent uploaded systems advanced together.  One MD step of every
// system is captured into a single CUDA graph in which each system's step (kick/drift/
// SHAKE, neighbour maintenance, forces with PME on its second stream, kick/RATTLE) is
// an independent branch forked from and joined to one master stream, so the GPU runs
// the small systems' kernels concurrently; each step is one graph launch.  Systems may
// join and leave between calls (the graph is re-captured on the next step).  Velocity
// reassignment (NVT by reassignment every temp_reset_every steps, src/fenzi.cu:463-473)
// splits a call at the reassignment steps of its systems, with the same counter as
// fz_step, so each system's trajectory is bit-identical alone and in any mix.
//
// fz_server: a request loop on a worker thread.  Submitted jobs (a loaded system and a
// step count) wait in a FIFO queue and are admitted while the estimated device memory
// of the admitted jobs stays within the HBM budget and a slot is free; admitted jobs
// are uploaded once, start from Maxwell-Boltzmann velocities at the input's temperature
// and seed, stay resident (coordinates, velocities, neighbour lists, PME
// grids) and advance together in the batch graph, in chunks that end when a job
// finishes; a finished job's final energies and positions are kept on the host, its
// device memory is freed, and queued jobs are admitted into the running mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "engine.h"

using namespace fz;

// ====================================================================== batched ensemble
// Batched kernels: one launch per kernel of the step covers every member.  The members'
// kernel arguments live in device arrays, and a block table per grid shape maps each
// launched block to (member, block of that member's own grid, grid size).
// Device storage of the arrays lives in a grow-only arena of the batch (members join and
// leave often in serving: no allocation, free or synchronisation per membership change);
// the host images are staged in pinned memory and copied with one asynchronous copy.
struct BatchArena {
  void* dev = nullptr;
  void* host = nullptr;  // pinned
  size_t cap = 0;
  ~BatchArena() {
    if (dev) cudaFree(dev);
    if (host) cudaFreeHost(host);
  }
};

struct BatchKernels {
  std::vector<char> image;                        // host image of every array
  std::vector<std::pair<size_t, void**>> fixups;  // (offset, pointer to set) per array
  fzk::RebuildArgs* rb = nullptr;
  fzk::NonbondedArgs* nb = nullptr;
  fzk::BondedArgs* bd = nullptr;
  fzk::PmeArgs* pme = nullptr;
  fzk::BatchTables t{};
  std::vector<fzk::ClassBatch> classes;
  std::vector<fzk::PmeSizeBatch> sizes;
  size_t spread_smem = 0;
  int max_ntypes = 0;
  long long launches = 0;  // kernels one batched step launches
  // appends v to the image (256-byte aligned); *out is set once the arena is known
  template <class X> fz_status upload(const std::vector<X>& v, X** out) {
    const size_t off = (image.size() + 255) & ~(size_t)255;
    image.resize(off + std::max<size_t>(1, v.size()) * sizeof(X));
    if (!v.empty()) std::memcpy(image.data() + off, v.data(), v.size() * sizeof(X));
    fixups.push_back({off, (void**)out});
    return FZ_OK;
  }
  // places the image in the arena (growing it if needed) and queues its copy on st
  fz_status place(BatchArena& ar, cudaStream_t st) {
    if (image.size() > ar.cap) {
      FZ_CUDA(cudaStreamSynchronize(st));
      if (ar.dev) FZ_CUDA(cudaFree(ar.dev));
      if (ar.host) FZ_CUDA(cudaFreeHost(ar.host));
      ar.dev = ar.host = nullptr;
      ar.cap = 0;
      const size_t cap = image.size() + image.size() / 2 + 4096;
      FZ_CUDA(cudaMalloc(&ar.dev, cap));
      FZ_CUDA(cudaMallocHost(&ar.host, cap));
      ar.cap = cap;
    } else {
      FZ_CUDA(cudaStreamSynchronize(st));  // the previous image's copy has been read
    }
    std::memcpy(ar.host, image.data(), image.size());
    FZ_CUDA(cudaMemcpyAsync(ar.dev, ar.host, image.size(), cudaMemcpyHostToDevice, st));
    for (auto& f : fixups) *f.second = (char*)ar.dev + f.first;
    return FZ_OK;
  }
};

struct fz_batch {
  std::vector<fz_system*> systems;
  int dev = -1;
  cudaStream_t master = nullptr;
  cudaEvent_t ev_start = nullptr, ev_master = nullptr;
  std::vector<cudaEvent_t> ev_done;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // batched kernels only: a graph of `chunk` consecutive steps (one launch per chunk)
  cudaGraph_t chunk_graph = nullptr;
  cudaGraphExec_t chunk_exec = nullptr;
  int chunk = 100;
  int* pinned_status = nullptr;
  long long steps = 0;
  std::unique_ptr<BatchKernels> bk;
  BatchArena arena;
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  void drop_graph() {
    bk.reset();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (chunk_exec) cudaGraphExecDestroy(chunk_exec);
    if (chunk_graph) cudaGraphDestroy(chunk_graph);
    exec = nullptr;
    graph = nullptr;
    chunk_exec = nullptr;
    chunk_graph = nullptr;
    for (auto e : ev_done) cudaEventDestroy(e);
    ev_done.clear();
    if (pinned_status) cudaFreeHost(pinned_status);
    pinned_status = nullptr;
  }
  ~fz_batch() {
    if (master) cudaStreamSynchronize(master);
    drop_graph();
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (aux) cudaStreamDestroy(aux);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_master) cudaEventDestroy(ev_master);
    if (master) cudaStreamDestroy(master);
  }
};

static std::string last_error_text() {
  char buf[1024];
  fz_last_error(buf, sizeof buf);
  return std::string(buf);
}

extern "C" fz_status fz_batch_create(fz_batch** out) {
  if (!out) return fail(FZ_ERR_ARG, "null output");
  *out = new fz_batch();
  return FZ_OK;
}

extern "C" fz_status fz_batch_add(fz_batch* b, fz_system* s) {
  if (!b || !s) return fail(FZ_ERR_ARG, "null argument");
  if (!s->eng) return fail(FZ_ERR_STATE, "fz_batch_add: system not uploaded (fz_upload)");
  if (b->dev >= 0 && s->eng->dev != b->dev) return fail(FZ_ERR_ARG, "fz_batch_add: systems must share one device");
  if (s->eng->npt) return fail(FZ_ERR_STATE, "fz_batch_add: barostat systems synchronise every step; step them alone");
  if (std::find(b->systems.begin(), b->systems.end(), s) != b->systems.end())
    return fail(FZ_ERR_ARG, "fz_batch_add: system already in the batch");
  b->dev = s->eng->dev;
  b->systems.push_back(s);
  b->drop_graph();
  return FZ_OK;
}

extern "C" fz_status fz_batch_remove(fz_batch* b, fz_system* s) {
  if (!b || !s) return fail(FZ_ERR_ARG, "null argument");
  auto it = std::find(b->systems.begin(), b->systems.end(), s);
  if (it == b->systems.end()) return fail(FZ_ERR_ARG, "fz_batch_remove: system not in the batch");
  if (b->master) cudaStreamSynchronize(b->master);
  b->systems.erase(it);
  b->drop_graph();
  if (b->systems.empty()) b->dev = -1;
  return FZ_OK;
}

// whether every member can run in the batched kernels (otherwise each member's step is
// its own branch of the batch graph)
static bool batched_kernels_ok(const fz_batch* b) {
  const char* v = std::getenv("FZ_BATCH_KERNELS");
  if (v && std::atoi(v) == 0) return false;
  for (const fz_system* s : b->systems) {
    const Engine* e = s->eng;
    if (e->cond_graph || e->restraint || e->npt || !fzk::pme_batchable(e->pme_args())) return false;
  }
  return true;
}

static void add_blocks(std::vector<int4>& tab, int arg, int nblocks) {
  for (int k = 0; k < nblocks; ++k) tab.push_back(make_int4(arg, k, nblocks, 0));
}

static fz_status build_batch_kernels(fz_batch* b) {
  auto bk = std::make_unique<BatchKernels>();
  const int ns = (int)b->systems.size();
  std::vector<fzk::RebuildArgs> rb;
  std::vector<fzk::NonbondedArgs> nb;
  std::vector<fzk::BondedArgs> bd;
  std::vector<fzk::PmeArgs> pme;
  std::vector<std::vector<int4>> tabs(fzk::BT_COUNT);
  // unit classes keyed by (atoms, constraints, SETTLE); PME grids keyed by size
  struct ClassAcc { int na, nc, settle; std::vector<fzk::IntegrateArgs> args; std::vector<int4> tab; };
  std::vector<ClassAcc> cls;
  struct SizeAcc { int N; std::vector<int4> plane, z; };
  std::vector<SizeAcc> sizes;
  // pair-kernel CTAs: the batch's total is nb_waves full waves of the batched pair
  // kernel (kNbBatchCtasPerSm per SM), shared out in proportion to the members' atoms,
  // at least one each.  Not the members' own nb_grid: the autotuner sizes that for a
  // member running alone, where a small system often does best on 2 CTAs per SM.
  long long natoms = 0;
  for (const fz_system* s : b->systems) natoms += s->top.n;
  bool big_bricks = true;
  if (const char* v = std::getenv("FZ_BATCH_BRICK")) big_bricks = std::atoi(v) != 0;
  // several waves of pair-kernel CTAs: each CTA drains its member's work queue and a
  // finished CTA's slot takes the next CTA of the launch, so members whose rounded
  // share of CTAs is short finish with the rest (one wave ends with the member of the
  // largest work per CTA, up to 1.5x the mean)
  int nb_waves = 2;
  if (const char* v = std::getenv("FZ_BATCH_NB_WAVES")) nb_waves = std::max(1, std::min(16, std::atoi(v)));
  for (int i = 0; i < ns; ++i) {
    Engine* e = b->systems[i]->eng;
    rb.push_back(e->rebuild_args());
    nb.push_back(e->nb_args());
    bd.push_back(e->bonded_args());
    pme.push_back(e->pme_args());
    if (big_bricks) {
      // a batch has CTAs to spare: bricks as large as the spread's shared region allows
      // (largest divisor of K in [4, 16]) give each spread / gather CTA hundreds of
      // atoms instead of the ~15 a member's solo shape (>= 256 bricks) leaves it; grid
      // charges are integer sums and the gather's sums run in the same order, so the
      // results do not change
      fzk::PmeArgs& q = pme.back();
      for (int d = 0; d < 3; ++d) {
        int best = 0;
        for (int c = 4; c <= 16; ++c)
          if (q.K[d] % c == 0) best = c;
        if (best) {
          q.B[d] = best;
          q.nb[d] = q.K[d] / best;
        }
      }
    }
    const fzk::SysParams& p = rb.back().p;
    const fzk::PmeArgs& pa = pme.back();
    const int nbr = pa.nb[0] * pa.nb[1] * pa.nb[2];
    const long long kt = (long long)pa.K[0] * pa.K[1] * pa.K[2];
    add_blocks(tabs[fzk::BT_ONE], i, 1);
    add_blocks(tabs[fzk::BT_ATOMS256], i, (p.n + 255) / 256);
    add_blocks(tabs[fzk::BT_COLUMNS], i, p.ncol[0] * p.ncol[1]);
    add_blocks(tabs[fzk::BT_SLOTS256], i, (p.nslots + 255) / 256);
    add_blocks(tabs[fzk::BT_BLOCKS8], i, (p.nslots / 32 + 7) / 8);
    add_blocks(tabs[fzk::BT_NB], i,
               std::max(1, (int)std::lround((double)e->n_sm * fzk::kNbBatchCtasPerSm * nb_waves * p.n /
                                            (double)std::max(1LL, natoms))));
    add_blocks(tabs[fzk::BT_BONDED], i, fzk::bonded_blocks(bd.back()));
    add_blocks(tabs[fzk::BT_BRICKS256], i, (nbr + 255) / 256);
    add_blocks(tabs[fzk::BT_BRICKS], i, nbr);
    add_blocks(tabs[fzk::BT_GRID256], i, (int)std::min<long long>(64, (kt + 255) / 256));
    bk->spread_smem = std::max(bk->spread_smem, fzk::pme_spread_smem(pa));
    bk->max_ntypes = std::max(bk->max_ntypes, p.ntypes);
    const fzk::IntegrateArgs ia = e->int_args();
    for (int c = 0; c < ia.ncls; ++c) {
      fzk::IntegrateArgs x = ia;
      x.u_begin = ia.cls_begin[c];
      x.u_end = ia.cls_begin[c + 1];
      const int na = ia.cls_na[c], ncn = ia.cls_nc[c], st = (na == 3 && ncn == 3 && ia.settle) ? 1 : 0;
      ClassAcc* acc = nullptr;
      for (auto& q : cls)
        if (q.na == na && q.nc == ncn && q.settle == st) acc = &q;
      if (!acc) {
        cls.push_back(ClassAcc{na, ncn, st, {}, {}});
        acc = &cls.back();
      }
      add_blocks(acc->tab, (int)acc->args.size(), (x.u_end - x.u_begin + 127) / 128);
      acc->args.push_back(x);
    }
    SizeAcc* sa = nullptr;
    for (auto& q : sizes)
      if (q.N == pa.K[0]) sa = &q;
    if (!sa) {
      sizes.push_back(SizeAcc{pa.K[0], {}, {}});
      sa = &sizes.back();
    }
    add_blocks(sa->plane, i, pa.K[2]);
    add_blocks(sa->z, i, fzk::pme_z_groups(pa));
  }
  fz_status r;
  if ((r = bk->upload(rb, &bk->rb)) || (r = bk->upload(nb, &bk->nb)) || (r = bk->upload(bd, &bk->bd)) ||
      (r = bk->upload(pme, &bk->pme)))
    return r;
  for (int k = 0; k < fzk::BT_COUNT; ++k) {
    if ((r = bk->upload(tabs[k], const_cast<int4**>(&bk->t.tab[k])))) return r;
    bk->t.n[k] = (int)tabs[k].size();
  }
  // the pointers in these structs are set when the image is placed: their addresses
  // must stay put, so the vectors are sized first
  bk->classes.resize(cls.size());
  for (size_t k = 0; k < cls.size(); ++k) {
    const auto& q = cls[k];
    bk->classes[k] = fzk::ClassBatch{q.na, q.nc, q.settle, nullptr, nullptr, (int)q.tab.size()};
    if ((r = bk->upload(q.args, const_cast<fzk::IntegrateArgs**>(&bk->classes[k].args))) ||
        (r = bk->upload(q.tab, const_cast<int4**>(&bk->classes[k].tab))))
      return r;
  }
  bk->sizes.resize(sizes.size());
  for (size_t k = 0; k < sizes.size(); ++k) {
    const auto& q = sizes[k];
    bk->sizes[k] = fzk::PmeSizeBatch{q.N, nullptr, (int)q.plane.size(), nullptr, (int)q.z.size()};
    if ((r = bk->upload(q.plane, const_cast<int4**>(&bk->sizes[k].plane_tab))) ||
        (r = bk->upload(q.z, const_cast<int4**>(&bk->sizes[k].z_tab))))
      return r;
  }
  if (!b->aux) {
    FZ_CUDA(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
    FZ_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    FZ_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
  }
  if ((r = bk->place(b->arena, b->master))) return r;
  bk->launches = 2 * (long long)bk->classes.size() + fzk::kRebuildBuildLaunches + fzk::kRebuildPruneLaunches +
                 1 + (bk->t.n[fzk::BT_BONDED] > 0 ? 1 : 0) + 7 + 3 * (long long)bk->sizes.size();
  b->bk = std::move(bk);
  return FZ_OK;
}

// the batched step: kick/drift (one launch per unit class), outer-list rebuild, then PME
// on a second stream beside prune, pair and bonded kernels, then kick/RATTLE.  open /
// close as for the single-system step: inside a chunk graph the kick/RATTLE of a step
// and the kick/drift of the next are one pass.
static void batched_step_body(fz_batch* b, cudaStream_t st, bool open = true, bool close = true) {
  BatchKernels& k = *b->bk;
  for (const auto& c : k.classes) {
    if (open) fzk::launch_kick_drift_b(c, st);
    else fzk::launch_close_kick_drift_b(c, st);
  }
  fzk::launch_rebuild_build_b(k.rb, k.t, st);
  cudaEventRecord(b->ev_fork, st);
  cudaStreamWaitEvent(b->aux, b->ev_fork, 0);
  fzk::launch_pme_b(k.pme, k.t, k.sizes.data(), (int)k.sizes.size(), k.spread_smem, b->aux);
  fzk::launch_rebuild_prune_b(k.rb, k.t, st);
  fzk::launch_nonbonded_b(k.nb, k.t, k.max_ntypes, st);
  fzk::launch_bonded_b(k.bd, k.t, st);
  cudaEventRecord(b->ev_join, b->aux);
  cudaStreamWaitEvent(st, b->ev_join, 0);
  if (close)
    for (const auto& c : k.classes) fzk::launch_kick_rattle_b(c, st);
}

static fz_status capture(fz_batch* b) {
  const int ns = (int)b->systems.size();
  fz_status r;
  for (fz_system* s : b->systems) {
    Engine* e = s->eng;
    if (!e->forces_valid) {
      FZ_CUDA(cudaMemsetAsync(e->facc, 0, 3 * sizeof(long long) * e->n, e->st));
      e->forces(false);
      e->forces_valid = true;
    }
    if ((r = e->check())) return r;
  }
  if (!b->master) {
    FZ_CUDA(cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking));
    FZ_CUDA(cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming));
    FZ_CUDA(cudaEventCreateWithFlags(&b->ev_master, cudaEventDisableTiming));
  }
  b->ev_done.resize(ns, nullptr);
  for (auto& e : b->ev_done) FZ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  FZ_CUDA(cudaMallocHost(&b->pinned_status, sizeof(int) * ns));
  if (batched_kernels_ok(b)) {
    if ((r = build_batch_kernels(b))) return r;
    FZ_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    batched_step_body(b, b->master);
    FZ_CUDA(cudaStreamEndCapture(b->master, &b->graph));
    FZ_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    if (const char* c = std::getenv("FZ_GRAPH_CHUNK"))
      if (b->chunk > 0) b->chunk = std::max(0, std::min(1000, std::atoi(c)));
    if (b->chunk > 1) {
      FZ_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
      const bool fuse = !std::getenv("FZ_FUSE_CLOSE") || std::atoi(std::getenv("FZ_FUSE_CLOSE")) != 0;
      for (int k = 0; k < b->chunk; ++k) batched_step_body(b, b->master, k == 0 || !fuse, k == b->chunk - 1 || !fuse);
      FZ_CUDA(cudaStreamEndCapture(b->master, &b->chunk_graph));
      FZ_CUDA(cudaGraphInstantiate(&b->chunk_exec, b->chunk_graph, 0));
    }
    return FZ_OK;
  }
  FZ_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
  FZ_CUDA(cudaEventRecord(b->ev_start, b->master));
  cudaError_t cap = cudaSuccess;
  for (int i = 0; i < ns; ++i) {
    Engine* e = b->systems[i]->eng;
    FZ_CUDA(cudaStreamWaitEvent(e->st, b->ev_start, 0));
    const long long l0 = e->launches;
    e->capture_error = cudaSuccess;
    e->step_body();
    if (e->capture_error != cudaSuccess) cap = e->capture_error;
    e->launches = l0;
    FZ_CUDA(cudaEventRecord(b->ev_done[i], e->st));
    FZ_CUDA(cudaStreamWaitEvent(b->master, b->ev_done[i], 0));
  }
  FZ_CUDA(cudaStreamEndCapture(b->master, &b->graph));
  if (cap != cudaSuccess) return fail(FZ_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(cap));
  FZ_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return FZ_OK;
}


extern "C" fz_status fz_batch_step(fz_batch* b, int nsteps) {
  if (!b || nsteps < 0) return fail(FZ_ERR_ARG, "bad argument");
  if (b->systems.empty() || nsteps == 0) return FZ_OK;
  FZ_CUDA(cudaSetDevice(b->dev));
  const int ns = (int)b->systems.size();
  fz_status r;
  if (!b->exec && (r = capture(b))) return r;
  // work queued on the systems' own streams precedes the batch
  for (int i = 0; i < ns; ++i) {
    FZ_CUDA(cudaEventRecord(b->ev_done[i], b->systems[i]->eng->st));
    FZ_CUDA(cudaStreamWaitEvent(b->master, b->ev_done[i], 0));
  }
  int left = nsteps;
  while (left > 0) {
    int k = left;
    for (fz_system* s : b->systems) {
      const Engine* e = s->eng;
      if (e->temp_reset_every > 0) k = std::min<long long>(k, e->temp_reset_every - e->step % e->temp_reset_every);
    }
    int j = 0;
    if (b->chunk_exec)
      for (; j + b->chunk <= k; j += b->chunk) FZ_CUDA(cudaGraphLaunch(b->chunk_exec, b->master));
    for (; j < k; ++j) FZ_CUDA(cudaGraphLaunch(b->exec, b->master));
    for (int i = 0; i < ns; ++i) {
      Engine* e = b->systems[i]->eng;
      e->step += k;
      e->launches += (long long)k * e->graph_step_launches();
      e->graph_since_check = true;
      if (e->temp_reset_every > 0 && e->step % e->temp_reset_every == 0) {
        FZ_CUDA(cudaEventRecord(b->ev_master, b->master));
        FZ_CUDA(cudaStreamWaitEvent(e->st, b->ev_master, 0));
        fzk::launch_reassign(e->int_args(), e->temperature, e->seed, (uint32_t)(e->step / e->temp_reset_every),
                             e->inv_mtot, e->psum, e->st);
        e->launches += 3 + e->ncls;
        FZ_CUDA(cudaEventRecord(b->ev_done[i], e->st));
        FZ_CUDA(cudaStreamWaitEvent(b->master, b->ev_done[i], 0));
      }
    }
    left -= k;
  }
  for (int i = 0; i < ns; ++i)
    FZ_CUDA(cudaMemcpyAsync(b->pinned_status + i, b->systems[i]->eng->status, sizeof(int), cudaMemcpyDeviceToHost,
                            b->master));
  // later per-system work is ordered after the batch
  FZ_CUDA(cudaEventRecord(b->ev_master, b->master));
  for (fz_system* s : b->systems) FZ_CUDA(cudaStreamWaitEvent(s->eng->st, b->ev_master, 0));
  FZ_CUDA(cudaStreamSynchronize(b->master));
  for (int i = 0; i < ns; ++i)
    if (b->pinned_status[i] && (r = b->systems[i]->eng->check()))
      return fail(r, "system " + std::to_string(i) + " of the batch: " + last_error_text());
  b->steps += nsteps;
  return FZ_OK;
}

extern "C" fz_status fz_batch_size(fz_batch* b, int* out) {
  if (!b || !out) return fail(FZ_ERR_ARG, "null argument");
  *out = (int)b->systems.size();
  return FZ_OK;
}

extern "C" fz_status fz_batch_free(fz_batch* b) {
  delete b;
  return FZ_OK;
}

// ====================================================================== serving loop
namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int id = 0;
  fz_system* sys = nullptr;
  long long nsteps = 0, done = 0;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  fz_status status = FZ_OK;
  std::string err;
  double t_submit = 0, t_start = -1, t_end = -1;
  size_t est_bytes = 0;
  fz_energies final{};
  std::vector<double> pos;
};

// Device bytes of one uploaded system, an upper estimate of build_engine's allocations:
// ~140 B per atom of atom, slot and PME-binning arrays, the per-block pair lists, masks
// and work items (~0.5 B per atom per unit of list capacity, the capacity estimated as
// build_engine does), the PME grids and charge staging (~24 B per grid point), and 8 MiB
// of fixed overhead.
size_t engine_bytes_estimate(const fz_system* s) {
  const double n = (double)s->top.n;
  const double V = s->cfg.box[0] * s->cfg.box[1] * s->cfg.box[2];
  const double rho = n / V;
  const double K3 = (double)s->cfg.pme_grid[0] * s->cfg.pme_grid[1] * s->cfg.pme_grid[2];
  const double R = std::max(s->cfg.pairlistdist, s->cfg.cutoff);
  const double a = 1.4 * std::cbrt(32.0 / rho);
  const double vm = a * a * a + 6 * a * a * R + 3 * M_PI * a * R * R + 4.0 / 3.0 * M_PI * R * R * R;
  const double ocap = std::max(256.0, 1.25 * rho * vm);
  return (size_t)(n * (140.0 + 0.5 * ocap) + 24.0 * K3) + ((size_t)8 << 20);
}

}  // namespace

struct fz_server {
  int dev = 0;
  size_t budget = 0;
  int chunk = 100, max_running = 64;
  Clock::time_point t0 = Clock::now();
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int> queue;
  std::unordered_map<int, std::unique_ptr<Job>> jobs;
  int next_id = 1;
  bool stop = false;
  std::thread worker;
  size_t in_use = 0;
  int running_now = 0, peak_running = 0;
  long long atom_steps = 0, finished = 0;
  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
};

void fz_server::run() {
  cudaSetDevice(dev);
  fz_batch* batch = nullptr;
  fz_batch_create(&batch);
  // the membership changes about every chunk (a job ends): a multi-step graph would be
  // captured for one replay, so the served batch replays its one-step graph
  batch->chunk = 0;
  std::vector<Job*> running;
  auto finish = [&](Job* j, fz_status st, const std::string& msg) {
    if (j->sys->eng) {
      fz_batch_remove(batch, j->sys);
      destroy_engine(j->sys->eng);
      j->sys->eng = nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    j->status = st;
    j->err = msg;
    j->state = st == FZ_OK ? 2 : 3;
    j->t_end = now();
    in_use -= j->est_bytes;
    finished++;
    cv_done.notify_all();
  };
  for (;;) {
    std::vector<Job*> admit;
    {
      std::unique_lock<std::mutex> lock(mu);
      for (;;) {
        while (!queue.empty() && (int)(running.size() + admit.size()) < max_running) {
          Job* j = jobs[queue.front()].get();
          if (j->est_bytes > budget) {  // can never fit: fail it
            queue.pop_front();
            j->status = FZ_ERR_CAPACITY;
            j->err = "job needs ~" + std::to_string(j->est_bytes >> 20) + " MiB, above the HBM budget";
            j->state = 3;
            j->t_end = now();
            finished++;
            cv_done.notify_all();
            continue;
          }
          if (in_use + j->est_bytes > budget) break;  // FIFO: wait for memory
          queue.pop_front();
          in_use += j->est_bytes;
          j->state = 1;
          j->t_start = now();
          admit.push_back(j);
        }
        if (!running.empty() || !admit.empty()) break;
        if (stop) {
          lock.unlock();
          fz_batch_free(batch);
          return;
        }
        cv_work.wait(lock);
      }
    }
    for (Job* j : admit) {
      // InitMem + InitVelocity of the reference's main (src/fenzi.cu:212-232): Maxwell-
      // Boltzmann velocities at the input's temperature and seed
      fz_status r = fz_upload(j->sys, dev, nullptr);
      if (!r) r = fz_reassign_velocities(j->sys, j->sys->cfg.temperature, (uint64_t)j->sys->cfg.seed, 0);
      if (!r) r = fz_batch_add(batch, j->sys);
      if (r) {
        finish(j, r, last_error_text());
        continue;
      }
      running.push_back(j);
    }
    {
      std::lock_guard<std::mutex> lock(mu);
      running_now = (int)running.size();
      peak_running = std::max(peak_running, running_now);
    }
    if (running.empty()) continue;
    long long k = chunk;
    for (Job* j : running) k = std::min(k, j->nsteps - j->done);
    fz_status r = fz_batch_step(batch, (int)k);
    if (r) {
      // find the failing systems; the others continue
      const std::string msg = last_error_text();
      std::vector<Job*> keep;
      for (Job* j : running) {
        if (fz_sync(j->sys) != FZ_OK)
          finish(j, FZ_ERR_CUDA, last_error_text());
        else
          keep.push_back(j);
      }
      if (keep.size() == running.size()) {  // not attributable: fail the whole mix
        for (Job* j : running) finish(j, r, msg);
        keep.clear();
      }
      running.swap(keep);
      continue;
    }
    std::vector<Job*> keep;
    for (Job* j : running) {
      j->done += k;
      {
        std::lock_guard<std::mutex> lock(mu);
        atom_steps += (long long)j->sys->top.n * k;
      }
      if (j->done < j->nsteps) {
        keep.push_back(j);
        continue;
      }
      fz_status st = fz_eval_props(j->sys, &j->final);
      if (!st) {
        j->pos.resize(3 * (size_t)j->sys->top.n);
        st = fz_get_positions(j->sys, j->pos.data());
      }
      finish(j, st, st ? last_error_text() : std::string());
    }
    running.swap(keep);
  }
}

extern "C" fz_status fz_server_estimate_bytes(const fz_system* sys, double* out) {
  if (!sys || !out) return fail(FZ_ERR_ARG, "null argument");
  *out = (double)engine_bytes_estimate(sys);
  return FZ_OK;
}

extern "C" fz_status fz_server_create(int device, double hbm_budget_bytes, int chunk_steps, int max_running,
                                      fz_server** out) {
  if (!out) return fail(FZ_ERR_ARG, "null output");
  if (!(hbm_budget_bytes > 0) || chunk_steps <= 0 || max_running <= 0)
    return fail(FZ_ERR_ARG, "fz_server_create: budget, chunk and slots must be positive");
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess) return fail(FZ_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(ce));
  if (device < 0 || device >= ndev) return fail(FZ_ERR_ARG, "fz_server_create: no such device");
  fz_server* sv = new fz_server();
  sv->dev = device;
  sv->budget = (size_t)hbm_budget_bytes;
  sv->chunk = chunk_steps;
  sv->max_running = max_running;
  sv->worker = std::thread([sv] { sv->run(); });
  *out = sv;
  return FZ_OK;
}

extern "C" fz_status fz_server_submit(fz_server* sv, fz_system* sys, long long nsteps, int* job_id) {
  if (!sv || !sys || !job_id) return fail(FZ_ERR_ARG, "null argument");
  if (nsteps <= 0) return fail(FZ_ERR_ARG, "fz_server_submit: nsteps must be positive");
  if (sys->eng) return fail(FZ_ERR_STATE, "fz_server_submit: the server uploads the system itself");
  std::unique_ptr<Job> j(new Job());
  j->sys = sys;
  j->nsteps = nsteps;
  j->est_bytes = engine_bytes_estimate(sys);
  std::lock_guard<std::mutex> lock(sv->mu);
  if (sv->stop) return fail(FZ_ERR_STATE, "fz_server_submit: server is stopping");
  j->id = sv->next_id++;
  j->t_submit = sv->now();
  *job_id = j->id;
  sv->queue.push_back(j->id);
  sv->jobs[j->id] = std::move(j);
  sv->cv_work.notify_all();
  return FZ_OK;
}

static void fill_info(const Job& j, fz_job_info* o) {
  o->job = j.id;
  o->state = j.state;
  o->status = j.status;
  o->nsteps = j.nsteps;
  o->steps_done = j.done;
  o->natom = j.sys->top.n;
  o->submit_s = j.t_submit;
  o->start_s = j.t_start;
  o->end_s = j.t_end;
  o->device_bytes = (double)j.est_bytes;
  o->final = j.final;
}

extern "C" fz_status fz_server_info(fz_server* sv, int job_id, fz_job_info* out) {
  if (!sv || !out) return fail(FZ_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(job_id);
  if (it == sv->jobs.end()) return fail(FZ_ERR_ARG, "fz_server_info: unknown job");
  fill_info(*it->second, out);
  return FZ_OK;
}

extern "C" fz_status fz_server_wait(fz_server* sv, int job_id, fz_job_info* out) {
  if (!sv) return fail(FZ_ERR_ARG, "null argument");
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(job_id);
  if (it == sv->jobs.end()) return fail(FZ_ERR_ARG, "fz_server_wait: unknown job");
  Job* j = it->second.get();
  sv->cv_done.wait(lock, [j] { return j->state >= 2; });
  if (out) fill_info(*j, out);
  if (j->status) return fail(j->status, "job " + std::to_string(j->id) + ": " + j->err);
  return FZ_OK;
}

extern "C" fz_status fz_server_positions(fz_server* sv, int job_id, double* out) {
  if (!sv || !out) return fail(FZ_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(sv->mu);
  auto it = sv->jobs.find(job_id);
  if (it == sv->jobs.end()) return fail(FZ_ERR_ARG, "fz_server_positions: unknown job");
  if (it->second->state != 2) return fail(FZ_ERR_STATE, "fz_server_positions: job has not finished");
  std::copy(it->second->pos.begin(), it->second->pos.end(), out);
  return FZ_OK;
}

extern "C" fz_status fz_server_stats(fz_server* sv, double* out4) {
  if (!sv || !out4) return fail(FZ_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(sv->mu);
  out4[0] = (double)sv->peak_running;
  out4[1] = (double)sv->atom_steps;
  out4[2] = (double)sv->in_use;
  out4[3] = (double)sv->finished;
  return FZ_OK;
}

extern "C" fz_status fz_server_free(fz_server* sv) {
  if (!sv) return FZ_OK;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
    sv->cv_work.notify_all();
  }
  if (sv->worker.joinable()) sv->worker.join();  // queued and running jobs finish first
  for (auto& kv : sv->jobs) fz_free(kv.second->sys);
  delete sv;
  return FZ_OK;
}
