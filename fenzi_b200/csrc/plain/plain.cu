// Host side of the plain comparator path (include/fenzi_plain.h): one engine per
// system, templated on the arithmetic type, driving the kernels of plain_*.cuh one
// launch per stage with a host synchronisation every step.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/fenzi_plain.h"
#include "../host/host.h"
#include "plain_kernels.cuh"
#include "plain_pme_int.cuh"
#include "plain_terms.cuh"

using fz::fail;

namespace fzp {

static fz_status cuda_fail(cudaError_t e, const char* what) {
  return fail(FZ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct Base {
  virtual ~Base() {}
  virtual fz_status set_state(const double* pos, const double* vel) = 0;
  virtual fz_status get_state(double* pos, double* vel) = 0;
  virtual fz_status compute_forces(double* out) = 0;
  virtual fz_status step(int nsteps) = 0;
  virtual fz_status eval(fz_energies* out) = 0;
  virtual fz_status counters(long long* out4) = 0;
};

inline int blocks(long long n, int bs = 256) { return (int)((n + bs - 1) / bs); }

template <class T> struct Engine final : Base {
  using V4 = typename Vec<T>::v4;
  using C = typename Vec<T>::cplx;
  int dev = 0;
  cudaStream_t st = nullptr;
  Prm<T> p{};
  int n = 0, Kt = 0;
  std::vector<void*> allocs;
  V4 *pos = nullptr, *pos_old = nullptr, *pos_build = nullptr, *vel = nullptr, *force = nullptr;
  T *inv_m = nullptr, *mass = nullptr, *evdw = nullptr, *eelec = nullptr, *epme = nullptr;
  int* type = nullptr;
  T *eps4 = nullptr, *sig2 = nullptr;
  int *excl_off = nullptr, *excl_idx = nullptr;
  int *cell_n = nullptr, *cell_atoms = nullptr, *nbl = nullptr, *nbn = nullptr;
  int *lat_n = nullptr, *lat_list = nullptr;
  C* grid = nullptr;
  T* infl = nullptr;
  cufftHandle plan = 0;
  bool have_plan = false;
  Terms<T> terms{};
  int nterms = 0;
  Clusters cl{};
  V4* cl_d = nullptr;
  double* e_acc = nullptr;
  int* status = nullptr;
  unsigned int* dmax = nullptr;
  double* h_e = nullptr;  // pinned: energy accumulators
  int* h_flags = nullptr; // pinned: {dmax bits, status}
  std::vector<double> q;
  double dt = 0, self_energy = 0, skin_half2 = 0, box[3] = {0, 0, 0};
  T tol_shake = 0, tol_rattle = 0;
  int maxit = 1000, ncons = 0;
  bool need_build = true, have_forces = false;
  long long rebuilds = 0, steps = 0, launches = 0;

  ~Engine() override {
    if (dev >= 0) cudaSetDevice(dev);
    if (st) cudaStreamSynchronize(st);
    if (have_plan) cufftDestroy(plan);
    for (void* a : allocs) cudaFree(a);
    if (h_e) cudaFreeHost(h_e);
    if (h_flags) cudaFreeHost(h_flags);
    if (st) cudaStreamDestroy(st);
  }

  template <class X> fz_status alloc(X** ptr, size_t count) {
    void* d = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(X);
    const cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "plain path: device allocation");
    cudaMemsetAsync(d, 0, bytes, st);
    allocs.push_back(d);
    *ptr = (X*)d;
    return FZ_OK;
  }
  template <class X> fz_status upload(X** ptr, const std::vector<X>& v) {
    fz_status r = alloc(ptr, v.size());
    if (r) return r;
    if (!v.empty()) cudaMemcpyAsync(*ptr, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st);
    return FZ_OK;
  }
  template <class X> void release(X*& ptr) {
    if (!ptr) return;
    cudaStreamSynchronize(st);
    auto it = std::find(allocs.begin(), allocs.end(), (void*)ptr);
    if (it != allocs.end()) allocs.erase(it);
    cudaFree(ptr);
    ptr = nullptr;
  }
  template <class X> std::vector<T> to_t(const std::vector<X>& v) { return std::vector<T>(v.begin(), v.end()); }

  fz_status create(const fz_system* sys, int device) {
    dev = device;
    cudaError_t ce = cudaSetDevice(dev);
    if (ce != cudaSuccess) return cuda_fail(ce, "plain path: cudaSetDevice");
    if ((ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess)
      return cuda_fail(ce, "plain path: stream");
    const fz_config& c = sys->cfg;
    const fz::Topology& t = sys->top;
    n = t.n;
    if (n <= 0) return fail(FZ_ERR_STATE, "plain path: the system has no atoms loaded");
    const int nt = (int)std::lround(std::sqrt((double)t.eps4.size()));
    p.n = n;
    p.nt = nt;
    const double rc = c.cutoff, ron = std::min(c.cuton, c.cutoff), rl = std::max(c.pairlistdist, c.cutoff);
    for (int d = 0; d < 3; ++d) {
      box[d] = c.box[d];
      p.L[d] = (T)c.box[d];
      p.iL[d] = (T)(1.0 / c.box[d]);
      p.K[d] = c.pme_grid[d];
      if (p.K[d] < 4) return fail(FZ_ERR_ARG, "plain path: PME grid sizes must be >= 4");
      p.nc[d] = std::max(1, (int)std::floor(c.box[d] / rl));
    }
    p.rc2 = (T)(rc * rc);
    p.ron2 = (T)(ron * ron);
    p.rl2 = (T)(rl * rl);
    p.beta = (T)c.kappa;
    p.cc = (T)fz::kCC;
    p.sw_c3 = ron < rc ? (T)(1.0 / std::pow(rc * rc - ron * ron, 3)) : (T)0;
    skin_half2 = 0.25 * (rl - rc) * (rl - rc);
    const double V = c.box[0] * c.box[1] * c.box[2];
    const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
    p.cell_cap = (int)(1.5 * n / ncell) + 64;
    p.maxnb = (int)(4.0 / 3.0 * M_PI * rl * rl * rl * n / V * 1.3) + 64;
    dt = c.timestep_ps * fz::kTU;
    self_energy = t.self_energy;
    tol_shake = sizeof(T) == 8 ? (T)1e-12 : (T)1e-6;
    tol_rattle = tol_shake;
    ncons = (int)t.cons_d.size();
    fz_status r;
    // atoms
    std::vector<V4> p4(n);
    std::vector<T> im(n), ms(n);
    q = t.q;
    for (int a = 0; a < n; ++a) {
      p4[a].x = (T)t.pos[3 * a];
      p4[a].y = (T)t.pos[3 * a + 1];
      p4[a].z = (T)t.pos[3 * a + 2];
      p4[a].w = (T)t.q[a];
      ms[a] = (T)t.mass[a];
      im[a] = t.mass[a] > 0 ? (T)(1.0 / t.mass[a]) : (T)0;
    }
    if ((r = upload(&pos, p4)) || (r = alloc(&pos_old, n)) || (r = alloc(&pos_build, n)) || (r = alloc(&vel, n)) ||
        (r = alloc(&force, n)) || (r = upload(&inv_m, im)) || (r = upload(&mass, ms)) || (r = alloc(&evdw, n)) ||
        (r = alloc(&eelec, n)) || (r = alloc(&epme, n)) || (r = upload(&type, t.type)) ||
        (r = upload(&eps4, to_t(t.eps4))) || (r = upload(&sig2, to_t(t.sig2))) || (r = upload(&excl_off, t.excl_off)) ||
        (r = upload(&excl_idx, t.excl_idx)))
      return r;
    if ((r = alloc(&cell_n, ncell)) || (r = alloc(&cell_atoms, (size_t)ncell * p.cell_cap)) ||
        (r = alloc(&nbl, (size_t)p.maxnb * n)) || (r = alloc(&nbn, n)))
      return r;
    // bonded terms
    {
      std::vector<int2> b, u, x, q14;
      std::vector<int4> an, dh, ip;
      for (size_t k = 0; k < t.bond_k.size(); ++k) b.push_back(make_int2(t.bond[2 * k], t.bond[2 * k + 1]));
      for (size_t k = 0; k < t.ub_k.size(); ++k) u.push_back(make_int2(t.ub[2 * k], t.ub[2 * k + 1]));
      for (size_t k = 0; k < t.angle_k.size(); ++k)
        an.push_back(make_int4(t.angle[3 * k], t.angle[3 * k + 1], t.angle[3 * k + 2], 0));
      for (size_t k = 0; k < t.dihe_k.size(); ++k)
        dh.push_back(make_int4(t.dihe[4 * k], t.dihe[4 * k + 1], t.dihe[4 * k + 2], t.dihe[4 * k + 3]));
      for (size_t k = 0; k < t.impr_k.size(); ++k)
        ip.push_back(make_int4(t.impr[4 * k], t.impr[4 * k + 1], t.impr[4 * k + 2], t.impr[4 * k + 3]));
      for (size_t k = 0; k < t.p14_pairs.size() / 2; ++k)
        q14.push_back(make_int2(t.p14_pairs[2 * k], t.p14_pairs[2 * k + 1]));
      for (size_t k = 0; k < t.excl_pairs.size() / 2; ++k)
        x.push_back(make_int2(t.excl_pairs[2 * k], t.excl_pairs[2 * k + 1]));
      int2 *db, *du, *d14, *dx;
      int4 *dan, *ddh, *dip;
      T *bk, *br, *uk, *ur, *ak, *at, *dk, *dd, *ik, *i0, *e14, *s14;
      int* dn;
      if ((r = upload(&db, b)) || (r = upload(&bk, to_t(t.bond_k))) || (r = upload(&br, to_t(t.bond_r0))) ||
          (r = upload(&du, u)) || (r = upload(&uk, to_t(t.ub_k))) || (r = upload(&ur, to_t(t.ub_r0))) ||
          (r = upload(&dan, an)) || (r = upload(&ak, to_t(t.angle_k))) || (r = upload(&at, to_t(t.angle_t0))) ||
          (r = upload(&ddh, dh)) || (r = upload(&dk, to_t(t.dihe_k))) || (r = upload(&dn, t.dihe_n)) ||
          (r = upload(&dd, to_t(t.dihe_d))) || (r = upload(&dip, ip)) || (r = upload(&ik, to_t(t.impr_k))) ||
          (r = upload(&i0, to_t(t.impr_p0))) || (r = upload(&d14, q14)) || (r = upload(&e14, to_t(t.eps4_14))) ||
          (r = upload(&s14, to_t(t.sig2_14))) || (r = upload(&dx, x)))
        return r;
      terms = Terms<T>{(int)b.size(), (int)u.size(), (int)an.size(), (int)dh.size(), (int)ip.size(), (int)q14.size(),
                       (int)x.size(), db, bk, br, du, uk, ur, dan, ak, at, ddh, dk, dn, dd, dip, ik, i0, d14, e14, s14,
                       dx, type};
      nterms = terms.nbond + terms.nub + terms.nangle + terms.ndihe + terms.nimpr + terms.n14 + terms.nexcl;
    }
    // SHAKE clusters
    {
      std::vector<int4> ca, cp;
      std::vector<V4> cd;
      for (const auto& k : t.clusters) {
        ca.push_back(make_int4(k.atom[0], k.atom[1], k.atom[2], k.atom[3]));
        int bits = 0;
        for (int j = 0; j < k.nc; ++j) bits |= (k.ca[j] << (4 * j)) | (k.cb[j] << (4 * j + 2));
        cp.push_back(make_int4(k.na, k.nc, bits, 0));
        V4 d;
        d.x = (T)k.d[0];
        d.y = (T)k.d[1];
        d.z = (T)k.d[2];
        d.w = 0;
        cd.push_back(d);
      }
      int4 *da, *dp;
      if ((r = upload(&da, ca)) || (r = upload(&dp, cp)) || (r = upload(&cl_d, cd))) return r;
      cl = Clusters{(int)ca.size(), da, dp};
    }
    // PME
    Kt = p.K[0] * p.K[1] * p.K[2];
    if ((r = alloc(&lat_n, Kt)) || (r = alloc(&lat_list, (size_t)Kt * kLatCap)) || (r = alloc(&grid, Kt))) return r;
    {
      // C(m) = CC exp(-pi^2 m^2 / beta^2) / (pi V m^2) B(m), B = prod 1/(2/3 + cos(2 pi m/K)/3)^2
      // (BCMultiply and InitDeviceConstants, src/cell_based_kernels.cu:1770-1903)
      std::vector<double> bm[3];
      for (int d = 0; d < 3; ++d) {
        bm[d].resize(p.K[d]);
        for (int m = 0; m < p.K[d]; ++m) {
          const double den = 2.0 / 3.0 + std::cos(2.0 * M_PI * m / p.K[d]) / 3.0;
          bm[d][m] = 1.0 / (den * den);
        }
      }
      std::vector<T> h(Kt);
      const double b2 = c.kappa * c.kappa;
      for (int ix = 0; ix < p.K[0]; ++ix)
        for (int iy = 0; iy < p.K[1]; ++iy)
          for (int iz = 0; iz < p.K[2]; ++iz) {
            const double mx = (ix <= p.K[0] / 2 ? ix : ix - p.K[0]) / c.box[0];
            const double my = (iy <= p.K[1] / 2 ? iy : iy - p.K[1]) / c.box[1];
            const double mz = (iz <= p.K[2] / 2 ? iz : iz - p.K[2]) / c.box[2];
            const double m2 = mx * mx + my * my + mz * mz;
            const size_t g = ((size_t)ix * p.K[1] + iy) * p.K[2] + iz;
            h[g] = m2 > 0 ? (T)(fz::kCC * std::exp(-M_PI * M_PI * m2 / b2) / (M_PI * V * m2) * bm[0][ix] * bm[1][iy] *
                                bm[2][iz])
                          : (T)0;
          }
      if ((r = upload(&infl, h))) return r;
    }
    if (cufftPlan3d(&plan, p.K[0], p.K[1], p.K[2], sizeof(T) == 8 ? CUFFT_Z2Z : CUFFT_C2C) != CUFFT_SUCCESS)
      return fail(FZ_ERR_CUDA, "plain path: cufftPlan3d failed");
    have_plan = true;
    cufftSetStream(plan, st);
    if ((r = alloc(&e_acc, PE_N)) || (r = alloc(&status, 2)) || (r = alloc(&dmax, 1))) return r;
    if ((ce = cudaMallocHost(&h_e, PE_N * sizeof(double))) != cudaSuccess ||
        (ce = cudaMallocHost(&h_flags, 2 * sizeof(int))) != cudaSuccess)
      return cuda_fail(ce, "plain path: pinned buffers");
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ce, "plain path: upload");
    return FZ_OK;
  }

  fz_status sync_check(const char* where) {
    const cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return cuda_fail(ce, where);
    return FZ_OK;
  }

  fz_status flags_status(int s) {
    if (s & PS_BAD_COORD) return fail(FZ_ERR_STATE, "plain path: non-finite or runaway coordinates");
    if (s & PS_SHAKE) return fail(FZ_ERR_SHAKE, "plain path: SHAKE/RATTLE did not converge");
    if (s & PS_LATTICE_OVF) return fail(FZ_ERR_CAPACITY, "plain path: more than 64 atoms on one PME grid point");
    return FZ_OK;
  }

  // cell list + full neighbour list; capacities grow on overflow and the build repeats
  fz_status build() {
    const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
    for (int attempt = 0; attempt < 6; ++attempt) {
      cudaMemsetAsync(cell_n, 0, ncell * sizeof(int), st);
      cudaMemsetAsync(status + 1, 0, sizeof(int), st);
      k_cells<T><<<blocks(n), 256, 0, st>>>(p, pos, pos_build, cell_n, cell_atoms, status + 1);
      k_nblist<T><<<blocks(n, 128), 128, 0, st>>>(p, pos, cell_n, cell_atoms, excl_off, excl_idx, nbl, nbn,
                                                  status + 1);
      launches += 2;
      cudaMemcpyAsync(h_flags + 1, status + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
      fz_status r = sync_check("plain path: list build");
      if (r) return r;
      const int s = h_flags[1];
      if (s & PS_BAD_COORD) return flags_status(s);
      if (!(s & (PS_CELL_OVF | PS_LIST_OVF))) {
        ++rebuilds;
        need_build = false;
        return FZ_OK;
      }
      if (s & PS_CELL_OVF) {
        release(cell_atoms);
        p.cell_cap = p.cell_cap * 3 / 2 + 32;
        if ((r = alloc(&cell_atoms, (size_t)ncell * p.cell_cap))) return r;
      }
      if (s & PS_LIST_OVF) {
        release(nbl);
        p.maxnb = p.maxnb * 3 / 2 + 32;
        if ((r = alloc(&nbl, (size_t)p.maxnb * n))) return r;
      }
    }
    return fail(FZ_ERR_CAPACITY, "plain path: neighbour capacities did not settle");
  }

  // ComputeAccelGPU: nonbonded (writes), bonded (atomic adds), PME (adds)
  void forces() {
    cudaMemsetAsync(e_acc, 0, PE_N * sizeof(double), st);
    k_nonbonded<T><<<blocks(n, 128), 128, 0, st>>>(p, pos, type, eps4, sig2, nbl, nbn, force, evdw, eelec);
    ++launches;
    if (nterms) {
      k_terms<T><<<blocks(nterms), 256, 0, st>>>(p, terms, pos, force, e_acc);
      ++launches;
    }
    cudaMemsetAsync(lat_n, 0, (size_t)Kt * sizeof(int), st);
    k_lattice<T><<<blocks(n), 256, 0, st>>>(p, pos, lat_n, lat_list, status);
    k_spread<T><<<blocks(Kt), 256, 0, st>>>(p, pos, lat_n, lat_list, grid);
    if constexpr (sizeof(T) == 8) cufftExecZ2Z(plan, grid, grid, CUFFT_FORWARD);
    else cufftExecC2C(plan, grid, grid, CUFFT_FORWARD);
    k_bcmult<T><<<blocks(Kt), 256, 0, st>>>(Kt, grid, infl);
    if constexpr (sizeof(T) == 8) cufftExecZ2Z(plan, grid, grid, CUFFT_INVERSE);
    else cufftExecC2C(plan, grid, grid, CUFFT_INVERSE);
    k_gather<T><<<blocks(n, 128), 128, 0, st>>>(p, pos, grid, force, epme);
    launches += 6;
  }

  fz_status ensure_forces() {
    fz_status r;
    if (need_build && (r = build())) return r;
    forces();
    have_forces = true;
    return FZ_OK;
  }

  // SingleStep (src/dynamics.cu:623-820): kick, drift, SHAKE, wrap; the displacement
  // test read on the host; list rebuild when due; forces; kick, RATTLE
  fz_status step(int nsteps) override {
    if (nsteps < 0) return fail(FZ_ERR_ARG, "plain path: negative step count");
    cudaSetDevice(dev);
    fz_status r;
    if (!have_forces && (r = ensure_forces())) return r;
    const T hdt = (T)(0.5 * dt), tdt = (T)dt, idt = (T)(1.0 / dt);
    for (int s = 0; s < nsteps; ++s) {
      cudaMemsetAsync(dmax, 0, sizeof(unsigned int), st);
      k_kick<T><<<blocks(n), 256, 0, st>>>(n, hdt, force, inv_m, vel);
      k_drift<T><<<blocks(n), 256, 0, st>>>(n, tdt, pos, vel, pos_old);
      launches += 2;
      if (cl.n) {
        k_shake<T><<<blocks(cl.n, 128), 128, 0, st>>>(p, cl, cl_d, pos_old, pos, vel, inv_m, idt, tol_shake, maxit,
                                                      status);
        ++launches;
      }
      k_wrap_disp<T><<<blocks(n), 256, 0, st>>>(p, pos, pos_build, dmax);
      ++launches;
      cudaMemcpyAsync(h_flags, dmax, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(h_flags + 1, status, sizeof(int), cudaMemcpyDeviceToHost, st);
      if ((r = sync_check("plain path: step"))) return r;
      if ((r = flags_status(h_flags[1]))) return r;
      float d2;
      std::memcpy(&d2, &h_flags[0], sizeof(float));
      if ((double)d2 > skin_half2) need_build = true;
      if ((r = ensure_forces())) return r;
      k_kick<T><<<blocks(n), 256, 0, st>>>(n, hdt, force, inv_m, vel);
      ++launches;
      if (cl.n) {
        k_rattle<T><<<blocks(cl.n, 128), 128, 0, st>>>(p, cl, cl_d, pos, vel, inv_m, tol_rattle, maxit, status);
        ++launches;
      }
      ++steps;
    }
    cudaMemcpyAsync(h_flags + 1, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((r = sync_check("plain path: step"))) return r;
    return flags_status(h_flags[1]);
  }

  fz_status set_state(const double* x, const double* v) override {
    cudaSetDevice(dev);
    std::vector<V4> h(n);
    fz_status r;
    if (x) {
      for (int a = 0; a < n; ++a) {
        h[a].x = (T)x[3 * a];
        h[a].y = (T)x[3 * a + 1];
        h[a].z = (T)x[3 * a + 2];
        h[a].w = (T)q[a];
      }
      cudaMemcpyAsync(pos, h.data(), n * sizeof(V4), cudaMemcpyHostToDevice, st);
      if ((r = sync_check("plain path: set positions"))) return r;
      need_build = true;
      have_forces = false;
    }
    if (v) {
      for (int a = 0; a < n; ++a) {
        h[a].x = (T)v[3 * a];
        h[a].y = (T)v[3 * a + 1];
        h[a].z = (T)v[3 * a + 2];
        h[a].w = 0;
      }
      cudaMemcpyAsync(vel, h.data(), n * sizeof(V4), cudaMemcpyHostToDevice, st);
      if ((r = sync_check("plain path: set velocities"))) return r;
    }
    return FZ_OK;
  }

  fz_status get_array(const V4* src, double* out) {
    std::vector<V4> h(n);
    cudaMemcpyAsync(h.data(), src, n * sizeof(V4), cudaMemcpyDeviceToHost, st);
    fz_status r = sync_check("plain path: read back");
    if (r) return r;
    for (int a = 0; a < n; ++a) {
      out[3 * a] = (double)h[a].x;
      out[3 * a + 1] = (double)h[a].y;
      out[3 * a + 2] = (double)h[a].z;
    }
    return FZ_OK;
  }

  fz_status get_state(double* x, double* v) override {
    cudaSetDevice(dev);
    fz_status r;
    if (x && (r = get_array(pos, x))) return r;
    if (v && (r = get_array(vel, v))) return r;
    return FZ_OK;
  }

  fz_status compute_forces(double* out) override {
    cudaSetDevice(dev);
    fz_status r;
    if ((r = ensure_forces())) return r;
    cudaMemcpyAsync(h_flags + 1, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((r = sync_check("plain path: forces"))) return r;
    if ((r = flags_status(h_flags[1]))) return r;
    return out ? get_array(force, out) : FZ_OK;
  }

  fz_status eval(fz_energies* out) override {
    cudaSetDevice(dev);
    fz_status r;
    if ((r = ensure_forces())) return r;
    k_energy<T><<<148, 256, 0, st>>>(n, evdw, eelec, epme, vel, mass, e_acc);
    ++launches;
    cudaMemcpyAsync(h_e, e_acc, PE_N * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_flags + 1, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((r = sync_check("plain path: energies"))) return r;
    if ((r = flags_status(h_flags[1]))) return r;
    std::memset(out, 0, sizeof(*out));
    out->bond = h_e[PE_BOND];
    out->angle = h_e[PE_ANGLE];
    out->ureyb = h_e[PE_UREYB];
    out->dihed = h_e[PE_DIHED];
    out->impr = h_e[PE_IMPR];
    out->vdw = h_e[PE_VDW];
    out->elec = h_e[PE_ELEC];
    out->pme = h_e[PE_PME];
    out->ewexcl = h_e[PE_EWEXCL];
    out->ewself = self_energy;
    out->potential = out->bond + out->angle + out->ureyb + out->dihed + out->impr + out->vdw + out->elec + out->pme +
                     out->ewexcl + out->ewself;
    out->kinetic = 0.5 * h_e[PE_KIN2];
    const double dof = 3.0 * n - 6.0 - ncons;
    out->temperature = dof > 0 ? 2.0 * out->kinetic / (fz::kRC * dof) : 0.0;
    out->step = steps;
    for (int d = 0; d < 3; ++d) out->box[d] = box[d];
    out->volume = box[0] * box[1] * box[2];
    out->conserved = out->kinetic + out->potential;
    return FZ_OK;
  }

  fz_status counters(long long* out4) override {
    cudaSetDevice(dev);
    std::vector<int> h(n);
    cudaMemcpyAsync(h.data(), nbn, n * sizeof(int), cudaMemcpyDeviceToHost, st);
    fz_status r = sync_check("plain path: counters");
    if (r) return r;
    long long s = 0;
    for (int v : h) s += v;
    out4[0] = rebuilds;
    out4[1] = s;
    out4[2] = steps;
    out4[3] = launches;
    return FZ_OK;
  }
};

}  // namespace fzp

struct fz_plain {
  fzp::Base* impl = nullptr;
};

extern "C" fz_status fz_plain_create(const fz_system* sys, int device, int fp64, fz_plain** out) {
  if (!sys || !out) return fail(FZ_ERR_ARG, "fz_plain_create: null argument");
  *out = nullptr;
  fz_status r;
  fzp::Base* b = nullptr;
  if (fp64) {
    auto* e = new fzp::Engine<double>();
    r = e->create(sys, device);
    b = e;
  } else {
    auto* e = new fzp::Engine<float>();
    r = e->create(sys, device);
    b = e;
  }
  if (r) {
    delete b;
    return r;
  }
  *out = new fz_plain{b};
  return FZ_OK;
}

extern "C" fz_status fz_plain_free(fz_plain* p) {
  if (!p) return FZ_OK;
  delete p->impl;
  delete p;
  return FZ_OK;
}

#define FZP_CHECK(p) \
  if (!(p) || !(p)->impl) return fail(FZ_ERR_ARG, "fenzi_plain: null handle")

extern "C" fz_status fz_plain_set_positions(fz_plain* p, const double* in3n) {
  FZP_CHECK(p);
  if (!in3n) return fail(FZ_ERR_ARG, "fz_plain_set_positions: null array");
  return p->impl->set_state(in3n, nullptr);
}
extern "C" fz_status fz_plain_set_velocities(fz_plain* p, const double* in3n) {
  FZP_CHECK(p);
  if (!in3n) return fail(FZ_ERR_ARG, "fz_plain_set_velocities: null array");
  return p->impl->set_state(nullptr, in3n);
}
extern "C" fz_status fz_plain_get_positions(fz_plain* p, double* out3n) {
  FZP_CHECK(p);
  if (!out3n) return fail(FZ_ERR_ARG, "fz_plain_get_positions: null array");
  return p->impl->get_state(out3n, nullptr);
}
extern "C" fz_status fz_plain_get_velocities(fz_plain* p, double* out3n) {
  FZP_CHECK(p);
  if (!out3n) return fail(FZ_ERR_ARG, "fz_plain_get_velocities: null array");
  return p->impl->get_state(nullptr, out3n);
}
extern "C" fz_status fz_plain_compute_forces(fz_plain* p, double* out3n) {
  FZP_CHECK(p);
  return p->impl->compute_forces(out3n);
}
extern "C" fz_status fz_plain_step(fz_plain* p, int nsteps) {
  FZP_CHECK(p);
  return p->impl->step(nsteps);
}
extern "C" fz_status fz_plain_eval_props(fz_plain* p, fz_energies* out) {
  FZP_CHECK(p);
  if (!out) return fail(FZ_ERR_ARG, "fz_plain_eval_props: null output");
  return p->impl->eval(out);
}
extern "C" fz_status fz_plain_get_counters(fz_plain* p, long long* out4) {
  FZP_CHECK(p);
  if (!out4) return fail(FZ_ERR_ARG, "fz_plain_get_counters: null output");
  return p->impl->counters(out4);
}
