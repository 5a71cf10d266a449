// PME reciprocal forces with no device allocation.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside another
// framework's memory pool or a pre-sized arena, or a host program that must not grow
// device memory after start-up.  fz_pme_reciprocal_static() serves them: it runs the
// same spread / R2C-FFT + influence function / C2R / gather kernels as the system
// path, but every scratch buffer lives in the fixed-size file-scope __device__ arrays
// below (about 4.4 MB on every GPU that loads the library, held until the process
// exits).  The caller passes its own device input (float4 x, y, z, q per atom) and
// output (int64 fixed-point forces) buffers.  The per-call tables (twiddles, B-spline
// moduli times the Gaussian, |m|^2) are computed on the device into the scratch, so a
// call copies nothing from host memory; only energy_out reads a value back.
//
// Set-up: the first call on a device, with that device current, resolves the device
// addresses of the scratch arrays with cudaGetSymbolAddress and caches them per
// device; make that first call before any stream capture.  The caller's current device
// is restored before every return.  All calls share the same
// scratch, which keeps the last call's contents: each call clears what must start at
// zero, and calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on the scratch and must be serialised by the caller.
#include <cmath>
#include <mutex>
#include <string>

#include "host/host.h"
#include "kernels/kernels.h"

namespace fz {
namespace {

constexpr int kSMaxAtoms = 262144;  // atoms per call
constexpr int kSMaxK = 64;          // grid points per dimension
constexpr int kSMaxBricks = 22 * 22 * 22;
constexpr int kSMaxDev = 64;

__device__ __align__(256) float s_grid[kSMaxK * kSMaxK * kSMaxK];
__device__ __align__(256) float2 s_cgrid[kSMaxK * kSMaxK * (kSMaxK / 2 + 1)];
__device__ __align__(256) int s_brick_of[kSMaxAtoms];
__device__ __align__(256) int s_brick_atoms[kSMaxAtoms];
__device__ __align__(256) int s_brick_count[kSMaxBricks];
__device__ __align__(256) int s_brick_cursor[kSMaxBricks];
__device__ __align__(256) int s_brick_start[kSMaxBricks + 1];
__device__ __align__(256) float2 s_tw[3][kSMaxK];
__device__ __align__(256) float s_gfac[3][kSMaxK];
__device__ __align__(256) float s_f2[3][kSMaxK];
__device__ __align__(256) long long s_energy[fzk::EN_COUNT];

struct Scratch {
  float* grid;
  float2* cgrid;
  int *brick_of, *brick_atoms, *brick_count, *brick_cursor, *brick_start;
  float2* tw;
  float *gfac, *f2;
  long long* energy;
};

Scratch g_scratch[kSMaxDev];
bool g_ready[kSMaxDev];
std::mutex g_mu;

fz_status setup(int device, Scratch** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ready[device]) {
    Scratch& s = g_scratch[device];
    cudaError_t e = cudaSuccess;
    float2* tw = nullptr;
    float *gf = nullptr, *f2 = nullptr;
    if ((e = cudaGetSymbolAddress((void**)&s.grid, s_grid)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.cgrid, s_cgrid)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.brick_of, s_brick_of)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.brick_atoms, s_brick_atoms)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.brick_count, s_brick_count)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.brick_cursor, s_brick_cursor)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.brick_start, s_brick_start)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&tw, s_tw)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&gf, s_gfac)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&f2, s_f2)) != cudaSuccess ||
        (e = cudaGetSymbolAddress((void**)&s.energy, s_energy)) != cudaSuccess)
      return fail(FZ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    s.tw = tw;
    s.gfac = gf;
    s.f2 = f2;
    g_ready[device] = true;
  }
  *out = &g_scratch[device];
  return FZ_OK;
}

bool fft_friendly(int n) {
  if (n < 4) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

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

// Per-call tables in FP64, rounded once to FP32, with the same expressions as the system
// path's host tables: twiddles e^{-2 pi i m/K}, f^2 = (m'/L)^2 and
// |b(m)|^2 exp(-pi^2 f^2 / beta^2) (order-4 Euler exponential-spline moduli); also clears
// the energy slots.  One block per dimension, one thread per grid index.
__global__ void k_static_tables(int K0, int K1, int K2, double L0, double L1, double L2, double beta) {
  const int d = blockIdx.x;
  const int Kd = d == 0 ? K0 : (d == 1 ? K1 : K2);
  const double L = d == 0 ? L0 : (d == 1 ? L1 : L2);
  if (d == 0)
    for (int k = threadIdx.x; k < fzk::EN_COUNT; k += blockDim.x) s_energy[k] = 0;
  const double b2 = beta * beta;
  for (int m = threadIdx.x; m < Kd; m += blockDim.x) {
    const double ang = -2.0 * M_PI * m / Kd;
    s_tw[d][m] = make_float2((float)cos(ang), (float)sin(ang));
    const double f = (m <= Kd / 2 ? m : m - Kd) / L;
    s_f2[d][m] = (float)(f * f);
    const double M4v[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
    double re = 0, im = 0;
    for (int k = 0; k < 3; ++k) {
      const double a = 2.0 * M_PI * (double)m * k / Kd;
      re += M4v[k] * cos(a);
      im += M4v[k] * sin(a);
    }
    s_gfac[d][m] = (float)((1.0 / (re * re + im * im)) * exp(-M_PI * M_PI * f * f / b2));
  }
}

// restores the caller's current device when the entry point returns
struct DeviceGuard {
  int prev = -1;
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace fz

using namespace fz;

extern "C" fz_status fz_pme_reciprocal_static(int device, void* stream, const float* pos4, int n, const double* box,
                                              const int* K, double beta, long long* facc, double* energy_out) {
  if (!pos4 || !facc || !box || !K) return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: null argument");
  if (device < 0 || device >= kSMaxDev) return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: bad device");
  if (n <= 0 || n > kSMaxAtoms)
    return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: atom count must be in 1.." + std::to_string(kSMaxAtoms));
  for (int d = 0; d < 3; ++d) {
    if (K[d] > kSMaxK || !fft_friendly(K[d]))
      return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: grid sizes must be 2^a 3^b 5^c in 4.." +
                                  std::to_string(kSMaxK));
    if (!(box[d] > 0)) return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: box edges must be positive");
  }
  if (!(beta > 0)) return fail(FZ_ERR_ARG, "fz_pme_reciprocal_static: beta must be positive");
  DeviceGuard guard;
  cudaError_t ce = cudaGetDevice(&guard.prev);
  if (ce != cudaSuccess) return fail(FZ_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
  if ((ce = cudaSetDevice(device)) != cudaSuccess)
    return fail(FZ_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));
  Scratch* s = nullptr;
  fz_status r = setup(device, &s);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  k_static_tables<<<3, 64, 0, st>>>(K[0], K[1], K[2], box[0], box[1], box[2], beta);
  if ((ce = cudaGetLastError()) != cudaSuccess ||
      (ce = cudaMemsetAsync(facc, 0, sizeof(long long) * 3 * (size_t)n, st)) != cudaSuccess)
    return fail(FZ_ERR_CUDA, std::string("fz_pme_reciprocal_static: ") + cudaGetErrorString(ce));
  fzk::PmeArgs a{};
  a.p.box = make_float3((float)box[0], (float)box[1], (float)box[2]);
  a.p.inv_box = make_float3((float)(1.0 / box[0]), (float)(1.0 / box[1]), (float)(1.0 / box[2]));
  a.p.beta = (float)beta;
  a.p.n = n;
  a.pos4 = reinterpret_cast<const float4*>(pos4);
  a.n = n;
  for (int d = 0; d < 3; ++d) {
    a.K[d] = K[d];
    a.B[d] = brick_edge(K[d]);
    a.nb[d] = K[d] / a.B[d];
    a.p.K[d] = K[d];
    a.tw[d] = s->tw + d * kSMaxK;
    a.gfac[d] = s->gfac + d * kSMaxK;
    a.f2[d] = s->f2 + d * kSMaxK;
  }
  a.brick_of = s->brick_of;
  a.brick_count = s->brick_count;
  a.brick_cursor = s->brick_cursor;
  a.brick_start = s->brick_start;
  a.brick_atoms = s->brick_atoms;
  a.grid = s->grid;
  a.cgrid = s->cgrid;
  a.gscale = (float)(kCC / (M_PI * box[0] * box[1] * box[2]));
  a.facc = facc;
  a.energy = s->energy;
  a.status = nullptr;  // the PME kernels report no status
  fzk::launch_pme(a, energy_out != nullptr, st);
  if ((ce = cudaGetLastError()) != cudaSuccess)
    return fail(FZ_ERR_CUDA, std::string("fz_pme_reciprocal_static launch: ") + cudaGetErrorString(ce));
  if (energy_out) {
    long long e = 0;
    if ((ce = cudaMemcpyAsync(&e, s->energy + fzk::EN_PME, sizeof(e), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(st)) != cudaSuccess)
      return fail(FZ_ERR_CUDA, std::string("fz_pme_reciprocal_static: ") + cudaGetErrorString(ce));
    *energy_out = (double)e / fzk::kFixE;
  }
  return FZ_OK;
}
