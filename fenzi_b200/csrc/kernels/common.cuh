// Shared device definitions for the sm_100a MD step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace fzk {

// AKMA constants (src/defs.in.h:156-158)
constexpr double kCC = 332.0716;
constexpr double kTU = 20.4548;
constexpr double kRC = 0.001987;
constexpr double kPi = 3.14159265358979323846;

// fixed-point scales: forces 2^32 per kcal/mol/A, energies 2^30 per kcal/mol
constexpr float kFixF = 4294967296.0f;
constexpr double kFixFd = 4294967296.0;
constexpr double kFixE = 1073741824.0;
constexpr double kFixQ = 1099511627776.0;  // PME charge grid, 2^40

// device status word bits (sticky, read by the host at chunk boundaries)
enum : int {
  ST_TILE_OVERFLOW = 1,
  ST_MASK_OVERFLOW = 2,
  ST_SLOT_OVERFLOW = 4,
  ST_COLUMN_OVERFLOW = 8,
  ST_SHAKE_NOCONV = 16,
  ST_BRICK_OVERFLOW = 32,
  ST_BAD_COORD = 64,
};

// energy slots (same order as fz_energies)
enum : int {
  EN_BOND = 0, EN_ANGLE, EN_UREYB, EN_DIHED, EN_IMPR, EN_VDW, EN_ELEC, EN_PME, EN_EWEXCL, EN_EWSELF,
  EN_KIN, EN_VIR_X, EN_VIR_Y, EN_VIR_Z,
  EN_KIN_HALF,  // half-step kinetic energy of a barostat step
  EN_COUNT = 16
};

// tile-list j entry: bits 0..26 slot, bits 27..31 periodic image code (0..26, 13 = none)
constexpr int kSlotBits = 27;
// pair-list granularity: each 32-slot block is split into kNG i-groups of kIG atoms;
// every i-group has its own pruned list of 32-entry j tiles (a tile is kIG x 32 pairs).
// Measured at 230,400 atoms (ms/step): kIG 32 0.655 (35 % of pair slots within rc),
// 16 0.632 (43 %), 8 0.642 (49 %, but a pruned list per 8 atoms and one j-force
// atomic flush per 256 pairs cost more than the pairs saved).
constexpr int kIG = 16;
constexpr int kNG = 32 / kIG;
constexpr uint32_t kSlotMask = (1u << 26) - 1u;  // bits 0..25: slot
constexpr uint32_t kExclBit = 1u << 26;          // bit 26: the j atom has an excluded partner in the i block
constexpr int kNoShift = 13;

// per-system parameters passed by value
struct SysParams {
  float3 box;        // edge lengths
  float3 inv_box;
  float rc2, ron2;   // cutoff^2, switch-on^2
  float sw_c3;       // 1/(rc2-ron2)^3
  float beta;
  float cc;          // Coulomb constant (float)
  float skin_half2;  // (0.5*(pairlist - cutoff))^2, rebuild trigger
  float rlist;       // pair-list radius
  int n;             // atoms
  int ntypes;        // LJ types (+1 padding type at index ntypes)
  int nslots;        // sorted slot capacity (multiple of 32)
  int ncol[2];       // column grid (x, y)
  int K[3];          // PME grid
};

// Programmatic dependent launch (sm_90+): a kernel launched with launch_pdl may be set
// up while its predecessor in the stream still runs; it waits here, before touching any
// memory, until the predecessor has completed and its writes are visible, so the stream
// order is kept and only the launch latency is hidden.  Every kernel that can be
// launched with launch_pdl calls this first.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class... P, class... A>
inline void launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

__device__ __forceinline__ long long to_fix(float f) { return __float2ll_rn(f * kFixF); }
__device__ __forceinline__ long long to_fix_d(double f) { return __double2ll_rn(f * kFixFd); }

__device__ __forceinline__ void red_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// FP64 warp sum (fixed butterfly order: deterministic)
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// adds a per-thread FP64 energy into a fixed-point slot, one atomic per warp
__device__ __forceinline__ void energy_add(long long* slot, double e) {
  e = warp_sum_d(e);
  if ((threadIdx.x & 31) == 0 && e != 0.0) red_add(slot, __double2ll_rn(e * kFixE));
}

// adds per-thread fixed-point values into a slot, one atomic per warp (exact)
__device__ __forceinline__ void energy_add_fix(long long* slot, long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0) red_add(slot, v);
}

__device__ __forceinline__ float3 min_image(float3 d, const SysParams& p) {
  d.x -= p.box.x * rintf(d.x * p.inv_box.x);
  d.y -= p.box.y * rintf(d.y * p.inv_box.y);
  d.z -= p.box.z * rintf(d.z * p.inv_box.z);
  return d;
}

__device__ __forceinline__ void min_image_d(double* d, const SysParams& p) {
  d[0] -= (double)p.box.x * rint(d[0] / (double)p.box.x);
  d[1] -= (double)p.box.y * rint(d[1] / (double)p.box.y);
  d[2] -= (double)p.box.z * rint(d[2] / (double)p.box.z);
}

// periodic image code -> shift vector (code = (sx+1) + 3 (sy+1) + 9 (sz+1))
__device__ __forceinline__ float3 shift_of(int code, const SysParams& p) {
  const int sx = code % 3 - 1, sy = (code / 3) % 3 - 1, sz = code / 9 - 1;
  return make_float3(sx * p.box.x, sy * p.box.y, sz * p.box.z);
}

}  // namespace fzk
