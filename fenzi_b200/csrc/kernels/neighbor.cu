// Device-side neighbour maintenance: replaces CellBuild/CellUpdate/CellClean and
// nbbuild_exclbitvec/nbbuild_excllist (src/cell_based_kernels.cu:198-399, 1048-1493)
// and the host-synchronised rebuild decision of SingleStep (src/dynamics.cu:695-737).
//
// Layout: atoms are binned into x-y columns of ~32/rho^(2/3) cross-section, each
// column is sorted by (z, atom id) and padded to a multiple of 32 slots, so every
// 32-slot "block" is a compact cell of ~32 atoms.  A tile is (i-block, 32 j-slots);
// j-slots are individual atoms within the pair-list radius of the i-block's bounding
// box, drawn from blocks J >= I (Newton's third law), each tagged with its periodic
// image.  Every kernel first reads the device rebuild flag and returns when no
// rebuild is due, so the sequence is launched unconditionally (graph friendly) and
// no host synchronisation is needed.
#include "common.cuh"
#include "kernels.h"

namespace fzk {

// wrap positions into [-L/2, L/2), record build positions, bin into columns
__device__ __forceinline__ void rb_bin_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag = A.flag;
  float4* pos4 = A.pos4;
  float4* pos_build = A.pos_build;
  int* col_of = A.col_of;
  int* col_count = A.col_count;
  int* status = A.status;

  if (!*flag) return;
  const int a = bid * blockDim.x + threadIdx.x;
  if (a >= p.n) return;
  float4 r = pos4[a];
  if (!(fabsf(r.x) < 1e7f && fabsf(r.y) < 1e7f && fabsf(r.z) < 1e7f)) {
    atomicOr(status, ST_BAD_COORD);
    r.x = r.y = r.z = 0.f;
  }
  r.x -= p.box.x * floorf((r.x + 0.5f * p.box.x) * p.inv_box.x);
  r.y -= p.box.y * floorf((r.y + 0.5f * p.box.y) * p.inv_box.y);
  r.z -= p.box.z * floorf((r.z + 0.5f * p.box.z) * p.inv_box.z);
  // guard the rounding edge x == L/2
  if (r.x >= 0.5f * p.box.x) r.x -= p.box.x;
  if (r.y >= 0.5f * p.box.y) r.y -= p.box.y;
  if (r.z >= 0.5f * p.box.z) r.z -= p.box.z;
  pos4[a] = r;
  pos_build[a] = r;
  int cx = (int)((r.x + 0.5f * p.box.x) * p.inv_box.x * p.ncol[0]);
  int cy = (int)((r.y + 0.5f * p.box.y) * p.inv_box.y * p.ncol[1]);
  cx = min(max(cx, 0), p.ncol[0] - 1);
  cy = min(max(cy, 0), p.ncol[1] - 1);
  const int c = cy * p.ncol[0] + cx;
  col_of[a] = c;
  const unsigned peers = __match_any_sync(__activemask(), c);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&col_count[c], __popc(peers));
}

__global__ void k_rb_bin(RebuildArgs a) { griddep_wait(); rb_bin_body(a, blockIdx.x, gridDim.x); }
__global__ void k_rb_bin_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_bin_body(a, t.y, t.z);
}


// exclusive scan of the 32-padded column sizes (one block)
__device__ __forceinline__ void rb_scan_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag = A.flag;
  const int* __restrict__ col_count = A.col_count;
  int* col_start = A.col_start;
  const int ncol = A.p.ncol[0] * A.p.ncol[1];
  int* counters = A.counters;
  int* status = A.status;

  if (!*flag) return;
  __shared__ int part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (ncol + nt - 1) / nt;
  const int b = t * per, e = min(ncol, b + per);
  int s = 0;
  for (int c = b; c < e; ++c) s += (col_count[c] + 31) & ~31;
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - s;
  for (int c = b; c < e; ++c) {
    col_start[c] = run;
    run += (col_count[c] + 31) & ~31;
  }
  if (t == nt - 1) {
    const int used = part[t];
    // the last 32 slots are reserved for the permanent dummy block
    if (used > p.nslots - 32) atomicOr(status, ST_SLOT_OVERFLOW);
    counters[CNT_SLOTS] = min(used, p.nslots - 32);
    col_start[ncol] = min(used, p.nslots - 32);
  }
}

__global__ void k_rb_scan(RebuildArgs a) { griddep_wait(); rb_scan_body(a, blockIdx.x, gridDim.x); }
__global__ void k_rb_scan_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_scan_body(a, t.y, t.z);
}


__device__ __forceinline__ void rb_scatter_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag = A.flag;
  const int* __restrict__ col_of = A.col_of;
  const int* __restrict__ col_start = A.col_start;
  int* col_cursor = A.col_cursor;
  int* col_tmp = A.col_tmp;

  if (!*flag) return;
  const int a = bid * blockDim.x + threadIdx.x;
  if (a >= p.n) return;
  const int c = col_of[a];
  const unsigned peers = __match_any_sync(__activemask(), c);
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if ((threadIdx.x & 31) == leader) base = atomicAdd(&col_cursor[c], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  const int k = base + __popc(peers & ((1u << (threadIdx.x & 31)) - 1u));
  const int s = col_start[c] + k;
  if (s < p.nslots - 32) col_tmp[s] = a;
}

__global__ void k_rb_scatter(RebuildArgs a) { griddep_wait(); rb_scatter_body(a, blockIdx.x, gridDim.x); }
__global__ void k_rb_scatter_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_scatter_body(a, t.y, t.z);
}


__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// one block per column: bitonic sort by (z, atom id), then fill the sorted arrays
__device__ __forceinline__ void rb_colsort_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag = A.flag;
  int* col_count = A.col_count;
  int* col_cursor = A.col_cursor;
  const int* __restrict__ col_start = A.col_start;
  const int* __restrict__ col_tmp = A.col_tmp;
  const float4* __restrict__ pos4 = A.pos4;
  const int* __restrict__ type = A.type;
  int* perm = A.perm;
  int* inv_perm = A.inv_perm;
  float4* xyzq_s = A.xyzq_s;
  int* typ_s = A.typ_s;
  int* blk_col = A.blk_col;
  int* status = A.status;

  if (!*flag) return;
  extern __shared__ unsigned long long keys[];
  const int c = bid;
  const int n = col_count[c];
  const int start = col_start[c];
  // the column's count and cursor are spent: zero them for the next rebuild's binning
  __syncthreads();
  if (threadIdx.x == 0) {
    col_count[c] = 0;
    col_cursor[c] = 0;
  }
  const int padded = (n + 31) & ~31;
  if (start + padded > p.nslots - 32) return;  // slot overflow already flagged
  if (n > kColCap) {
    if (threadIdx.x == 0) atomicOr(status, ST_COLUMN_OVERFLOW);
    return;
  }
  int m = 1;
  while (m < n) m <<= 1;
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    if (k < n) {
      const int a = col_tmp[start + k];
      keys[k] = ((unsigned long long)float_key(pos4[a].z) << 32) | (unsigned)a;
    } else {
      keys[k] = ~0ull;
    }
  }
  __syncthreads();
  for (int size = 2; size <= m; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int o = k ^ stride;
        if (o > k) {
          const bool up = (k & size) == 0;
          const unsigned long long x = keys[k], y = keys[o];
          if ((x > y) == up) {
            keys[k] = y;
            keys[o] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int k = threadIdx.x * 32; k < padded; k += 32 * blockDim.x) blk_col[(start + k) >> 5] = c;
  for (int k = threadIdx.x; k < padded; k += blockDim.x) {
    const int s = start + k;
    if (k < n) {
      const int a = (int)(keys[k] & 0xffffffffu);
      perm[s] = a;
      inv_perm[a] = s;
      xyzq_s[s] = pos4[a];
      typ_s[s] = type[a];
    } else {
      perm[s] = -1;
      // distinct far-away point, q = 0, padding LJ type: never within any cutoff
      xyzq_s[s] = make_float4(1.0e6f + (float)s, 1.0e6f, 1.0e6f, 0.f);
      typ_s[s] = p.ntypes;
    }
  }
}

__global__ void __launch_bounds__(256) k_rb_colsort(RebuildArgs a) { griddep_wait(); rb_colsort_body(a, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) k_rb_colsort_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_colsort_body(a, t.y, t.z);
}


// squared distance between two boxes given center offset d and half extents
__device__ __forceinline__ float box_gap2(float3 d, float3 h) {
  const float gx = fmaxf(0.f, fabsf(d.x) - h.x);
  const float gy = fmaxf(0.f, fabsf(d.y) - h.y);
  const float gz = fmaxf(0.f, fabsf(d.z) - h.z);
  return gx * gx + gy * gy + gz * gz;
}

// Outer pair list of i-block I: every atom of a block J >= I (Newton's third law), at
// every periodic image, whose position lies within rlist of block I's bounding box.
// The diagonal block (J == I, no image) is implicit and not stored.  Candidate j blocks
// are those of the columns within rlist in x-y (periodic column offsets carry the x/y
// image), each tested in z at its minimum image (or at all three z images for small
// boxes).  One warp walks column offsets it0 .. it1 - 1 (row-major over (oy, ox)) in
// order; with STORE it writes the entries from out[base + 0] on, else it only counts
// them.  Returns the number of entries met (stored or not).
template <bool STORE>
__device__ __forceinline__ int outer_scan(const RebuildArgs& A, int I, int it0, int it1, uint32_t* out, int base) {
  const SysParams& p = A.p;
  const int lane = threadIdx.x & 31;
  const float4 li = A.bb_lo[I], hi4 = A.bb_hi[I];
  const float3 ci = make_float3(0.5f * (li.x + hi4.x), 0.5f * (li.y + hi4.y), 0.5f * (li.z + hi4.z));
  const float3 hi = make_float3(0.5f * (hi4.x - li.x), 0.5f * (hi4.y - li.y), 0.5f * (hi4.z - li.z));
  const float rl2 = p.rlist * p.rlist;
  const int cI = A.blk_col[I];
  const int cx = cI % p.ncol[0], cy = cI / p.ncol[0];
  const int nz = A.all_images ? 3 : 1;
  const int nox = 2 * A.dcx + 1;
  int count = 0;
  for (int it = it0; it < it1; ++it) {
    const int oy = it / nox - A.dcy, ox = it % nox - A.dcx;
    int yy = cy + oy;
    const int sy = yy < 0 ? -1 : (yy >= p.ncol[1] ? 1 : 0);
    yy -= sy * p.ncol[1];
    int xx = cx + ox;
    const int sx = xx < 0 ? -1 : (xx >= p.ncol[0] ? 1 : 0);
    xx -= sx * p.ncol[0];
    const int col = yy * p.ncol[0] + xx;
    const int b0 = A.col_start[col] >> 5, b1 = A.col_start[col + 1] >> 5;
    for (int J0 = b0; J0 < b1; J0 += 32) {
      const int J = J0 + lane;
      const bool inr = J < b1 && J >= I;
      float3 cj = make_float3(0.f, 0.f, 0.f), hj = cj;
      if (inr) {
        const float4 lj = A.bb_lo[J], hj4 = A.bb_hi[J];
        cj = make_float3(0.5f * (lj.x + hj4.x), 0.5f * (lj.y + hj4.y), 0.5f * (lj.z + hj4.z));
        hj = make_float3(0.5f * (hj4.x - lj.x), 0.5f * (hj4.y - lj.y), 0.5f * (hj4.z - lj.z));
      }
      for (int iz = 0; iz < nz; ++iz) {
        bool pass = false;
        int code = kNoShift;
        if (inr) {
          float3 d = make_float3(cj.x - ci.x + sx * p.box.x, cj.y - ci.y + sy * p.box.y, cj.z - ci.z);
          const float sz = A.all_images ? (float)(iz - 1) : -rintf(d.z * p.inv_box.z);
          d.z += sz * p.box.z;
          code = (sx + 1) + 3 * (sy + 1) + 9 * ((int)sz + 1);
          pass = box_gap2(d, make_float3(hi.x + hj.x, hi.y + hj.y, hi.z + hj.z)) < rl2;
          // the self block: its diagonal is implicit, each +-image pair is taken once
          if (J == I && code >= kNoShift) pass = false;
        }
        unsigned bal = __ballot_sync(0xffffffffu, pass);
        while (bal) {
          const int src = __ffs(bal) - 1;
          bal &= bal - 1;
          const int Jc = J0 + src;
          const int cc = __shfl_sync(0xffffffffu, code, src);
          const int s = Jc * 32 + lane;
          const float3 sh = shift_of(cc, p);
          const float4 r = A.xyzq_s[s];
          const float3 d = make_float3(r.x + sh.x - ci.x, r.y + sh.y - ci.y, r.z + sh.z - ci.z);
          const bool ok = A.perm[s] >= 0 && box_gap2(d, hi) < rl2;
          const unsigned b2 = __ballot_sync(0xffffffffu, ok);
          const int pos = base + count + __popc(b2 & ((1u << lane) - 1u));
          if (STORE && ok && pos < A.ocap) {
            // flag entries whose atom has an excluded partner in block I: only those
            // need the prune's exclusion-mask walk (the partner walk only when I lies
            // in the range of the partners' blocks, which for most entries it does not)
            uint32_t fl = 0u;
            const int2 xr = A.xrange[s];
            if (I >= xr.x && I <= xr.y) {
              const int m = A.xn[s];
              for (int k = 0; k < m; ++k)
                if ((A.xs[(size_t)s * A.xmax + k] >> 5) == I) fl = kExclBit;
            }
            out[pos] = (uint32_t)s | fl | ((uint32_t)cc << kSlotBits);
          }
          count += __popc(b2);
        }
      }
    }
  }
  return count;
}

// warp per i-block; entries append to the block's own region outer[I * ocap ...] in a
// fixed order (deterministic)
__device__ __forceinline__ void rb_outer_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  if (!*A.flag) return;
  const int nblk = A.counters[CNT_SLOTS] >> 5;
  const int lane = threadIdx.x & 31;
  const int I = bid * 8 + (threadIdx.x >> 5);
  if (I >= nblk) return;
  const int nit = (2 * A.dcy + 1) * (2 * A.dcx + 1);
  const int count = outer_scan<true>(A, I, 0, nit, A.outer + (size_t)I * A.ocap, 0);
  if (lane == 0) {
    A.outer_n[I] = min(count, A.ocap);
    if (count > A.ocap) atomicOr(A.status, ST_TILE_OVERFLOW);
  }
}

// The same list with one CTA of kOuterWarps warps per i-block, for systems with too few
// blocks to fill the GPU with a warp per block: the column offsets are cut into
// contiguous runs, one per warp; each warp counts its run's entries, then stores them
// after those of the runs before it, so the list is entry for entry the one above.
constexpr int kOuterWarps = 8;

__device__ __forceinline__ void rb_outer_split_body(const RebuildArgs& A, int I) {
  griddep_wait();
  if (!*A.flag) return;
  const int nblk = A.counters[CNT_SLOTS] >> 5;
  if (I >= nblk) return;
  __shared__ int wcount[kOuterWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nit = (2 * A.dcy + 1) * (2 * A.dcx + 1);
  const int it0 = (warp * nit) / kOuterWarps, it1 = ((warp + 1) * nit) / kOuterWarps;
  const int mine = outer_scan<false>(A, I, it0, it1, nullptr, 0);
  if (lane == 0) wcount[warp] = mine;
  __syncthreads();
  int base = 0, total = 0;
  for (int w = 0; w < kOuterWarps; ++w) {
    base += w < warp ? wcount[w] : 0;
    total += wcount[w];
  }
  outer_scan<true>(A, I, it0, it1, A.outer + (size_t)I * A.ocap, base);
  if (threadIdx.x == 0) {
    A.outer_n[I] = min(total, A.ocap);
    if (total > A.ocap) atomicOr(A.status, ST_TILE_OVERFLOW);
  }
}

__global__ void __launch_bounds__(kOuterWarps * 32) k_rb_outer_split(RebuildArgs a) {
  griddep_wait();
  rb_outer_split_body(a, blockIdx.x);
}

__global__ void __launch_bounds__(256) k_rb_outer(RebuildArgs a) { griddep_wait(); rb_outer_body(a, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) k_rb_outer_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_outer_body(a, t.y, t.z);
}


// Per slot: the partner slots of its excluded atoms (1-2, 1-3, 1-4), for the prune's
// masks; per 32-slot block (one warp): the bounding box of its atoms
__device__ __forceinline__ void rb_slots_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag = A.flag;
  const int* __restrict__ counters = A.counters;
  const int* __restrict__ perm = A.perm;
  const int* __restrict__ inv_perm = A.inv_perm;
  const int* __restrict__ excl_off = A.excl_off;
  const int* __restrict__ excl_idx = A.excl_idx;
  int* xn = A.xn;
  int* xs = A.xs;
  int xmax = A.xmax;
  const float4* __restrict__ xyzq_s = A.xyzq_s;
  float4* bb_lo = A.bb_lo;
  float4* bb_hi = A.bb_hi;

  if (!*flag) return;
  const int sl = bid * blockDim.x + threadIdx.x;
  if (sl >= p.nslots) return;  // nslots is a multiple of 32: whole warps leave together
  const int a = perm[sl];
  int m = 0, blo = 0x7fffffff, bhi = -1;
  if (a >= 0) {
    const int e0 = excl_off[a];
    m = min(excl_off[a + 1] - e0, xmax);
    for (int k = 0; k < m; ++k) {
      const int ps = inv_perm[excl_idx[e0 + k]];
      xs[(size_t)sl * xmax + k] = ps;
      blo = min(blo, ps >> 5);
      bhi = max(bhi, ps >> 5);
    }
  }
  xn[sl] = m;
  A.xrange[sl] = make_int2(blo, bhi);
  const int w = sl >> 5, lane = sl & 31;
  if (w >= (counters[CNT_SLOTS] >> 5)) return;  // uniform per warp
  const bool ok = a >= 0;
  const float4 r = xyzq_s[sl];
  float lx = ok ? r.x : 3e38f, ly = ok ? r.y : 3e38f, lz = ok ? r.z : 3e38f;
  float hx = ok ? r.x : -3e38f, hy = ok ? r.y : -3e38f, hz = ok ? r.z : -3e38f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
    ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
    lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
    hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
    hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
    hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
  }
  if (lane == 0) {
    bb_lo[w] = make_float4(lx, ly, lz, 0.f);
    bb_hi[w] = make_float4(hx, hy, hz, 0.f);
  }
}

__global__ void k_rb_slots(RebuildArgs a) { griddep_wait(); rb_slots_body(a, blockIdx.x, gridDim.x); }
__global__ void k_rb_slots_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  rb_slots_body(a, t.y, t.z);
}


// Closes a rebuild (counts it, lowers its flag, raises the prune flag: a new outer list
// always gets a fresh inner list) and opens a prune (zeroes the list counters).
__device__ __forceinline__ void prune_begin_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  int* flag = A.flag;
  int* flag_prune = A.flag_prune;
  int* counters = A.counters;

  if (*flag) {
    counters[CNT_REBUILDS] += 1;
    *flag = 0;
    *flag_prune = 1;
  }
  if (!*flag_prune) return;
  counters[CNT_MASKS] = 0;
  counters[CNT_TILES] = 0;
  counters[CNT_ITEMS] = 0;
}

__global__ void k_prune_begin(RebuildArgs a) { griddep_wait(); prune_begin_body(a, blockIdx.x, gridDim.x); }
__global__ void k_prune_begin_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  prune_begin_body(a, t.y, t.z);
}


// Exclusion masks of one tile (this lane holding j entry je): the lane walks the
// excluded partners (1-2, 1-3, 1-4) of its own j slot (xs/xn: partner slots per slot,
// written at every rebuild) and, for each partner sitting in i-block I, sets bit
// `lane` in that partner's i-lane mask in shared memory.  The exclusion lists are
// symmetric, so i-lane l ends with bit k set exactly when j entry k is an excluded
// partner of i atom l; images are not distinguished (the box is at least twice the
// pair-list radius).
__device__ __forceinline__ uint32_t excl_mask(int I, uint32_t je, int lane, uint32_t* msk,
                                              const int* __restrict__ xn, const int* __restrict__ xs, int xmax) {
  msk[lane] = 0u;
  __syncwarp();
  const int sj = (int)(je & kSlotMask);
  const int m = xn[sj];
  for (int k = 0; k < m; ++k) {
    const int sp = xs[(size_t)sj * xmax + k];
    if ((sp >> 5) == I) atomicOr(&msk[sp & 31], 1u << lane);
  }
  __syncwarp();
  const uint32_t r = msk[lane];
  __syncwarp();
  return r;
}

// The prune's distance tests in packed form: the block's 32 i atoms are held in pairs
// (2p, 2p + 1), A[p] = (ax, ax', ay, ay') and B[p] = (az, az', aw, aw') with
// a = (-2 (q - o), |q - o|^2), so one f32x2 FMA chain tests an entry against two i
// atoms at once.  Each test is the scalar fma(ax, rx, fma(ay, ry, fma(az, rz, aw))) in
// the same order, and the minimum does not depend on the order taken, so the kept
// entries are exactly those of one test per atom.
__device__ __forceinline__ void prune_store_i(float4* iA, float4* iB, int lane, float ax, float ay, float az,
                                              float aw) {
  float* a = reinterpret_cast<float*>(iA) + (lane >> 1) * 4 + (lane & 1);
  float* b = reinterpret_cast<float*>(iB) + (lane >> 1) * 4 + (lane & 1);
  a[0] = ax;
  a[2] = ay;
  b[0] = az;
  b[2] = aw;
}
// minimum expanded distance of an entry (r relative to o) to the atoms of i-group g
__device__ __forceinline__ float prune_min_group(const float4* iA, const float4* iB, float2 x2, float2 y2, float2 z2,
                                                 int g) {
  float m = 3e38f;
#pragma unroll
  for (int p = 0; p < kIG / 2; ++p) {
    const float4 A = iA[g * (kIG / 2) + p], B = iB[g * (kIG / 2) + p];
    float2 d = __ffma2_rn(make_float2(B.x, B.y), z2, make_float2(B.z, B.w));
    d = __ffma2_rn(make_float2(A.z, A.w), y2, d);
    d = __ffma2_rn(make_float2(A.x, A.y), x2, d);
    m = fminf(m, fminf(d.x, d.y));
  }
  return m;
}

// Bounding box of each i-group's atoms relative to o, from every lane's own i atom q
// (padding slots left out: a group of padding only gets a negative extent, which no
// entry reaches), written by lane 0 of the warp to box[g * 6 ...] = centre, half extent.
__device__ __forceinline__ void group_boxes(float qx, float qy, float qz, bool real, float* box) {
  float lo[3] = {real ? qx : 3e38f, real ? qy : 3e38f, real ? qz : 3e38f};
  float hi[3] = {real ? qx : -3e38f, real ? qy : -3e38f, real ? qz : -3e38f};
#pragma unroll
  for (int off = kIG / 2; off > 0; off >>= 1)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], off));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], off));
    }
  const int lane = threadIdx.x & 31;
  if (lane % kIG == 0)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      box[(lane / kIG) * 6 + d] = 0.5f * (lo[d] + hi[d]);
      box[(lane / kIG) * 6 + 3 + d] = 0.5f * (hi[d] - lo[d]);
    }
}

// The distance tests of one chunk of 32 entries (r relative to o).  With SKIP, a
// group's tests are skipped by the whole warp when no entry of the chunk comes within
// the keep radius of the group's bounding box (plus 0.05 A^2, far above the rounding of
// either form), so the kept entries are exactly those of the full test.  Measured (us
// per MD step): the CTA-per-block prune of small systems gains (17,280 atoms 74.0 ->
// 70.2), the warp-per-block prune of large ones loses (230,400 atoms 414 -> 420), so
// only the former skips.
template <bool SKIP>
__device__ __forceinline__ void prune_min2(const float4* iA, const float4* iB, float rx, float ry, float rz,
                                           bool valid, float rp2_keep, const float* box, float* m2) {
  const float2 x2 = make_float2(rx, rx), y2 = make_float2(ry, ry), z2 = make_float2(rz, rz);
#pragma unroll
  for (int g = 0; g < kNG; ++g) {
    if (!SKIP) {
      m2[g] = prune_min_group(iA, iB, x2, y2, z2, g);
      continue;
    }
    const float* b = box + g * 6;
    const float bx = fmaxf(0.f, fabsf(rx - b[0]) - b[3]);
    const float by = fmaxf(0.f, fabsf(ry - b[1]) - b[4]);
    const float bz = fmaxf(0.f, fabsf(rz - b[2]) - b[5]);
    const bool near = valid && fmaf(bx, bx, fmaf(by, by, bz * bz)) <= rp2_keep + 0.05f;
    m2[g] = __any_sync(0xffffffffu, near) ? prune_min_group(iA, iB, x2, y2, z2, g) : 3e38f;
  }
}

// Inner (pruned) pair list, warp per i-block: keeps the outer entries that lie within
// rc + delta of at least one atom of the block at the current positions, packs them
// into full 32-entry tiles with their exclusion masks, and records the positions the
// list was made at.  Run after every rebuild and whenever an atom has moved more than
// delta/2 since the last prune, so no pair within rc is ever missed.
__device__ __forceinline__ void prune_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  const SysParams p = A.p;
  const int* __restrict__ flag_prune = A.flag_prune;
  int* counters = A.counters;
  const int* __restrict__ perm = A.perm;
  const int* __restrict__ xn = A.xn;
  const float4* __restrict__ xyzq_s = A.xyzq_s;
  const int* __restrict__ xs = A.xs;
  int xmax = A.xmax;
  const uint32_t* __restrict__ outer = A.outer;
  const int* __restrict__ outer_n = A.outer_n;
  uint32_t* inner = A.inner;
  int* inner_nt = A.inner_nt;
  int* inner_m = A.inner_m;
  uint32_t* masks = A.masks;
  uint32_t* dmask = A.dmask;
  int mask_cap = A.mask_cap;
  int ocap = A.ocap;
  float rp2 = A.rp2;
  float4* pos_prune = A.pos_prune;
  int2* items = A.items;
  int chunk = A.chunk;
  int* status = A.status;

  if (!*flag_prune) return;
  __shared__ float4 iA_all[8][16], iB_all[8][16];
  __shared__ uint32_t buf_all[8][kNG][64];
  __shared__ uint32_t msk_all[8][32];
  const int nblk = counters[CNT_SLOTS] >> 5;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = bid * 8 + warp;
  if (I >= nblk) return;
  float4* iA = iA_all[warp];
  float4* iB = iB_all[warp];
  uint32_t* msk = msk_all[warp];
  const int islot = I * 32 + lane;
  const float4 pi = xyzq_s[islot];
  const int ia = perm[islot];
  if (ia >= 0) pos_prune[ia] = pi;
  // distances are taken about the block's first atom o (slot 0 of a block is always
  // an atom): |r - q|^2 = |r - o|^2 + (|q - o|^2 - 2 (q - o).(r - o)), so each (i, j)
  // test is three FMAs and a min on (-2(q - o), |q - o|^2) held in shared memory
  const float4 o = xyzq_s[I * 32];
  {
    const float qx = pi.x - o.x, qy = pi.y - o.y, qz = pi.z - o.z;
    prune_store_i(iA, iB, lane, -2.f * qx, -2.f * qy, -2.f * qz, fmaf(qx, qx, fmaf(qy, qy, qz * qz)));
  }
  // diagonal tile mask (exclusions inside the block)
  dmask[islot] = excl_mask(I, (uint32_t)islot, lane, msk, xn, xs, xmax);
  const uint32_t dummy = (uint32_t)(p.nslots - 1) | ((uint32_t)kNoShift << kSlotBits);
  const int n = outer_n[I];
  const uint32_t* src = outer + (size_t)I * ocap;
  int count[kNG], ntile[kNG];
#pragma unroll
  for (int s = 0; s < kNG; ++s) count[s] = ntile[s] = 0;
  // one full 32-entry tile of i-group s: entries, and its exclusion words (one per i
  // atom of the group) when any pair is excluded
  auto emit = [&](int s) {
    uint32_t* buf = buf_all[warp][s];
    const int g = I * kNG + s;
    const uint32_t je = buf[lane];
    inner[(size_t)g * ocap + ntile[s] * 32 + lane] = je;
    uint32_t w = 0u;
    if (__ballot_sync(0xffffffffu, (je & kExclBit) != 0u)) {
      excl_mask(I, (je & kExclBit) ? je : dummy, lane, msk, xn, xs, xmax);
      w = lane < kIG ? msk[s * kIG + lane] : 0u;
    }
    int m = -1;
    if (__ballot_sync(0xffffffffu, w != 0)) {
      if (lane == 0) m = atomicAdd(&counters[CNT_MASKS], 1);
      m = __shfl_sync(0xffffffffu, m, 0);
      if (m >= mask_cap) {
        if (lane == 0) atomicOr(status, ST_MASK_OVERFLOW);
        m = -1;
      } else if (lane < kIG) {
        masks[(size_t)m * kIG + lane] = w;
      }
    }
    if (lane == 0) inner_m[(size_t)g * (ocap >> 5) + ntile[s]] = m;
    ++ntile[s];
    __syncwarp();
  };
  // the next chunk's entries and positions are loaded before this chunk's distance
  // tests, so the gathers overlap the arithmetic
  const float rp2_keep = rp2 + 1e-3f;
  uint32_t e_nx = lane < n ? src[lane] : dummy;
  float4 r_nx = xyzq_s[e_nx & kSlotMask];
  for (int c0 = 0; c0 < n; c0 += 32) {
    const bool valid = c0 + lane < n;
    const uint32_t e = e_nx;
    float4 r = r_nx;
    if (c0 + 32 < n) {
      e_nx = c0 + 32 + lane < n ? src[c0 + 32 + lane] : dummy;
      r_nx = xyzq_s[e_nx & kSlotMask];
    }
    const int code = (int)(e >> kSlotBits);
    if (code != kNoShift) {
      const float3 sh = shift_of(code, p);
      r.x += sh.x;
      r.y += sh.y;
      r.z += sh.z;
    }
    r.x -= o.x;
    r.y -= o.y;
    r.z -= o.z;
    const float rr = fmaf(r.x, r.x, fmaf(r.y, r.y, r.z * r.z));
    float m2[kNG];
#pragma unroll
    for (int s = 0; s < kNG; ++s) m2[s] = 3e38f;
    prune_min2<false>(iA, iB, r.x, r.y, r.z, valid, rp2_keep, nullptr, m2);
#pragma unroll
    for (int s = 0; s < kNG; ++s) {
      uint32_t* buf = buf_all[warp][s];
      // rp2_keep exceeds (rc + delta)^2 by far more than the rounding of the expanded
      // form (|r - o| <= ~20 A), so no entry the exact test keeps is dropped
      const bool keep = valid && m2[s] + rr < rp2_keep;
      const unsigned b = __ballot_sync(0xffffffffu, keep);
      if (keep) buf[count[s] + __popc(b & ((1u << lane) - 1u))] = e;
      __syncwarp();
      count[s] += __popc(b);
      if (count[s] >= 32) {
        emit(s);
        const uint32_t rest = buf[32 + lane];
        __syncwarp();
        buf[lane] = rest;
        __syncwarp();
        count[s] -= 32;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < kNG; ++s) {
    if (count[s] > 0) {
      uint32_t* buf = buf_all[warp][s];
      if (lane >= count[s]) buf[lane] = dummy;
      __syncwarp();
      emit(s);
    }
  }
  // work items for the pair kernel, per i-group: chunks of <= `chunk` tiles (tile 0
  // is the group against its own block, upper triangle)
#pragma unroll
  for (int s = 0; s < kNG; ++s) {
    const int g = I * kNG + s;
    const int nitems = (ntile[s] + 1 + chunk - 1) / chunk;
    int base = 0;
    if (lane == 0) {
      inner_nt[g] = ntile[s];
      atomicAdd(&counters[CNT_TILES], ntile[s] + 1);
      base = atomicAdd(&counters[CNT_ITEMS], nitems);
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    for (int k = lane; k < nitems; k += 32) items[base + k] = make_int2(g, k * chunk);
  }
}

__global__ void __launch_bounds__(256, 4) k_prune(RebuildArgs a) { griddep_wait(); prune_body(a, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256, 6) k_prune_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  prune_body(a, t.y, t.z);
}


// The same prune with one CTA of kPruneWarps warps per i-block, for systems with too
// few blocks to fill the GPU with a warp per block (a 9,000-atom box has ~290 blocks:
// ~36 CTAs of the kernel above).  The block's outer entries are cut into contiguous
// runs of whole 32-entry chunks, one run per warp; each warp keeps its entries for
// each i-group (the same distance test) and stores them compacted at its run's start
// in shared memory; the kept lists are then read in warp order, which is the outer
// list's order, so the inner tiles, their exclusion masks and the work items are
// identical to the warp-per-block prune's: the forces are bit-identical either way.
constexpr int kPruneWarps = 8;

__device__ __forceinline__ void prune_split_body(const RebuildArgs& A, int I) {
  griddep_wait();
  const SysParams p = A.p;
  if (!*A.flag_prune) return;
  const int nblk = A.counters[CNT_SLOTS] >> 5;
  if (I >= nblk) return;
  extern __shared__ uint32_t kept[];  // [kNG][ocap]
  __shared__ float4 iA[16], iB[16];
  __shared__ float box[kNG * 6];
  __shared__ uint32_t msk_all[kPruneWarps][32];
  __shared__ int cnt[kPruneWarps][kNG];
  __shared__ int off[kPruneWarps + 1][kNG];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* msk = msk_all[warp];
  const int ocap = A.ocap;
  const int islot = I * 32 + lane;
  const float4 o = A.xyzq_s[I * 32];
  if (warp == 0) {
    const float4 pi = A.xyzq_s[islot];
    const int ia = A.perm[islot];
    if (ia >= 0) A.pos_prune[ia] = pi;
    const float qx = pi.x - o.x, qy = pi.y - o.y, qz = pi.z - o.z;
    prune_store_i(iA, iB, lane, -2.f * qx, -2.f * qy, -2.f * qz, fmaf(qx, qx, fmaf(qy, qy, qz * qz)));
    group_boxes(qx, qy, qz, ia >= 0, box);
    A.dmask[islot] = excl_mask(I, (uint32_t)islot, lane, msk, A.xn, A.xs, A.xmax);
  }
  __syncthreads();
  const uint32_t dummy = (uint32_t)(p.nslots - 1) | ((uint32_t)kNoShift << kSlotBits);
  const int n = A.outer_n[I];
  const uint32_t* src = A.outer + (size_t)I * ocap;
  const int nch = (n + 31) >> 5;
  const int c_begin = (warp * nch) / kPruneWarps, c_end = ((warp + 1) * nch) / kPruneWarps;
  const float rp2_keep = A.rp2 + 1e-3f;
  int count[kNG];
#pragma unroll
  for (int s = 0; s < kNG; ++s) count[s] = 0;
  for (int c = c_begin; c < c_end; ++c) {
    const int e_i = c * 32 + lane;
    const bool valid = e_i < n;
    const uint32_t e = valid ? src[e_i] : dummy;
    float4 r = A.xyzq_s[e & kSlotMask];
    const int code = (int)(e >> kSlotBits);
    if (code != kNoShift) {
      const float3 sh = shift_of(code, p);
      r.x += sh.x;
      r.y += sh.y;
      r.z += sh.z;
    }
    r.x -= o.x;
    r.y -= o.y;
    r.z -= o.z;
    const float rr = fmaf(r.x, r.x, fmaf(r.y, r.y, r.z * r.z));
    float m2[kNG];
#pragma unroll
    for (int s = 0; s < kNG; ++s) m2[s] = 3e38f;
    prune_min2<true>(iA, iB, r.x, r.y, r.z, valid, rp2_keep, box, m2);
#pragma unroll
    for (int s = 0; s < kNG; ++s) {
      const bool keep = valid && m2[s] + rr < rp2_keep;
      const unsigned b = __ballot_sync(0xffffffffu, keep);
      if (keep) kept[s * ocap + c_begin * 32 + count[s] + __popc(b & ((1u << lane) - 1u))] = e;
      count[s] += __popc(b);
    }
  }
  if (lane == 0)
    for (int s = 0; s < kNG; ++s) cnt[warp][s] = count[s];
  __syncthreads();
  if (threadIdx.x < kNG) {
    const int s = threadIdx.x;
    int run = 0;
    for (int w = 0; w < kPruneWarps; ++w) {
      off[w][s] = run;
      run += cnt[w][s];
    }
    off[kPruneWarps][s] = run;
  }
  __syncthreads();
  // tiles: dense entry d of group s is entry d - off[w][s] of warp w's kept run
  for (int s = 0; s < kNG; ++s) {
    const int g = I * kNG + s;
    const int total = off[kPruneWarps][s];
    const int ntile = (total + 31) >> 5;
    for (int t = warp; t < ntile; t += kPruneWarps) {
      const int d = t * 32 + lane;
      uint32_t je = dummy;
      if (d < total) {
        int w = 0;
        while (w + 1 < kPruneWarps && off[w + 1][s] <= d) ++w;
        const int cb = (w * nch) / kPruneWarps;
        je = kept[s * ocap + cb * 32 + (d - off[w][s])];
      }
      A.inner[(size_t)g * ocap + t * 32 + lane] = je;
      uint32_t wd = 0u;
      if (__ballot_sync(0xffffffffu, (je & kExclBit) != 0u)) {
        excl_mask(I, (je & kExclBit) ? je : dummy, lane, msk, A.xn, A.xs, A.xmax);
        wd = lane < kIG ? msk[s * kIG + lane] : 0u;
      }
      int m = -1;
      if (__ballot_sync(0xffffffffu, wd != 0)) {
        if (lane == 0) m = atomicAdd(&A.counters[CNT_MASKS], 1);
        m = __shfl_sync(0xffffffffu, m, 0);
        if (m >= A.mask_cap) {
          if (lane == 0) atomicOr(A.status, ST_MASK_OVERFLOW);
          m = -1;
        } else if (lane < kIG) {
          A.masks[(size_t)m * kIG + lane] = wd;
        }
      }
      if (lane == 0) A.inner_m[(size_t)g * (ocap >> 5) + t] = m;
      __syncwarp();
    }
    if (warp == 0) {
      const int nitems = (ntile + 1 + A.chunk - 1) / A.chunk;
      int base = 0;
      if (lane == 0) {
        A.inner_nt[g] = ntile;
        atomicAdd(&A.counters[CNT_TILES], ntile + 1);
        base = atomicAdd(&A.counters[CNT_ITEMS], nitems);
      }
      base = __shfl_sync(0xffffffffu, base, 0);
      for (int k = lane; k < nitems; k += 32) A.items[base + k] = make_int2(g, k * A.chunk);
    }
  }
}

__global__ void __launch_bounds__(kPruneWarps * 32) k_prune_split(RebuildArgs a) {
  griddep_wait();
  prune_split_body(a, blockIdx.x);
}

__device__ __forceinline__ void prune_end_body(const RebuildArgs& A, int bid, int nbid) {
  griddep_wait();
  int* flag_prune = A.flag_prune;
  int* counters = A.counters;

  counters[CNT_WORK] = 0;  // the pair kernel's item counter (it always follows)
  if (!*flag_prune) return;
  counters[CNT_PRUNES] += 1;
  *flag_prune = 0;
}

__global__ void k_prune_end(RebuildArgs a) { griddep_wait(); prune_end_body(a, blockIdx.x, gridDim.x); }
__global__ void k_prune_end_b(const RebuildArgs* __restrict__ args, const int4* __restrict__ tab) { griddep_wait();
  const int4 t = tab[blockIdx.x];
  const RebuildArgs a = args[t.x];
  prune_end_body(a, t.y, t.z);
}


// sets a graph conditional node's value from a device flag (the neighbour kernels run
// inside an IF node only when their flag is raised)
__global__ void k_set_condition(cudaGraphConditionalHandle h, const int* __restrict__ flag,
                                const int* __restrict__ flag2) { griddep_wait();
  cudaGraphSetConditional(h, (*flag != 0 || (flag2 && *flag2 != 0)) ? 1u : 0u);
}

// ------------------------------------------------------------------ launchers
void launch_set_condition(cudaGraphConditionalHandle h, const int* flag, const int* flag2, cudaStream_t st) {
  k_set_condition<<<1, 1, 0, st>>>(h, flag, flag2);
}

void launch_rebuild(const RebuildArgs& a, cudaStream_t st) {
  launch_rebuild_build(a, st);
  launch_rebuild_prune(a, st);
}

void launch_rebuild_build(const RebuildArgs& a, cudaStream_t st) {
  const SysParams& p = a.p;
  const int ncol = p.ncol[0] * p.ncol[1];
  const int maxblk = (p.nslots) / 32;
  launch_pdl(k_rb_bin, dim3((p.n + 255) / 256), dim3(256), 0, st, a);
  launch_pdl(k_rb_scan, dim3(1), dim3(1024), 0, st, a);
  launch_pdl(k_rb_scatter, dim3((p.n + 255) / 256), dim3(256), 0, st, a);
  launch_pdl(k_rb_colsort, dim3(ncol), dim3(256), kColCap * sizeof(unsigned long long), st, a);
  launch_pdl(k_rb_slots, dim3((p.nslots + 255) / 256), dim3(256), 0, st, a);
  if (a.outer_split)
    launch_pdl(k_rb_outer_split, dim3(maxblk), dim3(kOuterWarps * 32), 0, st, a);
  else
    launch_pdl(k_rb_outer, dim3((maxblk + 7) / 8), dim3(256), 0, st, a);
}

void launch_rebuild_prune(const RebuildArgs& a, cudaStream_t st) {
  const SysParams& p = a.p;
  const int maxblk = (p.nslots) / 32;
  launch_pdl(k_prune_begin, dim3(1), dim3(1), 0, st, a);
  if (a.prune_split) {
    const size_t smem = (size_t)kNG * a.ocap * sizeof(uint32_t);
    launch_pdl(k_prune_split, dim3(maxblk), dim3(kPruneWarps * 32), smem, st, a);
  } else {
    launch_pdl(k_prune, dim3((maxblk + 7) / 8), dim3(256), 0, st, a);
  }
  launch_pdl(k_prune_end, dim3(1), dim3(1), 0, st, a);
}

// (sets the kernel's dynamic shared-memory limit on the current device)
bool prune_split_fits(int ocap) {
  const size_t smem = (size_t)kNG * ocap * sizeof(uint32_t);
  if (cudaFuncSetAttribute(k_prune_split, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return smem <= 160 * 1024;
}

// ------------------------------------------------------------------ batched launchers
// One launch per kernel over many systems: block b of the launch runs block t.y (of
// t.z) of system t.x, t = tab[b]; the per-system grids are those of the launchers above.
void rebuild_grids(const RebuildArgs& a, int* g6) {
  const SysParams& p = a.p;
  const int maxblk = p.nslots / 32;
  g6[0] = (p.n + 255) / 256;          // bin, scatter
  g6[1] = p.ncol[0] * p.ncol[1];      // colsort
  g6[2] = (p.nslots + 255) / 256;     // slots
  g6[3] = (maxblk + 7) / 8;           // outer, prune
}

void launch_rebuild_build_b(const RebuildArgs* args, const BatchTables& t, cudaStream_t st) {
  launch_pdl(k_rb_bin_b, dim3(t.n[BT_ATOMS256]), dim3(256), 0, st, args, t.tab[BT_ATOMS256]);
  launch_pdl(k_rb_scan_b, dim3(t.n[BT_ONE]), dim3(1024), 0, st, args, t.tab[BT_ONE]);
  launch_pdl(k_rb_scatter_b, dim3(t.n[BT_ATOMS256]), dim3(256), 0, st, args, t.tab[BT_ATOMS256]);
  launch_pdl(k_rb_colsort_b, dim3(t.n[BT_COLUMNS]), dim3(256), kColCap * sizeof(unsigned long long), st, args, t.tab[BT_COLUMNS]);
  launch_pdl(k_rb_slots_b, dim3(t.n[BT_SLOTS256]), dim3(256), 0, st, args, t.tab[BT_SLOTS256]);
  launch_pdl(k_rb_outer_b, dim3(t.n[BT_BLOCKS8]), dim3(256), 0, st, args, t.tab[BT_BLOCKS8]);
}

void launch_rebuild_prune_b(const RebuildArgs* args, const BatchTables& t, cudaStream_t st) {
  launch_pdl(k_prune_begin_b, dim3(t.n[BT_ONE]), dim3(1), 0, st, args, t.tab[BT_ONE]);
  launch_pdl(k_prune_b, dim3(t.n[BT_BLOCKS8]), dim3(256), 0, st, args, t.tab[BT_BLOCKS8]);
  launch_pdl(k_prune_end_b, dim3(t.n[BT_ONE]), dim3(1), 0, st, args, t.tab[BT_ONE]);
}

}  // namespace fzk
