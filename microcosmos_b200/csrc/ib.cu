// Immersed-boundary coupling (src/microcosmos/solver/fluid.py:202-386) and the
// deterministic scatter-add machinery it shares with the steric cloud-in-cell deposit
// (src/microcosmos/forces.py:98-115).
//
// Scatter-adds are never done with float atomics.  Each contribution k (IB: k = n*K*K + s,
// CIC: k = corner*N + n — the order in which the reference's scatters apply them) is
// appended to the bin of its 16x16-cell tile with its cell's position in the tile packed
// above it (an integer atomic picks the slot; a full bin spills to an overflow list).  One CTA per tile then counting-sorts the bin by cell,
// orders each cell's run by k and sums it sequentially — the reference's in-order
// scatter-add, bit-reproducibly.  The IB iterations work on the compact list of touched
// cells ("heads") instead of full (H, W) grids.
#include "lbm_cell.cuh"

namespace mc {

struct BinView {
  const int* cell;
  const float* w;
  int* store;
  int* tcount;
  int* ovf;
  int* ctl;
  int cap;
  int count;
  int gw;      // width of the grid the cells index (lattice for IB, domain grid for CIC)
  int ntx;     // bin tiles per row of that grid
  int ntiles;  // bin tiles of that grid
};

__device__ __forceinline__ BinView bin_view(const RDesc& d, int which) {
  BinView v;
  if (which == 0) {
    v.cell = d.ib_cell; v.w = d.ib_w; v.store = d.ib_store; v.tcount = d.ib_tcount; v.ovf = d.ib_ovf;
    v.ctl = d.ib_ctl; v.cap = d.ib_cap; v.count = d.M;
    v.gw = d.lW; v.ntx = d.lntile_x; v.ntiles = d.lntile_x * d.lntile_y;
  } else {
    v.cell = d.c_cell; v.w = d.c_w; v.store = d.c_store; v.tcount = d.c_tcount; v.ovf = d.c_ovf;
    v.ctl = d.c_ctl; v.cap = d.c_cap; v.count = d.enable_steric ? 4 * d.N : 0;
    v.gw = d.W; v.ntx = d.ntile_x; v.ntiles = d.ntile_x * d.ntile_y;
  }
  return v;
}

__device__ __forceinline__ int tile_of(const BinView& v, int cell) {
  const int cy = cell / v.gw, cx = cell - cy * v.gw;
  return (cy / kBinTile) * v.ntx + cx / kBinTile;
}
__device__ __forceinline__ unsigned local_of(const BinView& v, int cell) {
  const int cy = cell / v.gw, cx = cell - cy * v.gw;
  return (unsigned)((cy % kBinTile) * kBinTile + (cx % kBinTile));
}

__device__ void bitonic_sort_smem(unsigned* s, int P) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
}

__device__ __forceinline__ int lower_bound_u(const unsigned* a, int len, unsigned key) {
  int lo = 0, hi = len;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Per-cell reduction work.  IB: coverage -> 1/max(cov, 1), the macroscopic state pulled
// from h[parity] (density, clamped velocity), u_corrected = velocity (fluid.py:268-290);
// the caller has already linked the run's contributions to `slot`.
__device__ __forceinline__ void ib_head(const RDesc& d, int parity, int cell, float cov, int slot, int len,
                                        int run_pos) {
  d.h_cell[slot] = cell;
  d.h_start[slot] = run_pos;
  d.h_len[slot] = len;
  d.s_inv[slot] = 1.0f / max_prop(cov, 1.0f);
  const int y = cell / d.lW, x = cell - y * d.lW;
  const size_t HW = (size_t)d.lH * d.lW;
  const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
  const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  float f[9];
  const float* hp = d.h[parity];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int ys = imod_floor(y - ey[q], d.lH), xs = imod_floor(x - ex[q], d.lW);
    f[q] = hp[q * HW + (size_t)ys * d.lW + xs];
  }
  float rho, vx, vy;
  macroscopic(f, d.vmax, d.vmax_q4, rho, vx, vy);
  d.s_rho[slot] = rho;
  d.s_vx[slot] = vx;
  d.s_vy[slot] = vy;
  d.s_ucx[slot] = vx;
  d.s_ucy[slot] = vy;
}

// Work for one touched cell whose contributions are run[0..len) in increasing k, read
// from global memory (spilled tiles only).  CIC: deposit = in-order sum (forces.py:98-115).
__device__ __forceinline__ void head_work(const RDesc& d, const BinView& v, int which, int parity, const int* run,
                                          int len, int run_pos) {
  const int k0 = run[0];
  const int cell = v.cell[k0];
  float acc = v.w[k0];
  for (int j = 1; j < len; ++j) acc = acc + v.w[run[j]];
  if (which == 1) {
    d.dep[cell] = acc;
    return;
  }
  const int slot = atomicAdd(v.ctl + 2, 1);
  for (int j = 0; j < len; ++j) d.ib_slot[run[j]] = slot;
  ib_head(d, parity, cell, acc, slot, len, run_pos);
}

// One CTA on one bin tile: sort the tile's contributions by (cell, k) and reduce every
// touched cell's run.  Tiles of at most capS contributions are sorted in shared memory;
// larger ones take the global-arena path.  skeys: dynamic shared memory of 4 * capS words, capS <= the
// bin capacity of every rollout of the launch (a power of two).
__device__ __forceinline__ int pc(int c) { return c + (c >> 3); }

__device__ void tile_work(const RDesc& d, int which, int parity, int t, unsigned* skeys, int capS) {
  const int kCapS = capS;
  const int kChunk = 4 * capS;  // keys per shared-memory chunk sort on the spill path
  // per-cell counters at padded slots pc(c) = c + c / 8: the scan below gives each lane 8
  // consecutive cells, and the padding puts the lanes' slots on distinct banks
  __shared__ int cnt[kBinTile * kBinTile + kBinTile * kBinTile / 8];
  __shared__ int cpos[kBinTile * kBinTile + kBinTile * kBinTile / 8];
  __shared__ int hpos[kBinTile * kBinTile + kBinTile * kBinTile / 8];  // rank of a touched cell among the tile's
  __shared__ int tlist[kBinTile * kBinTile];  // the touched cells, by rank
  __shared__ int s_spill, s_heads, s_base, s_fill;
  const BinView v = bin_view(d, which);
  if (v.count == 0) return;
  const int total = v.tcount[t];
  if (total == 0) return;
  const int tid = threadIdx.x;
  const int ntiles = v.ntiles;
  int* bin = v.store + (size_t)t * v.cap;

  // fast path: the whole tile sorted in shared memory (capacity capS <= the bin capacity)
  if (total <= min(v.cap, kCapS)) {
    // shared layout: [0, C) packed (cell, rank) | [C, 2C) k | [2C, 3C) sorted k | [3C, 4C) sorted w
    unsigned* lr = skeys;
    int* kin = reinterpret_cast<int*>(skeys + kCapS);
    int* kout = reinterpret_cast<int*>(skeys + 2 * kCapS);
    float* wout = reinterpret_cast<float*>(skeys + 3 * kCapS);
    for (int c = tid; c < kBinTile * kBinTile; c += blockDim.x) cnt[pc(c)] = 0;
    if (tid == 0) s_heads = 0;
    __syncthreads();
    // counting sort by local cell; positions inside a cell come from shared atomics
    // (arbitrary order), so each cell's run is then ordered by k
    for (int i = tid; i < total; i += blockDim.x) {
      const unsigned e = (unsigned)bin[i];  // (local cell << 24) | k
      const unsigned lc = e >> 24;
      const int k = (int)(e & 0xffffffu);
      const int pos = atomicAdd(cnt + pc(lc), 1);
      lr[i] = (lc << 24) | (unsigned)pos;
      kin[i] = k;
    }
    __syncthreads();
    // exclusive scan of the 256 cell counts (one warp, 8 per lane) and the head count
    if (tid < 32) {
      int loc[8];
      int sum = 0, nz = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        loc[q] = cnt[tid * 9 + q];  // pc(tid * 8 + q)
        sum += loc[q];
        nz += loc[q] > 0;
      }
      int incl = sum, inz = nz;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        int z = __shfl_up_sync(0xffffffffu, inz, o);
        if (tid >= o) {
          incl += y;
          inz += z;
        }
      }
      int run = incl - sum, hrun = inz - nz;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        cpos[tid * 9 + q] = run;
        hpos[tid * 9 + q] = hrun;
        run += loc[q];
        hrun += loc[q] > 0;
      }
      if (tid == 31) s_heads = inz;
    }
    __syncthreads();
    // one slot range per tile for its touched cells (IB); the touched cells listed by rank
    if (which == 0 && tid == 0) s_base = atomicAdd(v.ctl + 2, s_heads);
    for (int c = tid; c < kBinTile * kBinTile; c += blockDim.x)
      if (cnt[pc(c)] > 0) tlist[hpos[pc(c)]] = c;
    for (int i = tid; i < total; i += blockDim.x) {
      const unsigned key = lr[i];
      const int lc = (int)(key >> 24), pos = (int)(key & 0xffffffu);
      const int k = kin[i];
      kout[cpos[pc(lc)] + pos] = k;
      wout[cpos[pc(lc)] + pos] = v.w[k];
    }
    __syncthreads();
    // one thread per touched cell: order its run by k (runs are short), then reduce it
    const int nheads = s_heads;
    for (int hi = tid; hi < nheads; hi += blockDim.x) {
      const int c = tlist[hi];
      const int len = cnt[pc(c)];
      int* rk = kout + cpos[pc(c)];
      float* rw = wout + cpos[pc(c)];
      for (int a = 1; a < len; ++a) {
        const int key = rk[a];
        const float kw = rw[a];
        int b = a - 1;
        while (b >= 0 && rk[b] > key) {
          rk[b + 1] = rk[b];
          rw[b + 1] = rw[b];
          --b;
        }
        rk[b + 1] = key;
        rw[b + 1] = kw;
      }
      float acc = rw[0];
      for (int j = 1; j < len; ++j) acc = acc + rw[j];
      const int cell = v.cell[rk[0]];
      if (which == 1) {
        d.dep[cell] = acc;
      } else {
        const int slot = s_base + hpos[pc(c)];
        for (int j = 0; j < len; ++j) d.ib_slot[rk[j]] = slot;
        ib_head(d, parity, cell, acc, slot, len, t * v.cap + cpos[pc(c)]);
      }
    }
    __syncthreads();
    if (which == 0) {
      // runs for the spread: contributing node and weight, contiguous per touched cell
      const int K2 = d.K * d.K;
      float* binw = d.ib_store_w + (size_t)t * v.cap;
      for (int i = tid; i < total; i += blockDim.x) {
        bin[i] = kout[i] / K2;
        binw[i] = wout[i];
      }
    }
    if (tid == 0) v.tcount[t] = 0;
    return;
  }

  // Spilled tile: gather its bin and its overflow entries into a private arena region,
  // sort by (cell, k) with shared-memory chunk sorts and rank merges, then reduce.
  if (tid == 0) s_spill = atomicAdd(v.ctl + 1, 2 * total);
  __syncthreads();
  const int base = ntiles * v.cap + s_spill;
  unsigned* bufA = reinterpret_cast<unsigned*>(v.store) + base;
  unsigned* bufB = bufA + total;
  const int nbin = min(total, v.cap);
  for (int i = tid; i < nbin; i += blockDim.x) bufB[i] = (unsigned)bin[i];  // already (local << 24) | k
  if (tid == 0) s_fill = nbin;
  __syncthreads();
  if (total > v.cap) {
    // the overflow list is unordered: every thread scans a stride of it for this tile's
    // entries (their order is restored by the sort below)
    const int no = v.ctl[0];
    for (int i = tid; i < no; i += blockDim.x) {
      const int k = v.ovf[i];
      if (tile_of(v, v.cell[k]) == t) bufB[atomicAdd(&s_fill, 1)] = (local_of(v, v.cell[k]) << 24) | (unsigned)k;
    }
  }
  __syncthreads();
  const int m = total;
  for (int c0 = 0; c0 < m; c0 += kChunk) {
    const int len = min(kChunk, m - c0);
    int P = 1;
    while (P < len) P <<= 1;
    for (int i = tid; i < P; i += blockDim.x) skeys[i] = i < len ? bufB[c0 + i] : 0xffffffffu;
    __syncthreads();
    bitonic_sort_smem(skeys, P);
    for (int i = tid; i < len; i += blockDim.x) bufA[c0 + i] = skeys[i];
    __syncthreads();
  }
  unsigned* src = bufA;
  unsigned* dst = bufB;
  for (int wdt = kChunk; wdt < m; wdt <<= 1) {
    for (int i = tid; i < m; i += blockDim.x) {
      const int ps = (i / (2 * wdt)) * (2 * wdt);
      const int a_len = min(wdt, m - ps);
      const int b0 = ps + a_len;
      const int b_len = max(0, min(wdt, m - b0));
      const unsigned key = src[i];
      int pos;
      if (i < b0)
        pos = (i - ps) + lower_bound_u(src + b0, b_len, key);
      else
        pos = (i - b0) + lower_bound_u(src + ps, a_len, key);
      dst[ps + pos] = key;
    }
    __syncthreads();
    unsigned* tmp = src;
    src = dst;
    dst = tmp;
  }
  // runs are located on the sorted keys; their k values go to the other buffer
  const unsigned* keys = src;
  int* kv = reinterpret_cast<int*>(dst);
  for (int i = tid; i < m; i += blockDim.x) kv[i] = (int)(keys[i] & 0xffffffu);
  __syncthreads();
  const int kv_pos = base + (int)(reinterpret_cast<unsigned*>(kv) - bufA);
  for (int i = tid; i < m; i += blockDim.x) {
    const unsigned lc = keys[i] >> 24;
    if (i > 0 && (keys[i - 1] >> 24) == lc) continue;
    int len = 1;
    while (i + len < m && (keys[i + len] >> 24) == lc) ++len;
    head_work(d, v, which, parity, kv + i, len, kv_pos + i);
  }
  __syncthreads();
  if (which == 0) {
    const int K2 = d.K * d.K;
    for (int i = tid; i < m; i += blockDim.x) {
      const int k = kv[i];
      d.ib_store_w[kv_pos + i] = v.w[k];
      kv[i] = k / K2;
    }
  }
  if (tid == 0) v.tcount[t] = 0;
}

// The bin tiles that received contributions this step, listed by the producers as
// (rollout, tile) pairs (most tiles of a large or batched grid are empty and never
// listed).  A grid of as many CTAs as the GPU holds at once takes the listed tiles one at
// a time from a cursor (wl_count[2], reset with the list), so that no CTA is launched only
// to find nothing to do and uneven tiles balance across the CTAs.
__global__ void __launch_bounds__(256) k_bin_tiles(const RDesc* __restrict__ D, const int2* __restrict__ wl,
                                                   int* __restrict__ wl_count, int which, int parity, int capS) {
  extern __shared__ unsigned dyn[];
  __shared__ int s_item;
  const int count = *wl_count;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(wl_count + 2, 1);
    __syncthreads();
    const int i = s_item;
    if (i >= count) break;  // uniform across the CTA
    const int2 item = wl[i];
    tile_work(D[item.x], which, parity, item.y, dyn, capS);
    __syncthreads();  // the shared arrays and s_item are reused by the next item
  }
}

// Weighted sum of a head-indexed field over the K*K stencil of one node, in stencil order
// (the reference's sum over axis 1 of values * weights, fluid.py:90-97).
template <int K2>
__device__ __forceinline__ void stencil_sum(const RDesc& d, int node, const float* __restrict__ ax,
                                            const float* __restrict__ ay, float& sx, float& sy) {
  int slot[K2];
  float w[K2];
  const int base = node * K2;
  if (K2 % 4 == 0) {
#pragma unroll
    for (int s = 0; s < K2; s += 4) {
      const int4 q = *reinterpret_cast<const int4*>(d.ib_slot + base + s);
      const float4 v = *reinterpret_cast<const float4*>(d.ib_w + base + s);
      slot[s] = q.x; slot[s + 1] = q.y; slot[s + 2] = q.z; slot[s + 3] = q.w;
      w[s] = v.x; w[s + 1] = v.y; w[s + 2] = v.z; w[s + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int s = 0; s < K2; ++s) {
      slot[s] = d.ib_slot[base + s];
      w[s] = d.ib_w[base + s];
    }
  }
  float vx[K2], vy[K2];
#pragma unroll
  for (int s = 0; s < K2; ++s) {
    vx[s] = ax[slot[s]];
    vy[s] = ay[slot[s]];
  }
  float x = 0.0f, y = 0.0f;
#pragma unroll
  for (int s = 0; s < K2; ++s) {
    x = x + vx[s] * w[s];
    y = y + vy[s] * w[s];
  }
  sx = x;
  sy = y;
}

__device__ __forceinline__ void stencil_sum_any(const RDesc& d, int node, const float* __restrict__ ax,
                                                const float* __restrict__ ay, float& sx, float& sy) {
  switch (d.K) {
    case 4: stencil_sum<16>(d, node, ax, ay, sx, sy); return;
    case 2: stencil_sum<4>(d, node, ax, ay, sx, sy); return;
    case 3: stencil_sum<9>(d, node, ax, ay, sx, sy); return;
    default: break;
  }
  const int K2 = d.K * d.K;
  float x = 0.0f, y = 0.0f;
  for (int s = 0; s < K2; ++s) {
    const int k = node * K2 + s;
    const int p = d.ib_slot[k];
    const float w = d.ib_w[k];
    x = x + ax[p] * w;
    y = y + ay[p] * w;
  }
  sx = x;
  sy = y;
}

// Body force of touched cell p from its corrected velocity after the last multi-direct
// forcing round (fluid.py:327-339): post clamp of u_corrected, F = (u_c - u) rho, optional
// force clamp.
__device__ __forceinline__ void head_force(const RDesc& d, int p, float ucx, float ucy) {
  const float c2 = clamp_factor(ucx, ucy, d.vmax);
  ucx = ucx * c2;
  ucy = ucy * c2;
  const float rho = d.s_rho[p];
  float Fx = (ucx - d.s_vx[p]) * rho;
  float Fy = (ucy - d.s_vy[p]) * rho;
  if (d.force_clamp) {
    const float c3 = clamp_factor(Fx, Fy, d.vmax);
    Fx = Fx * c3;
    Fy = Fy * c3;
  }
  d.s_fx[p] = Fx;
  d.s_fy[p] = Fy;
}

// Multi-direct forcing, interpolation half (fluid.py:292-302): per IB point, u at the point
// = sum_s w_s u_corrected(cell_s); correction = (U_point - u) * relaxation, clamped.
__global__ void __launch_bounds__(256) k_ib_interp(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                   int it) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int node = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (node >= d.NI || it >= d.ib_iters) return;  // node = IB point
  float ux, uy;
  stencil_sum_any(d, node, d.s_ucx, d.s_ucy, ux, uy);
  const float sx = (d.nvl[2 * node] - ux) * d.relax;
  const float sy = (d.nvl[2 * node + 1] - uy) * d.relax;
  const float cf = clamp_factor(sx, sy, d.vmax);
  d.delta[2 * node] = sx * cf;
  d.delta[2 * node + 1] = sy * cf;
}

// Multi-direct forcing, spread half (fluid.py:304-310): per touched cell, the in-order sum
// of correction * weight over its contributions, times 1/max(coverage, 1), added to
// u_corrected.
__global__ void __launch_bounds__(256) k_ib_spread(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                   int it, int fuse_finalize) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  // the plan's last round also computes each touched cell's body force (k_ib_finalize's
  // work for the same cell) when every rollout of the plan runs the same number of rounds
  const bool fin = fuse_finalize && it == d.ib_iters - 1;
  if (fin && p == 0) d.ib_ctl[5] = d.ib_ctl[2];
  if (it >= d.ib_iters || p >= d.ib_ctl[2]) return;
  const int len = d.h_len[p];
  const int* rn = d.ib_store + d.h_start[p];      // contributing nodes, in k order
  const float* rw = d.ib_store_w + d.h_start[p];  // their weights
  float dx = 0.0f, dy = 0.0f;
  // runs are short: fetch 8 entries at a time (the last group predicated) so that all
  // their loads are in flight together; the sum keeps the run order
  for (int j = 0; j < len; j += 8) {
    int nd[8];
    float w[8], ex[8], ey[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const bool ok = j + q < len;
      nd[q] = ok ? rn[j + q] : 0;
      w[q] = ok ? rw[j + q] : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const bool ok = j + q < len;
      ex[q] = ok ? d.delta[2 * nd[q]] : 0.0f;
      ey[q] = ok ? d.delta[2 * nd[q] + 1] : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if (j + q < len) {
        dx = dx + ex[q] * w[q];
        dy = dy + ey[q] * w[q];
      }
    }
  }
  const float inv = d.s_inv[p];
  const float ucx = d.s_ucx[p] + dx * inv, ucy = d.s_ucy[p] + dy * inv;
  d.s_ucx[p] = ucx;
  d.s_ucy[p] = ucy;
  if (fin) head_force(d, p, ucx, ucy);
}

// ---------------------------------------------------------------- fused IB iterations
// Barrier among the CTAs of one rollout inside a cooperative launch (all CTAs resident).
// The spin is bounded: on timeout the rollout's MC_FLAG_TIMEOUT is set and the kernel
// continues (its results are then invalid) instead of hanging the device.
__device__ __forceinline__ void rollout_barrier(int* ctl, int nb, unsigned* flags) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* gen = ctl + 4;
    const int g = *gen;
    __threadfence();
    if (atomicAdd(ctl + 3, 1) == nb - 1) {
      atomicExch(ctl + 3, 0);
      __threadfence();
      atomicAdd(ctl + 4, 1);
    } else {
      unsigned it = 0;
      while (*gen == g) {
        if (++it > (1u << 22)) {
          atomicOr(flags, 2u);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// All ibm_iterations of the multi-direct forcing and the body force of every rollout in one
// cooperative launch: [interpolate (nodes) | barrier | spread (touched cells) | barrier] x
// iterations, then the finalize of every touched cell.  Same arithmetic and order as
// k_ib_interp / k_ib_spread / k_ib_finalize; values written in one phase and read in the
// next are loaded with __ldcg (L2, not the SM's L1).
// The shared body: threads t0, t0 + stride, ... of one rollout; `sync` is the barrier among
// all of the rollout's threads.
template <typename Sync>
__device__ __forceinline__ void ib_iterations(const RDesc& d, int t0, int stride, Sync sync) {
  const int nheads = __ldcg(d.ib_ctl + 2);
  const int K2 = d.K * d.K;
  for (int it = 0; it < d.ib_iters; ++it) {
    for (int node = t0; node < d.NI; node += stride) {  // IB points
      float ux = 0.0f, uy = 0.0f;
      const int base = node * K2;
      if (K2 == 16) {
        int slot[16];
        float w[16];
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
          const int4 a = *reinterpret_cast<const int4*>(d.ib_slot + base + q);
          const float4 b = *reinterpret_cast<const float4*>(d.ib_w + base + q);
          slot[q] = a.x; slot[q + 1] = a.y; slot[q + 2] = a.z; slot[q + 3] = a.w;
          w[q] = b.x; w[q + 1] = b.y; w[q + 2] = b.z; w[q + 3] = b.w;
        }
        float vx[16], vy[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          vx[q] = __ldcg(d.s_ucx + slot[q]);
          vy[q] = __ldcg(d.s_ucy + slot[q]);
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          ux = ux + vx[q] * w[q];
          uy = uy + vy[q] * w[q];
        }
      } else {
        for (int q = 0; q < K2; ++q) {
          const int sl = d.ib_slot[base + q];
          const float w = d.ib_w[base + q];
          ux = ux + __ldcg(d.s_ucx + sl) * w;
          uy = uy + __ldcg(d.s_ucy + sl) * w;
        }
      }
      const float sx = (d.nvl[2 * node] - ux) * d.relax;
      const float sy = (d.nvl[2 * node + 1] - uy) * d.relax;
      const float cf = clamp_factor(sx, sy, d.vmax);
      d.delta[2 * node] = sx * cf;
      d.delta[2 * node + 1] = sy * cf;
    }
    sync();
    for (int p = t0; p < nheads; p += stride) {
      const int len = d.h_len[p];
      const int* rn = d.ib_store + d.h_start[p];
      const float* rw = d.ib_store_w + d.h_start[p];
      float dx = 0.0f, dy = 0.0f;
      int j = 0;
      for (; j + 8 <= len; j += 8) {
        int nd[8];
        float w[8], ex[8], ey[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          nd[q] = rn[j + q];
          w[q] = rw[j + q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          ex[q] = __ldcg(d.delta + 2 * nd[q]);
          ey[q] = __ldcg(d.delta + 2 * nd[q] + 1);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          dx = dx + ex[q] * w[q];
          dy = dy + ey[q] * w[q];
        }
      }
      for (; j < len; ++j) {
        const int node = rn[j];
        const float w = rw[j];
        dx = dx + __ldcg(d.delta + 2 * node) * w;
        dy = dy + __ldcg(d.delta + 2 * node + 1) * w;
      }
      const float inv = d.s_inv[p];
      d.s_ucx[p] = __ldcg(d.s_ucx + p) + dx * inv;
      d.s_ucy[p] = __ldcg(d.s_ucy + p) + dy * inv;
    }
    sync();
  }
  for (int p = t0; p < nheads; p += stride) {
    float ucx = __ldcg(d.s_ucx + p), ucy = __ldcg(d.s_ucy + p);
    const float c2 = clamp_factor(ucx, ucy, d.vmax);
    ucx = ucx * c2;
    ucy = ucy * c2;
    const float rho = d.s_rho[p];
    float Fx = (ucx - d.s_vx[p]) * rho;
    float Fy = (ucy - d.s_vy[p]) * rho;
    if (d.force_clamp) {
      const float c3 = clamp_factor(Fx, Fy, d.vmax);
      Fx = Fx * c3;
      Fy = Fy * c3;
    }
    d.s_fx[p] = Fx;
    d.s_fy[p] = Fy;
  }
  if (t0 == 0) d.ib_ctl[5] = nheads;  // for k_collide_heads
}

__global__ void __launch_bounds__(256) k_ib_coop(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                 int parity) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int nb = off[r + 1] - off[r];
  const int lb = blockIdx.x - off[r];
  ib_iterations(d, lb * blockDim.x + threadIdx.x, nb * blockDim.x,
                [&] { rollout_barrier(d.ib_ctl, nb, d.flags); });
}

// The same iterations with one thread-block cluster per rollout (cluster c = rollout c):
// the hardware cluster barrier (release / acquire at cluster scope) separates the phases,
// so a rollout's 2 x iterations + 1 dependent steps cost no kernel boundaries and no
// software barrier.  Every CTA of a cluster reaches every barrier: the early return below
// is uniform across the cluster.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int T>
__global__ void __launch_bounds__(T) k_ib_cluster(const RDesc* __restrict__ D, int n) {
  unsigned rank, ncta, cid;
  asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
  asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncta));
  asm("mov.u32 %0, %%clusterid.x;" : "=r"(cid));
  if ((int)cid >= n) return;
  const RDesc& d = D[cid];
  if (!d.enable_fluid || d.NI == 0) return;
  ib_iterations(d, (int)(rank * blockDim.x + threadIdx.x), (int)(ncta * blockDim.x), [] { cluster_sync_all(); });
}

// Post-accumulation clamp and body force F = (u_corrected - u) rho (fluid.py:327-339) per
// touched cell, for the node reaction and for k_collide_heads, which collides these cells
// after the dense pass.  The head count is saved in ib_ctl[5] for k_collide_heads.
__global__ void __launch_bounds__(256) k_ib_finalize(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                     int parity) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  const int nheads = d.ib_ctl[2];
  if (p == 0) d.ib_ctl[5] = nheads;
  if (p >= nheads) return;
  head_force(d, p, d.s_ucx[p], d.s_ucy[p]);
}

// Node reaction (fluid.py:364-382), final wrap (simulate.py:97-98), non-finite check and
// per-step node recording (simulate.py:21-32).
__global__ void __launch_bounds__(256) k_reaction(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                  const int* __restrict__ tdev) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int node = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (node == 0) {
    // this step's deposit has been reduced: reset the CIC bin controls
    d.c_ctl[0] = 0;
    d.c_ctl[1] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.wl_ctl[1] = 0;  // the plan's CIC tile list and its cursor
    d.wl_ctl[3] = 0;
  }
  if (node >= d.N) return;
  float vx = d.vel[2 * node], vy = d.vel[2 * node + 1];
  if (d.enable_fluid) {
    float fx, fy;
    stencil_sum_any(d, node, d.s_fx, d.s_fy, fx, fy);
    if (d.NI > d.N) {
      // synthetic pair: the mean of the two points' forces (fluid.py:371-374)
      float gx, gy;
      stencil_sum_any(d, node + d.N, d.s_fx, d.s_fy, gx, gy);
      fx = 0.5f * (fx + gx);
      fy = 0.5f * (fy + gy);
    }
    vx = vx - (fx / d.node_mass) / d.sdt_x;
    vy = vy - (fy / d.node_mass) / d.sdt_y;
    d.vel[2 * node] = vx;
    d.vel[2 * node + 1] = vy;
  }
  const float px = fmod_floor(d.pos[2 * node], (float)d.W);
  const float py = fmod_floor(d.pos[2 * node + 1], (float)d.H);
  d.pos[2 * node] = px;
  d.pos[2 * node + 1] = py;
  if (!(isfinite(px) && isfinite(py) && isfinite(vx) && isfinite(vy))) atomicOr(d.flags, 1u);
  if (d.rec_every > 0) {
    const int t = *tdev;
    if ((t + 1) % d.rec_every == 0) {
      const size_t e = (size_t)((t + 1) / d.rec_every - 1) * d.N * 2;
      if (d.rec_pos) {
        d.rec_pos[e + 2 * node] = px;
        d.rec_pos[e + 2 * node + 1] = py;
      }
      if (d.rec_vel) {
        d.rec_vel[e + 2 * node] = vx;
        d.rec_vel[e + 2 * node + 1] = vy;
      }
    }
  }
}

// One output sample of a linear, antialiased resize along one axis (JAX's image resize,
// method "linear": triangle kernel widened by max(m/n, 1), weights normalised by their sum
// over the input, zero outside the sampled range): input m -> output n, output index o.
// Writes the first input index and up to kResizeTaps normalised weights; returns the count.
constexpr int kResizeTaps = 16;
__device__ int resize_taps(int o, int m, int n, float inv, float ks, int& i0, float* w) {
  if (m == n) {
    i0 = o;
    w[0] = 1.0f;
    return 1;
  }
  const float sf = ((float)o + 0.5f) * inv - 0.5f;
  int a = (int)floorf(sf - ks), b = (int)ceilf(sf + ks);
  a = a < 0 ? 0 : a;
  b = b > m - 1 ? m - 1 : b;
  if (b - a + 1 > kResizeTaps) b = a + kResizeTaps - 1;  // plans keep the support within the taps
  float tot = 0.0f;
  for (int i = a; i <= b; ++i) {
    float x = fabsf(sf - (float)i) / ks;
    const float v = 1.0f - fabsf(x);
    w[i - a] = v > 0.0f ? v : 0.0f;
    tot = tot + w[i - a];
  }
  const bool inside = sf >= -0.5f && sf <= (float)m - 0.5f;
  const bool norm = fabsf(tot) > 1000.0f * MC_EPSIL;
  for (int i = a; i <= b; ++i) w[i - a] = (inside && norm) ? w[i - a] / tot : 0.0f;
  i0 = a;
  return b - a + 1;
}

// Per-step field recording (steric, fluid_velocity) on recording steps.  The recorded u*
// is on the domain grid: a copy when the lattice is the domain grid, else the linear
// resize of simulate.py:24-29.
__global__ void k_record_fields(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                const int* __restrict__ tdev) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  if (d.rec_every <= 0) return;
  const int t = *tdev;
  if ((t + 1) % d.rec_every != 0) return;
  const size_t e = (size_t)((t + 1) / d.rec_every - 1);
  const size_t HW = (size_t)d.H * d.W, LHW = (size_t)d.lH * d.lW;
  const bool same = d.lH == d.H && d.lW == d.W;
  const size_t stride = (size_t)(off[r + 1] - off[r]) * blockDim.x;
  for (size_t i = (size_t)(blockIdx.x - off[r]) * blockDim.x + threadIdx.x; i < HW; i += stride) {
    if (d.rec_steric) d.rec_steric[e * HW + i] = d.steric[i];
    if (!d.rec_fluid) continue;
    if (same) {
      d.rec_fluid[e * 2 * HW + i] = d.fluid_vel[i];
      d.rec_fluid[e * 2 * HW + HW + i] = d.fluid_vel[HW + i];
      continue;
    }
    const int y = (int)(i / d.W), x = (int)(i - (size_t)y * d.W);
    float wy[kResizeTaps], wx[kResizeTaps];
    int y0, x0;
    const int ny = resize_taps(y, d.lH, d.H, d.rs_inv_y, d.rs_ks_y, y0, wy);
    const int nx = resize_taps(x, d.lW, d.W, d.rs_inv_x, d.rs_ks_x, x0, wx);
    for (int c = 0; c < 2; ++c) {
      const float* u = d.fluid_vel + c * LHW;
      float acc = 0.0f;
      for (int a = 0; a < ny; ++a) {
        float row = 0.0f;
        for (int b = 0; b < nx; ++b) row = row + wx[b] * u[(size_t)(y0 + a) * d.lW + x0 + b];
        acc = acc + wy[a] * row;
      }
      d.rec_fluid[e * 2 * HW + c * HW + i] = acc;
    }
  }
}

__global__ void k_tick(int* tdev) { *tdev += 1; }

cudaError_t tiles_blocks_per_sm(int threads, int capS, int* out) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k_bin_tiles, threads, (size_t)4 * capS * sizeof(unsigned));
}
void launch_bin_tiles(const Launch& L, const int2* wl, int* wl_count, int which, int parity, int capS,
                      int threads) {
  k_bin_tiles<<<L.grid, threads, (size_t)4 * capS * sizeof(unsigned), L.s>>>(L.d, wl, wl_count, which, parity, capS);
}
// `bytes` is the per-block opt-in limit; the kernel's static shared memory comes off it.
cudaError_t tiles_set_smem(size_t bytes) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_bin_tiles);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_bin_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(bytes - a.sharedSizeBytes));
}
void launch_ib_interp(const Launch& L, int it) { k_ib_interp<<<L.grid, kNodeThreads, 0, L.s>>>(L.d, L.off, L.n, it); }
void launch_ib_spread(const Launch& L, int it, int fuse_finalize) {
  k_ib_spread<<<L.grid, kHeadThreads, 0, L.s>>>(L.d, L.off, L.n, it, fuse_finalize);
}
cudaError_t launch_ib_coop(const Launch& L, int parity) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = L.s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_ib_coop, L.d, L.off, L.n, parity);
}
// One cluster of `ctas` CTAs of `threads` (256 or 1024) threads per rollout (1 <= ctas <=
// 16; above 8 the non-portable size is allowed on the kernel first).
cudaError_t launch_ib_cluster(const RDesc* d, int n, int ctas, int threads, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(n * ctas));
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (threads == 1024) return cudaLaunchKernelEx(&cfg, k_ib_cluster<1024>, d, n);
  return cudaLaunchKernelEx(&cfg, k_ib_cluster<256>, d, n);
}
cudaError_t ib_cluster_allow_16() {
  cudaError_t e = cudaFuncSetAttribute(k_ib_cluster<256>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_ib_cluster<1024>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}
cudaError_t ib_coop_blocks_per_sm(int* out) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k_ib_coop, 256, 0);
}

void launch_ib_finalize(const Launch& L, int parity) {
  k_ib_finalize<<<L.grid, kHeadThreads, 0, L.s>>>(L.d, L.off, L.n, parity);
}
void launch_reaction(const Launch& L, const int* tdev) {
  k_reaction<<<L.grid, kNodeThreads, 0, L.s>>>(L.d, L.off, L.n, tdev);
}
void launch_record_fields(const Launch& L, const int* tdev) {
  k_record_fields<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, tdev);
}
void launch_tick(int* tdev, cudaStream_t s) { k_tick<<<1, 1, 0, s>>>(tdev); }

}  // namespace mc
