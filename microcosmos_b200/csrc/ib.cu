// Immersed-boundary coupling (src/microcosmos/solver/fluid.py:202-386) and the
// deterministic scatter-add machinery it shares with the steric cloud-in-cell deposit
// (src/microcosmos/forces.py:98-115).
//
// Scatter-adds are never done with float atomics.  Each contribution k (IB: k = n*K*K + s,
// CIC: k = corner*N + n — the order in which the reference's scatters apply them) is
// binned into a 16x16-cell tile (integer atomics: counts only), the tile's contributions
// are sorted by (cell, k) in shared memory, and every run of equal cells is summed
// sequentially in k order.  The result is bit-reproducible and equals the reference's
// in-order scatter-add.  The IB iterations then work on the compact set of touched cells
// ("slots", indexed by the sorted position of each cell's first contribution) instead
// of full (H, W) grids.
#include "lbm_cell.cuh"

namespace mc {

struct BinView {
  const int* cell;
  const float* w;
  int* binned;
  int* sorted;
  int* tcount;
  int* tfill;
  int* toff;
  int count;
};

__device__ __forceinline__ BinView bin_view(const RDesc& d, int which) {
  BinView v;
  if (which == 0) {
    v.cell = d.ib_cell; v.w = d.ib_w; v.binned = d.ib_binned; v.sorted = d.ib_sorted;
    v.tcount = d.ib_tcount; v.tfill = d.ib_tfill; v.toff = d.ib_toff; v.count = d.M;
  } else {
    v.cell = d.c_cell; v.w = d.c_w; v.binned = d.c_binned; v.sorted = d.c_sorted;
    v.tcount = d.c_tcount; v.tfill = d.c_tfill; v.toff = d.c_toff; v.count = d.enable_steric ? 4 * d.N : 0;
  }
  return v;
}

__device__ __forceinline__ int tile_of(const RDesc& d, int cell) {
  const int cy = cell / d.W, cx = cell - cy * d.W;
  return (cy / kBinTile) * d.ntile_x + cx / kBinTile;
}
__device__ __forceinline__ unsigned local_of(const RDesc& d, int cell) {
  const int cy = cell / d.W, cx = cell - cy * d.W;
  return (unsigned)((cy % kBinTile) * kBinTile + (cx % kBinTile));
}

// Exclusive scan of the tile counts of every rollout (one CTA per rollout).
__global__ void __launch_bounds__(1024) k_bin_scan(const RDesc* __restrict__ D, int n, int which) {
  const int r = blockIdx.x;
  if (r >= n) return;
  const RDesc& d = D[r];
  BinView v = bin_view(d, which);
  if (v.count == 0 || v.tcount == nullptr) return;
  const int nt = d.ntile_x * d.ntile_y;
  __shared__ int wsum[32];
  __shared__ int carry_s;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < nt; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int x = (i < nt) ? v.tcount[i] : 0;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int s = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    const int carry = carry_s;
    const int pre = (wid > 0 ? wsum[wid - 1] : 0) + incl - x;
    if (i < nt) {
      v.toff[i] = carry + pre;
      v.tfill[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry_s = carry + wsum[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) v.toff[nt] = carry_s;
}

// Place every contribution into its tile's segment (order inside a tile is arbitrary;
// the per-tile sort restores the reference order).
__global__ void __launch_bounds__(256) k_bin_scatter(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                     int which) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  BinView v = bin_view(d, which);
  const int k = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (k >= v.count) return;
  const int t = tile_of(d, v.cell[k]);
  const int p = v.toff[t] + atomicAdd(v.tfill + t, 1);
  v.binned[p] = k;
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

// Per tile: sort contributions by (cell, k), then reduce each run of equal cells.
// which == 0 (IB): per touched cell, kernel coverage -> 1/max(cov, 1), the macroscopic
//   state pulled from h[parity] (density, clamped velocity), u_corrected = velocity, and
//   contribution -> slot links.   (fluid.py:268-290)
// which == 1 (CIC): deposit grid value = sum of the run's weights.   (forces.py:98-115)
__global__ void __launch_bounds__(256) k_bin_sort(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                  int which, int parity) {
  __shared__ unsigned skeys[kSortCap];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  BinView v = bin_view(d, which);
  const int t = blockIdx.x - off[r];
  if (v.count == 0) return;
  const int s = v.toff[t];
  const int m = v.toff[t + 1] - s;
  if (m == 0) {
    if (threadIdx.x == 0) v.tcount[t] = 0;
    return;
  }
  unsigned* kp;
  if (m <= kSortCap) {
    int P = 1;
    while (P < m) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
      unsigned key = 0xffffffffu;
      if (i < m) {
        const int k = v.binned[s + i];
        key = (local_of(d, v.cell[k]) << 24) | (unsigned)k;
      }
      skeys[i] = key;
    }
    __syncthreads();
    bitonic_sort_smem(skeys, P);
    kp = skeys;
  } else {
    // chunks of kSortCap sorted in shared memory, then pairwise merges by rank
    unsigned* bufA = reinterpret_cast<unsigned*>(v.sorted) + s;
    unsigned* bufB = reinterpret_cast<unsigned*>(v.binned) + s;
    for (int c0 = 0; c0 < m; c0 += kSortCap) {
      const int len = min(kSortCap, m - c0);
      int P = 1;
      while (P < len) P <<= 1;
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        unsigned key = 0xffffffffu;
        if (i < len) {
          const int k = v.binned[s + c0 + i];
          key = (local_of(d, v.cell[k]) << 24) | (unsigned)k;
        }
        skeys[i] = key;
      }
      __syncthreads();
      bitonic_sort_smem(skeys, P);
      for (int i = threadIdx.x; i < len; i += blockDim.x) bufA[c0 + i] = skeys[i];
      __syncthreads();
    }
    unsigned* src = bufA;
    unsigned* dst = bufB;
    for (int wdt = kSortCap; wdt < m; wdt <<= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
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
    if (src != bufA) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) bufA[i] = src[i];
      __syncthreads();
    }
    kp = bufA;
  }

  const float vmax = d.vmax;
  const size_t HW = (size_t)d.H * d.W;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const unsigned key = kp[i];
    const unsigned lc = key >> 24;
    const bool head = (i == 0) || ((kp[i - 1] >> 24) != lc);
    int len = 0;
    if (head) {
      len = 1;
      while (i + len < m && (kp[i + len] >> 24) == lc) ++len;
    }
    if (which == 1) {
      if (head) {
        const int k0 = (int)(key & 0xffffffu);
        float acc = v.w[k0];
        for (int j = 1; j < len; ++j) acc = acc + v.w[(int)(kp[i + j] & 0xffffffu)];
        d.dep[v.cell[k0]] = acc;
      }
    } else {
      int h0 = i;
      while (h0 > 0 && (kp[h0 - 1] >> 24) == lc) --h0;
      const int k = (int)(key & 0xffffffu);
      d.ib_slot[k] = s + h0;
      d.s_len[s + i] = len;
      if (head) {
        const int cell = v.cell[k];
        float cov = v.w[k];
        for (int j = 1; j < len; ++j) cov = cov + v.w[(int)(kp[i + j] & 0xffffffu)];
        const int p = s + i;
        d.s_cell[p] = cell;
        d.s_inv[p] = 1.0f / max_prop(cov, 1.0f);
        const int y = cell / d.W, x = cell - y * d.W;
        const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        float f[9];
        const float* hp = d.h[parity];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          const int ys = imod_floor(y - ey[q], d.H), xs = imod_floor(x - ex[q], d.W);
          f[q] = hp[q * HW + (size_t)ys * d.W + xs];
        }
        float rho, vx, vy;
        macroscopic(f, vmax, rho, vx, vy);
        d.s_rho[p] = rho;
        d.s_vx[p] = vx;
        d.s_vy[p] = vy;
        d.s_ucx[p] = vx;
        d.s_ucy[p] = vy;
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < m; i += blockDim.x) v.sorted[s + i] = (int)(kp[i] & 0xffffffu);
  if (threadIdx.x == 0) v.tcount[t] = 0;
}

// Multi-direct forcing, interpolation half (fluid.py:292-302): per IB point, u at the point
// = sum_s w_s u_corrected(cell_s); correction = (U_point - u) * relaxation, clamped.
__global__ void __launch_bounds__(256) k_ib_interp(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                   int it) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int node = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (node >= d.N || it >= d.ib_iters) return;
  const int K2 = d.K * d.K;
  float ux = 0.0f, uy = 0.0f;
  for (int s = 0; s < K2; ++s) {
    const int k = node * K2 + s;
    const int p = d.ib_slot[k];
    const float w = d.ib_w[k];
    ux = ux + d.s_ucx[p] * w;
    uy = uy + d.s_ucy[p] * w;
  }
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
                                                   int it) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (p >= d.M || it >= d.ib_iters) return;
  const int len = d.s_len[p];
  if (len == 0) return;
  const int K2 = d.K * d.K;
  float dx = 0.0f, dy = 0.0f;
  for (int j = 0; j < len; ++j) {
    const int k = d.ib_sorted[p + j];
    const int node = k / K2;
    const float w = d.ib_w[k];
    dx = dx + d.delta[2 * node] * w;
    dy = dy + d.delta[2 * node + 1] * w;
  }
  const float inv = d.s_inv[p];
  d.s_ucx[p] = d.s_ucx[p] + dx * inv;
  d.s_ucy[p] = d.s_ucy[p] + dy * inv;
}

// Post-accumulation clamp and body force F = (u_corrected - u) rho (fluid.py:327-339),
// published to the dense pass through the force overlay.
__global__ void __launch_bounds__(256) k_ib_finalize(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (p >= d.M) return;
  if (d.s_len[p] == 0) return;
  float ucx = d.s_ucx[p], ucy = d.s_ucy[p];
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
  const int cell = d.s_cell[p];
  const size_t HW = (size_t)d.H * d.W;
  d.fov[cell] = Fx;
  d.fov[HW + cell] = Fy;
  const int y = cell / d.W, x = cell - y * d.W;
  d.lbm_flag[(y / kLbmTileY) * d.lbm_tx + x / d.lbm_tw] = 1;
}

// Node reaction (fluid.py:364-382), final wrap (simulate.py:97-98), non-finite check and
// per-step node recording (simulate.py:21-32).
__global__ void __launch_bounds__(256) k_reaction(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                                  const int* __restrict__ tdev) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int node = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (node >= d.N) return;
  float vx = d.vel[2 * node], vy = d.vel[2 * node + 1];
  if (d.enable_fluid) {
    const int K2 = d.K * d.K;
    float fx = 0.0f, fy = 0.0f;
    for (int s = 0; s < K2; ++s) {
      const int k = node * K2 + s;
      const int p = d.ib_slot[k];
      const float w = d.ib_w[k];
      fx = fx + d.s_fx[p] * w;
      fy = fy + d.s_fy[p] * w;
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

// Per-step field recording (steric, fluid_velocity) on recording steps.
__global__ void k_record_fields(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                const int* __restrict__ tdev) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  if (d.rec_every <= 0) return;
  const int t = *tdev;
  if ((t + 1) % d.rec_every != 0) return;
  const size_t e = (size_t)((t + 1) / d.rec_every - 1);
  const size_t HW = (size_t)d.H * d.W;
  const size_t stride = (size_t)(off[r + 1] - off[r]) * blockDim.x;
  for (size_t i = (size_t)(blockIdx.x - off[r]) * blockDim.x + threadIdx.x; i < HW; i += stride) {
    if (d.rec_steric) d.rec_steric[e * HW + i] = d.steric[i];
    if (d.rec_fluid) {
      d.rec_fluid[e * 2 * HW + i] = d.fluid_vel[i];
      d.rec_fluid[e * 2 * HW + HW + i] = d.fluid_vel[HW + i];
    }
  }
}

__global__ void k_tick(int* tdev) { *tdev += 1; }

void launch_bin_scan(const Launch& L, int which) { k_bin_scan<<<L.n, 1024, 0, L.s>>>(L.d, L.n, which); }
void launch_bin_scatter(const Launch& L, int which) { k_bin_scatter<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, which); }
void launch_bin_sort(const Launch& L, int which, int parity) {
  k_bin_sort<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, which, parity);
}
void launch_ib_interp(const Launch& L, int it) { k_ib_interp<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, it); }
void launch_ib_spread(const Launch& L, int it) { k_ib_spread<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, it); }
void launch_ib_finalize(const Launch& L) { k_ib_finalize<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n); }
void launch_reaction(const Launch& L, const int* tdev) { k_reaction<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, tdev); }
void launch_record_fields(const Launch& L, const int* tdev) {
  k_record_fields<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, tdev);
}
void launch_tick(int* tdev, cudaStream_t s) { k_tick<<<1, 1, 0, s>>>(tdev); }

}  // namespace mc
