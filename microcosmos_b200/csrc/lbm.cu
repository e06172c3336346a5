// Dense D2Q9 pass: one fused pull-stream + TRT/Guo collide kernel over SoA fp32
// populations, plus the entry/exit conversions between the reference's post-stream
// layout (fields.f_grid) and the pull-scheme post-collision state.
//
// Reference semantics (src/microcosmos/solver/fluid.py:268-357): collide at every cell,
// then push-stream f_new[y+cy, x+cx] = f_post[y, x] (jnp.roll) with an EPSIL floor.
// Here the state between steps is h = f_post (post-collision); a step pulls
// f(x) = h(x - c_i), collides at x and writes h'(x) in place of its own cell, so every
// store is an aligned float4 and every load is an aligned float4 plus a warp shuffle for
// the +-1 column shifts.  fields.f_grid = stream(h) is materialised only at exit.
#include "lbm_cell.cuh"

namespace mc {

// Load the VEC populations of direction (cx, cy) pulled to cells x0c..x0c+VEC-1 of a row:
// `rb` is the element index of the source row (y - cy) in this direction's plane, `xl` / `xr`
// the wrapped columns left of the lane's first cell and right of its last one.  Aligned
// vector loads; the +-1 column shifts come from the neighbouring lane by warp shuffle, the
// warp's edge lanes (and a lane at the lattice's right edge) load their halo value.  All
// lanes of the warp must call this together.  Indices are 32-bit (9 h w < 2^31 is checked
// when a plan is built).
template <int VEC>
__device__ __forceinline__ void pull_dir(const float* __restrict__ h, int rb, int x0c, int xl, int xr, bool edge_l,
                                         bool edge_r, int cx, float v[VEC]) {
  if (VEC == 4) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(h + (rb + x0c)));
    if (cx == 0) {
      v[0] = a.x; v[1 % VEC] = a.y; v[2 % VEC] = a.z; v[3 % VEC] = a.w;
    } else if (cx == 1) {
      float up = __shfl_up_sync(0xffffffffu, a.w, 1);
      if (edge_l) up = __ldg(h + (rb + xl));
      v[0] = up; v[1 % VEC] = a.x; v[2 % VEC] = a.y; v[3 % VEC] = a.z;
    } else {
      float dn = __shfl_down_sync(0xffffffffu, a.x, 1);
      if (edge_r) dn = __ldg(h + (rb + xr));
      v[0] = a.y; v[1 % VEC] = a.z; v[2 % VEC] = a.w; v[3 % VEC] = dn;
    }
  } else if (VEC == 2) {
    const float2 a = __ldg(reinterpret_cast<const float2*>(h + (rb + x0c)));
    if (cx == 0) {
      v[0] = a.x; v[1 % VEC] = a.y;
    } else if (cx == 1) {
      float up = __shfl_up_sync(0xffffffffu, a.y, 1);
      if (edge_l) up = __ldg(h + (rb + xl));
      v[0] = up; v[1 % VEC] = a.x;
    } else {
      float dn = __shfl_down_sync(0xffffffffu, a.x, 1);
      if (edge_r) dn = __ldg(h + (rb + xr));
      v[0] = a.y; v[1 % VEC] = dn;
    }
  } else {
    v[0] = __ldg(h + (rb + (cx == 0 ? x0c : cx == 1 ? xl : xr)));
  }
}

// One cell of the dense pass: density and velocity of the pulled populations, then the
// force-free TRT collision (exact fast path when |u| <= vmax / 2, the velocity clamps
// otherwise) and the EPSIL floor; u* of the cell in (usx, usy).
__device__ __forceinline__ void dense_cell(const RDesc& d, const float f[9], float hwp, float hwm, float cp,
                                           float cm, float o[9], float& usx, float& usy) {
  // rho = max(sum f, 0.1), u = sum e f / rho (fluid.py:136-142)
  float rho = f[0];
#pragma unroll
  for (int i = 1; i < 9; ++i) rho = rho + f[i];
  rho = max_nan(rho, 0.1f);
  const float ux = (((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8]) / rho;
  const float uy = (((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8]) / rho;
  const float usq = ux * ux + uy * uy;
  if (usq + MC_EPSIL <= d.vmax_q4) {
    // |u| <= vmax/2: both velocity clamp factors are exactly 1 and F = 0
    collide_free(f, rho, ux, uy, usq, d.wp, hwp, hwm, o);
    usx = ux;
    usy = uy;
  } else {
    // the velocity clamps (fluid.py:268-274, 327-339) with the unchanged velocity
    float r2, vx, vy, Fx, Fy;
    macroscopic(f, d.vmax, d.vmax_q4, r2, vx, vy);
    free_cell_force(r2, vx, vy, d.vmax, d.vmax_q4, d.force_clamp, Fx, Fy);
    collide(f, r2, vx, vy, Fx, Fy, d.wp, d.wm, cp, cm, o, usx, usy);
  }
}

// One row of VEC cells per lane: pull, collide, store.  All lanes of the warp call it.
template <int VEC>
__device__ __forceinline__ void lbm_row(const RDesc& d, const float* __restrict__ hin, float* __restrict__ hout,
                                        int H, int W, int HW, int y, int x0, int x0c, bool x_ok, int lane,
                                        int write_u, float hwp, float hwm, float cp, float cm) {
  float fin[9][VEC];
  {
    const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    // element index of row y - cy, for cy = -1, 0, +1 (periodic)
    const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
    const int r_cm = yp * W, r_c0 = y * W, r_cp = ym * W;
    // wrapped halo columns (VEC = 1: the left and right neighbours themselves)
    const int xl = x0c == 0 ? W - 1 : x0c - 1;
    const int xr = x0c + VEC >= W ? x0c + VEC - W : x0c + VEC;
    const bool edge_l = lane == 0, edge_r = lane == 31 || x0c + VEC >= W;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int rb = i * HW + (ey[i] == 1 ? r_cp : ey[i] == -1 ? r_cm : r_c0);
      pull_dir<VEC>(hin, rb, x0c, xl, xr, edge_l, edge_r, ex[i], fin[i]);
    }
  }
  float out[9][VEC];
  float usx[VEC], usy[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    float f[9], o[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = fin[i][c];
    dense_cell(d, f, hwp, hwm, cp, cm, o, usx[c], usy[c]);
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i][c] = o[i];
  }
  if (x_ok) {
    const int base = y * W + x0;
    if (VEC == 4) {
#pragma unroll
      for (int i = 0; i < 9; ++i)
        *reinterpret_cast<float4*>(hout + (i * HW + base)) = make_float4(out[i][0], out[i][1 % VEC], out[i][2 % VEC],
                                                                       out[i][3 % VEC]);
      if (write_u) {
        *reinterpret_cast<float4*>(d.fluid_vel + base) = make_float4(usx[0], usx[1 % VEC], usx[2 % VEC], usx[3 % VEC]);
        *reinterpret_cast<float4*>(d.fluid_vel + (HW + base)) =
            make_float4(usy[0], usy[1 % VEC], usy[2 % VEC], usy[3 % VEC]);
      }
    } else if (VEC == 2) {
#pragma unroll
      for (int i = 0; i < 9; ++i)
        *reinterpret_cast<float2*>(hout + (i * HW + base)) = make_float2(out[i][0], out[i][1 % VEC]);
      if (write_u) {
        *reinterpret_cast<float2*>(d.fluid_vel + base) = make_float2(usx[0], usx[1 % VEC]);
        *reinterpret_cast<float2*>(d.fluid_vel + (HW + base)) = make_float2(usy[0], usy[1 % VEC]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) hout[i * HW + base] = out[i][0];
      if (write_u) {
        d.fluid_vel[base] = usx[0];
        d.fluid_vel[HW + base] = usy[0];
      }
    }
  }
}

// The dense pass.  Every cell is collided as if no IB point touched it (F = 0, or the
// force of the velocity clamps alone); the cells the IB touched this step ("heads") are
// collided again with their body force by k_collide_heads, which runs after this kernel
// and overwrites them.  The pass therefore reads no force field and has no force branch.
// CTA tile: 32 * VEC columns x lbm_th rows, blockDim = (32, WY) with WY = min(lbm_th, 4)
// warps; warp wy takes rows wy, wy + WY, ... of the tile (RPW rows each, lbm_th = WY * RPW),
// so the per-thread set-up (rollout lookup, tile position, descriptor loads) is paid once
// for VEC * RPW cells.
template <int VEC, int RPW>
__global__ void __launch_bounds__(128) k_lbm(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                             int parity, int write_u) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const int ntx = d.lbm_tx;
  const int tx = lb % ntx, ty = lb / ntx;
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int H = d.lH, W = d.lW;
  const int x0 = tx * (32 * VEC) + lane * VEC;
  const bool x_ok = x0 < W;
  const int x0c = x_ok ? x0 : (W - VEC);
  const int HW = H * W;
  const float* __restrict__ hin = d.h[parity];
  float* __restrict__ hout = d.h[parity ^ 1];
  const float hwp = 0.5f * d.wp, hwm = 0.5f * d.wm;
  const float cp = 1.0f - 0.5f * d.wp, cm = 1.0f - 0.5f * d.wm;
  const int y0 = ty * d.lbm_th + wy;
#pragma unroll 1
  for (int k = 0; k < RPW; ++k) {
    const int y = y0 + k * (int)blockDim.y;
    if (y >= H) break;  // uniform across the warp
    lbm_row<VEC>(d, hin, hout, H, W, HW, y, x0, x0c, x_ok, lane, write_u, hwp, hwm, cp, cm);
  }
}

// ---------------------------------------------------------------- staged dense pass
// The same pass with its source rows staged in shared memory by bulk asynchronous copies
// (cp.async.bulk global -> shared, completion counted in bytes on an mbarrier).  An item is
// a band of whole lattice rows of one rollout (R = max(1, kStageCells / W) rows, the last
// band of a rollout shorter); for each of the 9 directions the band's source rows y - cy
// (periodic, at most two contiguous pieces) are copied into one shared-memory plane, so a
// population is fetched from HBM once and each bulk copy moves up to 4 KB.  A persistent
// grid walks the items, each CTA keeping `stages` items in flight: while it collides one
// band, the next stages - 1 bands are arriving.  Requires lW % 4 == 0 (16-byte rows) and
// lW <= kStageCells; every cell is collided with exactly the arithmetic of k_lbm.
// Thread t of an item owns cells 4t .. 4t + 3 of the band (row-major); the +-1 column
// shifts come from the neighbouring lane by shuffle or, at a warp or row edge, from the
// row's wrapped column in shared memory.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// bytes: a multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool bar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of a stage barrier (about a second at most): false when
// it gave up.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, unsigned parity) {
  for (unsigned it = 0; it < (1u << 24); ++it) {
    if (bar_test(bar, parity)) return true;
    if (it >= 32) __nanosleep(64);
  }
  return false;
}

// Thread 0: copy item g's 9 source planes into stage buffer `st`, arming `bar`.
__device__ __forceinline__ void stage_item(const RDesc* __restrict__ D, const int* __restrict__ off, int n, int g,
                                           int parity, float* st, uint64_t* bar) {
  const int r = find_rollout(off, n, g);
  const RDesc& d = D[r];
  const int H = d.lH, W = d.lW, R = d.lbm_th;
  const int y0 = (g - off[r]) * R;
  const int rows = min(R, H - y0);
  const int HW = H * W;
  const float* __restrict__ hin = d.h[parity];
  const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  bar_expect_tx(bar, 9u * (unsigned)(rows * W) * 4u);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    int ys = y0 - ey[i];
    ys = ys < 0 ? ys + H : ys >= H ? ys - H : ys;
    const int n1 = min(rows, H - ys);
    float* dst = st + i * kStageCells;
    bulk_load(dst, hin + (i * HW + ys * W), (unsigned)(n1 * W) * 4u, bar);
    if (n1 < rows) bulk_load(dst + n1 * W, hin + i * HW, (unsigned)((rows - n1) * W) * 4u, bar);
  }
}

__global__ void __launch_bounds__(kStagedThreads, 2)
    k_lbm_staged(const RDesc* __restrict__ D, const int* __restrict__ off, int n, int nitems, int parity, int write_u,
                 int stages) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  float* buf = reinterpret_cast<float*>(smem_raw + 128);
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) bar_init(bar + s, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < stages; ++s) {
      const int g = blockIdx.x + s * gridDim.x;
      if (g < nitems) stage_item(D, off, n, g, parity, buf + s * 9 * kStageCells, bar + s);
    }
  }
  __syncthreads();
  for (int j = 0;; ++j) {
    const int g = blockIdx.x + j * gridDim.x;
    if (g >= nitems) break;
    const int s = j % stages;
    const float* st = buf + s * 9 * kStageCells;
    const int r = find_rollout(off, n, g);
    const RDesc& d = D[r];
    const bool ok = bar_wait(bar + s, (unsigned)(j / stages) & 1u);
    if (__syncthreads_or(!ok)) {
      // a copy never completed: flag the rollout, wait (bounded) for this CTA's copies in
      // flight so that none lands after the CTA has exited, and stop
      if (tid == 0) {
        atomicOr(d.flags, 2u);  // MC_FLAG_TIMEOUT
        for (int k = j; k < j + stages && blockIdx.x + k * gridDim.x < nitems; ++k)
          bar_wait(bar + k % stages, (unsigned)(k / stages) & 1u);
      }
      return;
    }
    const int H = d.lH, W = d.lW, R = d.lbm_th;
    const int y0 = (g - off[r]) * R;
    const int chunks = min(R, H - y0) * W / 4;
    const bool active = tid < chunks;
    const int c = active ? tid : chunks - 1;  // idle lanes shadow the last chunk (shuffles)
    const int row = (c * 4) / W, x = c * 4 - row * W;
    const int xl = x == 0 ? W - 1 : x - 1, xr = x + 4 >= W ? x + 4 - W : x + 4;
    const bool edge_l = lane == 0 || x == 0, edge_r = lane == 31 || x + 4 >= W;
    const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    float fin[9][4];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float* p = st + i * kStageCells + row * W;
      const float4 a = *reinterpret_cast<const float4*>(p + x);
      if (ex[i] == 0) {
        fin[i][0] = a.x; fin[i][1] = a.y; fin[i][2] = a.z; fin[i][3] = a.w;
      } else if (ex[i] == 1) {
        float up = __shfl_up_sync(0xffffffffu, a.w, 1);
        if (edge_l) up = p[xl];
        fin[i][0] = up; fin[i][1] = a.x; fin[i][2] = a.y; fin[i][3] = a.z;
      } else {
        float dn = __shfl_down_sync(0xffffffffu, a.x, 1);
        if (edge_r) dn = p[xr];
        fin[i][0] = a.y; fin[i][1] = a.z; fin[i][2] = a.w; fin[i][3] = dn;
      }
    }
    if (active) {
      const float hwp = 0.5f * d.wp, hwm = 0.5f * d.wm;
      const float cp = 1.0f - 0.5f * d.wp, cm = 1.0f - 0.5f * d.wm;
      float out[9][4], usx[4], usy[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float f[9], o[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = fin[i][q];
        dense_cell(d, f, hwp, hwm, cp, cm, o, usx[q], usy[q]);
#pragma unroll
        for (int i = 0; i < 9; ++i) out[i][q] = o[i];
      }
      const int HW = H * W, base = (y0 + row) * W + x;
      float* __restrict__ hout = d.h[parity ^ 1];
#pragma unroll
      for (int i = 0; i < 9; ++i)
        *reinterpret_cast<float4*>(hout + (i * HW + base)) = make_float4(out[i][0], out[i][1], out[i][2], out[i][3]);
      if (write_u) {
        *reinterpret_cast<float4*>(d.fluid_vel + base) = make_float4(usx[0], usx[1], usx[2], usx[3]);
        *reinterpret_cast<float4*>(d.fluid_vel + (HW + base)) = make_float4(usy[0], usy[1], usy[2], usy[3]);
      }
    }
    // every thread has read stage s: refill it with the item `stages` ahead
    __syncthreads();
    if (tid == 0) {
      const int gn = g + stages * gridDim.x;
      if (gn < nitems) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        stage_item(D, off, n, gn, parity, buf + s * 9 * kStageCells, bar + s);
      }
    }
  }
}

// The cells touched by IB points this step, one thread each: the TRT + Guo collision with
// the body force F = (u_corrected - u) rho that k_ib_finalize left per head (fluid.py:327-350),
// written over the dense pass's force-free result.  The populations are pulled again; the
// density and clamped velocity are the ones the tile kernel computed from the same values.
// (Storing the pulled populations per head in the tile kernel instead was measured: the
// stores cost the tile kernel more than the coalesced reads saved here.)
// The head count is the copy k_ib_finalize saved in ib_ctl[5] (the next step's node
// pipeline resets ib_ctl[2] while this kernel may still run).
__global__ void __launch_bounds__(kHeadThreads) k_collide_heads(const RDesc* __restrict__ D, const int* __restrict__ off,
                                                       int n, int parity, int write_u) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (!d.enable_fluid || p >= __ldcg(d.ib_ctl + 5)) return;
  const int cell = d.h_cell[p];
  const int W = d.lW, H = d.lH;
  const int y = cell / W, x = cell - y * W;
  const size_t HW = (size_t)H * W;
  const float* __restrict__ hin = d.h[parity];
  float* __restrict__ hout = d.h[parity ^ 1];
  float f[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int ys = imod_floor(y - kEy[i], H), xs = imod_floor(x - kEx[i], W);
    f[i] = hin[i * HW + (size_t)ys * W + xs];
  }
  const float cp = 1.0f - 0.5f * d.wp, cm = 1.0f - 0.5f * d.wm;
  float o[9], usx, usy;
  collide(f, d.s_rho[p], d.s_vx[p], d.s_vy[p], d.s_fx[p], d.s_fy[p], d.wp, d.wm, cp, cm, o, usx, usy);
#pragma unroll
  for (int i = 0; i < 9; ++i) hout[i * HW + cell] = o[i];
  if (write_u) {
    d.fluid_vel[cell] = usx;
    d.fluid_vel[HW + cell] = usy;
  }
}

// h_i(y, x) = f_grid_i((y + cy) % H, (x + cx) % W): the inverse of the push streaming, so
// that the first pulled step reads exactly fields.f_grid.
__global__ void k_unstream(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const size_t HW = (size_t)d.lH * d.lW;
  const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
  const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  for (size_t idx = (size_t)lb * blockDim.x + threadIdx.x; idx < HW; idx += (size_t)(off[r + 1] - off[r]) * blockDim.x) {
    int y = (int)(idx / d.lW), x = (int)(idx % d.lW);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      int ys = imod_floor(y + ey[i], d.lH), xs = imod_floor(x + ex[i], d.lW);
      d.h[0][i * HW + idx] = max_prop(d.f_grid[i * HW + (size_t)ys * d.lW + xs], MC_EPSIL);
    }
  }
}

// fields.f_grid_i(y, x) = max(h_i((y - cy) % H, (x - cx) % W), EPSIL): the push streaming
// of the reference (fluid.py:352-357) applied to the final post-collision state.
__global__ void k_stream_out(const RDesc* __restrict__ D, const int* __restrict__ off, int n, int parity,
                             float* __restrict__ dst) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const size_t HW = (size_t)d.lH * d.lW;
  const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
  const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  const float* h = d.h[parity];
  float* out = dst ? dst : d.f_grid;  // dst: a snapshot buffer of a one-rollout plan
  for (size_t idx = (size_t)lb * blockDim.x + threadIdx.x; idx < HW; idx += (size_t)(off[r + 1] - off[r]) * blockDim.x) {
    int y = (int)(idx / d.lW), x = (int)(idx % d.lW);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      int ys = imod_floor(y - ey[i], d.lH), xs = imod_floor(x - ex[i], d.lW);
      out[i * HW + idx] = max_prop(h[i * HW + (size_t)ys * d.lW + xs], MC_EPSIL);
    }
  }
}

// Workspace initialisation: deposit grid = 0, counters = 0.
__global__ void k_clear_ws(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const size_t stride = (size_t)(off[r + 1] - off[r]) * blockDim.x;
  const size_t HW = (size_t)d.H * d.W;
  const size_t t0 = (size_t)lb * blockDim.x + threadIdx.x;
  if (d.dep)
    for (size_t i = t0; i < HW; i += stride) d.dep[i] = 0.0f;
  const int nt = d.ntile_x * d.ntile_y, lnt = d.lntile_x * d.lntile_y;
  for (size_t i = t0; i < (size_t)lnt; i += stride) d.ib_tcount[i] = 0;
  for (size_t i = t0; i < (size_t)nt; i += stride) d.c_tcount[i] = 0;
  if (t0 < 8) {
    d.ib_ctl[t0] = 0;
    d.c_ctl[t0] = 0;
  }
  if (t0 == 0) *d.flags = 0u;
}

template <int VEC>
void launch_lbm_vec(const Launch& L, int parity, int write_u, int rows) {
  const int wy = rows < 4 ? rows : 4;
  dim3 block(32, wy);
  switch (rows / wy) {
    case 1: k_lbm<VEC, 1><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u); break;
    case 2: k_lbm<VEC, 2><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u); break;
    case 4: k_lbm<VEC, 4><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u); break;
    default: k_lbm<VEC, 8><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u); break;
  }
}

size_t lbm_staged_smem(int stages) { return 128 + (size_t)stages * 9 * kStageCells * sizeof(float); }

cudaError_t lbm_staged_set_smem(size_t bytes) {
  return cudaFuncSetAttribute(k_lbm_staged, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t lbm_staged_blocks_per_sm(int stages, int* out) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, k_lbm_staged, kStagedThreads, lbm_staged_smem(stages));
}

// L.grid: the number of items (bands) of the plan; ctas: the persistent grid
void launch_lbm_staged(const Launch& L, int parity, int write_u, int stages, int ctas) {
  const int grid = ctas < L.grid ? ctas : L.grid;
  if (grid <= 0) return;
  k_lbm_staged<<<grid, kStagedThreads, lbm_staged_smem(stages), L.s>>>(L.d, L.off, L.n, L.grid, parity, write_u,
                                                                       stages);
}

// rows: the tile height (2, 4, 8, 16 or 32); up to 4 warps per CTA, each looping over
// rows / 4 of them
void launch_lbm(const Launch& L, int parity, int write_u, int vec, int rows) {
  if (vec == 4)
    launch_lbm_vec<4>(L, parity, write_u, rows);
  else if (vec == 2)
    launch_lbm_vec<2>(L, parity, write_u, rows);
  else
    launch_lbm_vec<1>(L, parity, write_u, rows);
}

// Whether f is one of the dense-pass kernels (tiled shapes or the staged form).
bool is_dense_pass_kernel(const void* f) {
  const void* ks[] = {(const void*)k_lbm<1, 1>, (const void*)k_lbm<1, 2>, (const void*)k_lbm<1, 4>,
                      (const void*)k_lbm<1, 8>, (const void*)k_lbm<2, 1>, (const void*)k_lbm<2, 2>,
                      (const void*)k_lbm<2, 4>, (const void*)k_lbm<2, 8>, (const void*)k_lbm<4, 1>,
                      (const void*)k_lbm<4, 2>, (const void*)k_lbm<4, 4>, (const void*)k_lbm<4, 8>,
                      (const void*)k_lbm_staged};
  for (const void* k : ks)
    if (k == f) return true;
  return false;
}

void launch_collide_heads(const Launch& L, int parity, int write_u) {
  k_collide_heads<<<L.grid, kHeadThreads, 0, L.s>>>(L.d, L.off, L.n, parity, write_u);
}

void launch_unstream(const Launch& L) { k_unstream<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n); }
void launch_stream_out(const Launch& L, int parity, float* dst) {
  k_stream_out<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, parity, dst);
}
void launch_clear_ws(const Launch& L) { k_clear_ws<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n); }

}  // namespace mc
