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

// Load the 4 (VEC=4) or 1 (VEC=1) populations of direction (cx, cy) pulled to cells
// x0..x0+VEC-1 of row y.  All lanes of the warp must call this together.
template <int VEC>
__device__ __forceinline__ void pull_dir(const float* __restrict__ plane, int H, int W, int y, int x0c, int lane,
                                         int cx, int cy, float v[VEC]) {
  int ys = y - cy;
  ys = ys < 0 ? ys + H : (ys >= H ? ys - H : ys);
  const float* row = plane + (size_t)ys * W;
  if (VEC == 4) {
    float4 a = __ldg(reinterpret_cast<const float4*>(row + x0c));
    if (cx == 0) {
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else if (cx == 1) {
      float up = __shfl_up_sync(0xffffffffu, a.w, 1);
      if (lane == 0) up = __ldg(row + (x0c == 0 ? W - 1 : x0c - 1));
      v[0] = up; v[1] = a.x; v[2] = a.y; v[3] = a.z;
    } else {
      float dn = __shfl_down_sync(0xffffffffu, a.x, 1);
      if (lane == 31 || x0c + 4 >= W) dn = __ldg(row + (x0c + 4 >= W ? x0c + 4 - W : x0c + 4));
      v[0] = a.y; v[1] = a.z; v[2] = a.w; v[3] = dn;
    }
  } else if (VEC == 2) {
    float2 a = __ldg(reinterpret_cast<const float2*>(row + x0c));
    if (cx == 0) {
      v[0] = a.x; v[1 % VEC] = a.y;
    } else if (cx == 1) {
      float up = __shfl_up_sync(0xffffffffu, a.y, 1);
      if (lane == 0) up = __ldg(row + (x0c == 0 ? W - 1 : x0c - 1));
      v[0] = up; v[1 % VEC] = a.x;
    } else {
      float dn = __shfl_down_sync(0xffffffffu, a.x, 1);
      if (lane == 31 || x0c + 2 >= W) dn = __ldg(row + (x0c + 2 >= W ? x0c + 2 - W : x0c + 2));
      v[0] = a.y; v[1 % VEC] = dn;
    }
  } else {
    int xs = x0c - cx;
    xs = xs < 0 ? xs + W : (xs >= W ? xs - W : xs);
    v[0] = __ldg(row + xs);
  }
}

template <int VEC>
__global__ void __launch_bounds__(256) k_lbm(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                             int parity, int write_u) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const int tx = lb % d.lbm_tx, ty = lb / d.lbm_tx;
  const int lane = threadIdx.x;
  const int H = d.lH, W = d.lW;
  const int y = ty * d.lbm_th + threadIdx.y;
  const int x0 = tx * (32 * VEC) + lane * VEC;
  const bool row_ok = y < H;
  const bool x_ok = x0 < W;
  const int x0c = x_ok ? x0 : (W - VEC);
  const size_t HW = (size_t)H * W;
  const float* __restrict__ hin = d.h[parity];
  float* __restrict__ hout = d.h[parity ^ 1];
  // tile flags are double-buffered by step parity: this step's finalize set flag[parity];
  // the other set belongs to the previous step and is cleared here for the next one
  const int nflag = d.lbm_tx * d.lbm_ty;
  const int flag_idx = ty * d.lbm_tx + tx;
  const bool has_ov = d.lbm_flag[parity * nflag + flag_idx] != 0;
  if (threadIdx.x == 0 && threadIdx.y == 0) d.lbm_flag[(parity ^ 1) * nflag + flag_idx] = 0;

  if (row_ok) {
    float fin[9][VEC];
    const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
#pragma unroll
    for (int i = 0; i < 9; ++i) pull_dir<VEC>(hin + i * HW, H, W, y, x0c, lane, ex[i], ey[i], fin[i]);

    float ovx[VEC], ovy[VEC];
    bool ov[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) ov[c] = false;
    if (has_ov && x_ok) {
      const size_t base = (size_t)y * W + x0;
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        float a = d.fov[base + c], b = d.fov[HW + base + c];
        ov[c] = !is_sentinel(a);
        ovx[c] = a;
        ovy[c] = b;
        if (ov[c]) {
          d.fov[base + c] = nan_f();
          d.fov[HW + base + c] = nan_f();
        }
      }
    }
    const float cp = 1.0f - 0.5f * d.wp, cm = 1.0f - 0.5f * d.wm;
    float out[9][VEC];
    float usx[VEC], usy[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      float f[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) f[i] = fin[i][c];
      float rho, vx, vy, Fx, Fy;
      macroscopic(f, d.vmax, d.vmax_q4, rho, vx, vy);
      if (ov[c]) {
        Fx = ovx[c];
        Fy = ovy[c];
      } else {
        free_cell_force(rho, vx, vy, d.vmax, d.vmax_q4, d.force_clamp, Fx, Fy);
      }
      float o[9];
      collide(f, rho, vx, vy, Fx, Fy, d.wp, d.wm, cp, cm, o, usx[c], usy[c]);
#pragma unroll
      for (int i = 0; i < 9; ++i) out[i][c] = o[i];
    }
    if (x_ok) {
      const size_t base = (size_t)y * W + x0;
      if (VEC == 4) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
          *reinterpret_cast<float4*>(hout + i * HW + base) = make_float4(out[i][0], out[i][1], out[i][2], out[i][3]);
        if (write_u) {
          *reinterpret_cast<float4*>(d.fluid_vel + base) = make_float4(usx[0], usx[1], usx[2], usx[3]);
          *reinterpret_cast<float4*>(d.fluid_vel + HW + base) = make_float4(usy[0], usy[1], usy[2], usy[3]);
        }
      } else if (VEC == 2) {
#pragma unroll
        for (int i = 0; i < 9; ++i)
          *reinterpret_cast<float2*>(hout + i * HW + base) = make_float2(out[i][0], out[i][1 % VEC]);
        if (write_u) {
          *reinterpret_cast<float2*>(d.fluid_vel + base) = make_float2(usx[0], usx[1 % VEC]);
          *reinterpret_cast<float2*>(d.fluid_vel + HW + base) = make_float2(usy[0], usy[1 % VEC]);
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

// Workspace initialisation: overlay = NaN sentinel, deposit grid = 0, counters = 0.
__global__ void k_clear_ws(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const size_t stride = (size_t)(off[r + 1] - off[r]) * blockDim.x;
  const size_t HW = (size_t)d.H * d.W, LHW = (size_t)d.lH * d.lW;
  const size_t t0 = (size_t)lb * blockDim.x + threadIdx.x;
  for (size_t i = t0; i < 2 * LHW; i += stride) d.fov[i] = nan_f();
  if (d.dep)
    for (size_t i = t0; i < HW; i += stride) d.dep[i] = 0.0f;
  const int nt = d.ntile_x * d.ntile_y, lnt = d.lntile_x * d.lntile_y;
  for (size_t i = t0; i < (size_t)lnt; i += stride) d.ib_tcount[i] = 0;
  for (size_t i = t0; i < (size_t)nt; i += stride) d.c_tcount[i] = 0;
  for (size_t i = t0; i < (size_t)2 * d.lbm_tx * d.lbm_ty; i += stride) d.lbm_flag[i] = 0;
  if (t0 < 8) {
    d.ib_ctl[t0] = 0;
    d.c_ctl[t0] = 0;
  }
  if (t0 == 0) *d.flags = 0u;
}

void launch_lbm(const Launch& L, int parity, int write_u, int vec, int rows) {
  dim3 block(32, rows);
  if (vec == 4)
    k_lbm<4><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u);
  else if (vec == 2)
    k_lbm<2><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u);
  else
    k_lbm<1><<<L.grid, block, 0, L.s>>>(L.d, L.off, L.n, parity, write_u);
}

void launch_unstream(const Launch& L) { k_unstream<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n); }
void launch_stream_out(const Launch& L, int parity, float* dst) {
  k_stream_out<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n, parity, dst);
}
void launch_clear_ws(const Launch& L) { k_clear_ws<<<L.grid, 256, 0, L.s>>>(L.d, L.off, L.n); }

}  // namespace mc
