// Node-side kernels of one step (src/microcosmos/simulate.py:37-84):
//   k_predict: damping, inertial prediction, steric cloud-in-cell contributions;
//   k_steric:  per node, the steric force added to the prediction (forces.py:41-81);
//   k_chain:   one warp per chain rod (the topology make_edges(.., "line", F) builds),
//              node/edge state in registers, neighbours exchanged with shuffles;
//   k_node:    one CTA per rod of any other topology (trees, loops), state in shared
//              memory, scatter-adds as gather lists in the reference's order.
//   k_stencil: per node, the velocity from positions and the IB stencil (fluid.py:40-87).
// Both rod kernels evaluate the curvature actuation and run cycles_per_step Jacobi
// iterations of pbd_rod_constraint (solver/pbd.py:14-91).
#include "lbm_cell.cuh"

namespace mc {

__device__ __forceinline__ int bin_tile(const RDesc& d, int cy, int cx) {
  return (cy / kBinTile) * d.ntile_x + cx / kBinTile;
}

__global__ void __launch_bounds__(256) k_predict(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int node = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (node == 0) {
    // the previous step's IB work is complete: reset this step's IB bin controls
    d.ib_ctl[0] = 0;
    d.ib_ctl[1] = 0;
    d.ib_ctl[2] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.wl_ctl[0] = 0;  // the plan's IB tile list and its cursor
    d.wl_ctl[2] = 0;
  }
  if (node >= d.N) return;
  const float px = d.pos[2 * node], py = d.pos[2 * node + 1];
  const float vx = d.vel[2 * node] * d.damping, vy = d.vel[2 * node + 1] * d.damping;
  d.prev[2 * node] = px;
  d.prev[2 * node + 1] = py;
  d.vel[2 * node] = vx;
  d.vel[2 * node + 1] = vy;
  const float qx = px + vx * d.dt, qy = py + vy * d.dt;
  d.pred[2 * node] = qx;
  d.pred[2 * node + 1] = qy;
  if (!d.enable_steric) return;
  // update_steric_potential (forces.py:84-115): CIC weights of the wrapped prediction
  const float W = (float)d.W, H = (float)d.H;
  const float x = fmod_floor(qx, W), y = fmod_floor(qy, H);
  d.predw[2 * node] = x;
  d.predw[2 * node + 1] = y;
  const float fx = floorf(x), fy = floorf(y);
  const int x0 = imod_floor((int)fx, d.W), y0 = imod_floor((int)fy, d.H);
  const int x1 = (x0 + 1) % d.W, y1 = (y0 + 1) % d.H;
  const float dx = x - fx, dy = y - fy;
  const float s = d.st_scatter;
  const float w[4] = {((1.0f - dx) * (1.0f - dy)) * s, (dx * (1.0f - dy)) * s, ((1.0f - dx) * dy) * s, (dx * dy) * s};
  const int cy[4] = {y0, y0, y1, y1};
  const int cx[4] = {x0, x1, x0, x1};
  int tile[4], first[4], cnt[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    tile[c] = bin_tile(d, cy[c], cx[c]);
    first[c] = c;
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (e < c && tile[e] == tile[c] && first[c] == c) first[c] = e;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    cnt[c] = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) cnt[c] += (first[e] == c) ? 1 : 0;
  }
  int base[4], rank[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    base[c] = cnt[c] ? atomicAdd(d.c_tcount + tile[c], cnt[c]) : -1;
    if (base[c] == 0) d.wl_cic[atomicAdd(d.wl_ctl + 1, 1)] = make_int2(d.ridx, tile[c]);
    rank[c] = 0;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int k = c * d.N + node;
    d.c_cell[k] = cy[c] * d.W + cx[c];
    d.c_w[k] = w[c];
    const int g = first[c];
    const int pos = base[g] + rank[g]++;
    if (pos < d.c_cap) {
      d.c_store[(size_t)tile[c] * d.c_cap + pos] = bin_entry(cy[c], cx[c], k);
    } else {
      d.c_ovf[atomicAdd(d.c_ctl, 1)] = k;
    }
  }
}

// map_coordinates(V, [yy, xx], order=1, mode="wrap") (forces.py:30-34)
__device__ __forceinline__ float sample_wrap(const float* __restrict__ V, int H, int W, float yy, float xx) {
  const float ly = floorf(yy), lx = floorf(xx);
  const float ty = yy - ly, tx = xx - lx;
  const float wy0 = 1.0f - ty, wx0 = 1.0f - tx;
  const int iy = (int)ly, ix = (int)lx;
  const int iy0 = imod_floor(iy, H), iy1 = imod_floor(iy + 1, H);
  const int ix0 = imod_floor(ix, W), ix1 = imod_floor(ix + 1, W);
  float acc = (wy0 * wx0) * V[(size_t)iy0 * W + ix0];
  acc = acc + (wy0 * tx) * V[(size_t)iy0 * W + ix1];
  acc = acc + (ty * wx0) * V[(size_t)iy1 * W + ix0];
  acc = acc + (ty * tx) * V[(size_t)iy1 * W + ix1];
  return acc;
}

// compute_field_steric_force_corrected for node gi (forces.py:41-81): -grad V by central
// differences of bilinear samples, minus the analytic Gaussian of global neighbours
// gi-n..gi+n (the 0 <= j < N mask only, as in the reference).
__device__ float2 steric_force(const RDesc& d, int gi) {
  const float W = (float)d.W, H = (float)d.H;
  const float px = d.predw[2 * gi], py = d.predw[2 * gi + 1];
  const float* V = d.steric;
  const float gx = (sample_wrap(V, d.H, d.W, py, px + 0.5f) - sample_wrap(V, d.H, d.W, py, px - 0.5f)) / 1.0f;
  const float gy = (sample_wrap(V, d.H, d.W, py + 0.5f, px) - sample_wrap(V, d.H, d.W, py - 0.5f, px)) / 1.0f;
  float fx = -gx, fy = -gy;
  const int nsk = d.st_skip;
  if (nsk > 0) {
    float ax = 0.0f, ay = 0.0f;
    for (int o = -nsk; o <= nsk; ++o) {
      const int j = gi + o;
      const float valid = (j >= 0 && j < d.N) ? 1.0f : 0.0f;
      const int js = j < 0 ? 0 : (j >= d.N ? d.N - 1 : j);
      const float qx = d.predw[2 * js], qy = d.predw[2 * js + 1];
      const float2 rr = min_image(px, py, qx, qy, W, H);
      const float d2 = rr.x * rr.x + rr.y * rr.y;
      const float K = expf(-d2 / d.st_2s2) / d.st_norm;
      const float kv = K * valid;
      ax = ax + kv * rr.x;
      ay = ay + kv * rr.y;
    }
    fx = fx - d.st_coef * ax;
    fy = fy - d.st_coef * ay;
  }
  return make_float2(fx, fy);
}

// Predicted position of node gi after the steric displacement (simulate.py:55-63).
__device__ __forceinline__ float2 node_start(const RDesc& d, int gi) {
  float qx = d.pred[2 * gi], qy = d.pred[2 * gi + 1];
  if (d.enable_steric) {
    const float2 f = steric_force(d, gi);
    qx = qx + (f.x * d.st_strength) * d.dt;
    qy = qy + (f.y * d.st_strength) * d.dt;
  }
  return make_float2(qx, qy);
}

// Rest angle of pair gb at step t (the caller-side curvature actuation, if any).
__device__ __forceinline__ float rest_angle(const RDesc& d, int gb, int t) {
  if (!d.act_amp) return d.rest_ang[gb];
  const float arg = d.act_omega[gb] * (float)(d.act_t0 + t) + d.act_phase[gb];
  const float a = d.act_c[gb] + d.act_amp[gb] * sinf(arg);
  d.rest_ang[gb] = a;
  return a;
}

// One theta correction (pbd.py:35-40) and one edge force (pbd.py:60-81).
__device__ __forceinline__ float bend_corr(float th_in, float th_out, float rest, float kb) {
  float diff = th_out - th_in;
  diff = fmod_floor(diff + MC_PI_F, MC_2PI_F) - MC_PI_F;
  return ((diff - rest) * kb) * 0.5f;
}

__device__ __forceinline__ float2 edge_force(const RDesc& d, float th, float L0, float xs, float ys, float xt,
                                             float yt) {
  float sn, cs;
  sincosf(th, &sn, &cs);
  const float tx = cs * L0, ty = sn * L0;
  const float2 cur = min_image(xt, yt, xs, ys, (float)d.W, (float)d.H);
  const float L = sqrtf(cur.x * cur.x + cur.y * cur.y);
  const float Lc = max_prop(L, 1e-8f);
  const float stx = (cur.x / Lc) * (L - L0), sty = (cur.y / Lc) * (L - L0);
  const float shx = (cur.x - tx) - stx, shy = (cur.y - ty) - sty;
  return make_float2(((stx + shx * d.k_shear) * d.k_stretch) * 0.5f, ((sty + shy * d.k_shear) * d.k_stretch) * 0.5f);
}

// IB point p in lattice units (fluid.py:236-263): node p's position times the grid scale,
// or with synthetic pairs (p < N: +, p >= N: -, node = p mod N) that point moved by
// width * perp * mean_scale, where perp is the normal of the chain tangent, the sum of the
// node's edge vectors in the reference's update order (src updates, then tgt updates),
// normalised by sqrt(|t|^2 + EPSIL).
__device__ __forceinline__ float2 ib_point(const RDesc& d, int p, int node, float x, float y) {
  const float gx = x * d.scale_x, gy = y * d.scale_y;
  if (!(d.syn_w > 0.0f)) return make_float2(gx, gy);
  float tx = 0.0f, ty = 0.0f;
  for (int j = d.ne_off[node]; j < d.ne_off[node + 1]; ++j) {
    const int e = d.ne_idx[j] >> 1;
    const int s = d.pairs[2 * e], g = d.pairs[2 * e + 1];
    const float2 ev = min_image(d.pos[2 * g], d.pos[2 * g + 1], d.pos[2 * s], d.pos[2 * s + 1], (float)d.W, (float)d.H);
    tx = tx + ev.x;
    ty = ty + ev.y;
  }
  const float nrm = sqrtf((tx * tx + ty * ty) + MC_EPSIL);
  const float ux = tx / nrm, uy = ty / nrm;
  const float ox = (d.syn_w * (-uy)) * d.syn_ms, oy = (d.syn_w * ux) * d.syn_ms;
  return p < d.N ? make_float2(gx + ox, gy + oy) : make_float2(gx - ox, gy - oy);
}

// Velocity (simulate.py:83-84), the IB point in lattice units (fluid.py:236-239) and its
// K x K stencil (fluid.py:40-79) appended to the IB bins, and the clearing of the node's
// CIC deposit cells (the deposit grid stays zero between steps).  The stencil spans at
// most 2 x 2 bin tiles, so its contributions take their bin slots with one atomic per tile.
__global__ void __launch_bounds__(256) k_stencil(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int p = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;  // IB point
  if (p >= d.NI) return;
  const int gi = p < d.N ? p : p - d.N;
  const float x = d.pos[2 * gi], y = d.pos[2 * gi + 1];
  const float vx = (x - d.prev[2 * gi]) / d.dt, vy = (y - d.prev[2 * gi + 1]) / d.dt;
  if (p < d.N) {
    d.vel[2 * gi] = vx;
    d.vel[2 * gi + 1] = vy;
    if (d.enable_steric) {
#pragma unroll
      for (int c = 0; c < 4; ++c) d.dep[d.c_cell[c * d.N + gi]] = 0.0f;
    }
  }
  if (!d.enable_fluid) return;
  const int K = d.K, K2 = K * K;
  const float2 gp = ib_point(d, p, gi, x, y);
  const float gx = gp.x, gy = gp.y;
  d.nvl[2 * p] = (vx * d.scale_x) * d.dt;
  d.nvl[2 * p + 1] = (vy * d.scale_y) * d.dt;
  const int half = (K - 1) / 2;
  const float hw = (float)K / 2.0f;
  const float sx = floorf(gx) - (float)half, sy = floorf(gy) - (float)half;
  float wx[8], wy[8];
  int cx[8], cy[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    if (a < K) {
      const float rx = fabsf((sx + (float)a) - gx) / hw;
      const float ry = fabsf((sy + (float)a) - gy) / hw;
      wx[a] = rx <= 2.0f ? 0.25f * (1.0f + cosf((MC_PI_F * rx) / 2.0f)) : 0.0f;
      wy[a] = ry <= 2.0f ? 0.25f * (1.0f + cosf((MC_PI_F * ry) / 2.0f)) : 0.0f;
      cx[a] = imod_floor((int)(sx + (float)a), d.lW);
      cy[a] = imod_floor((int)(sy + (float)a), d.lH);
    }
  }
  float sum = 0.0f;
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (a < K && b < K) sum = sum + wx[a] * wy[b];
  const float den = sum + MC_EPSIL;
  // tile split of the stencil: columns (rows) whose tile differs from the first one's.
  // A window of K <= 8 consecutive cells meets at most two tiles unless the grid's last
  // tile is narrower than the window; then every contribution takes its own slot.
  const int tx0 = cx[0] / kBinTile, ty0 = cy[0] / kBinTile;
  int txo = -1, tyo = -1, nx1 = 0, ny1 = 0;
  bool split_ok = true;
#pragma unroll
  for (int a = 1; a < 8; ++a) {
    if (a < K) {
      const int tx = cx[a] / kBinTile, ty = cy[a] / kBinTile;
      if (tx != tx0) {
        if (txo >= 0 && tx != txo) split_ok = false;
        txo = tx;
        ++nx1;
      }
      if (ty != ty0) {
        if (tyo >= 0 && ty != tyo) split_ok = false;
        tyo = ty;
        ++ny1;
      }
    }
  }
  if (txo < 0) txo = tx0;
  if (tyo < 0) tyo = ty0;
  const int nx0 = K - nx1, ny0 = K - ny1;
  int base[4];
  const int tiles[4] = {ty0 * d.lntile_x + tx0, ty0 * d.lntile_x + txo, tyo * d.lntile_x + tx0, tyo * d.lntile_x + txo};
  const int counts[4] = {nx0 * ny0, nx1 * ny0, nx0 * ny1, nx1 * ny1};
  if (split_ok) {
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      base[g] = counts[g] ? atomicAdd(d.ib_tcount + tiles[g], counts[g]) : -1;
      if (base[g] == 0) d.wl_ib[atomicAdd(d.wl_ctl, 1)] = make_int2(d.ridx, tiles[g]);
    }
  }
  int rank[4] = {0, 0, 0, 0};
  const int cap = d.ib_cap;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    if (a < K) {
      const int xs = (cx[a] / kBinTile != tx0) ? 1 : 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        if (b < K) {
          const int ys = (cy[b] / kBinTile != ty0) ? 1 : 0;
          const int g = xs + 2 * ys;
          const int k = p * K2 + a * K + b;
          d.ib_cell[k] = cy[b] * d.lW + cx[a];
          d.ib_w[k] = (wx[a] * wy[b]) / den;
          int tile, pos;
          if (split_ok) {
            tile = tiles[g];
            pos = base[g] + rank[g]++;
          } else {
            tile = (cy[b] / kBinTile) * d.lntile_x + cx[a] / kBinTile;
            pos = atomicAdd(d.ib_tcount + tile, 1);
            if (pos == 0) d.wl_ib[atomicAdd(d.wl_ctl, 1)] = make_int2(d.ridx, tile);
          }
          if (pos < cap) {
            d.ib_store[(size_t)tile * cap + pos] = bin_entry(cy[b], cx[a], k);
          } else {
            d.ib_ovf[atomicAdd(d.ib_ctl, 1)] = k;
          }
        }
      }
    }
  }
}

// The same work with one 16-lane group per node (K <= 4): lane s = a*K + b owns stencil
// entry s.  The weight normalisation sum is taken by the group's first lane in entry
// order, so the result equals the one-thread-per-node kernel's; bin slots are taken with
// one atomic per (warp, tile) group.
__global__ void __launch_bounds__(256) k_stencil16(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int t = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  const int p = t >> 4, s = t & 15;  // IB point, stencil entry
  const int lane = threadIdx.x & 31;
  const unsigned gmask = 0xffffu << (lane & 16);
  if (p >= d.NI) return;  // both halves of a warp exit together unless NI is odd
  const int gi = p < d.N ? p : p - d.N;
  const float x = d.pos[2 * gi], y = d.pos[2 * gi + 1];
  const float vx = (x - d.prev[2 * gi]) / d.dt, vy = (y - d.prev[2 * gi + 1]) / d.dt;
  if (p < d.N) {
    if (s == 0) {
      d.vel[2 * gi] = vx;
      d.vel[2 * gi + 1] = vy;
    }
    if (d.enable_steric && s < 4) d.dep[d.c_cell[s * d.N + gi]] = 0.0f;
  }
  if (!d.enable_fluid) return;
  const int K = d.K, K2 = K * K;
  const float2 gp = ib_point(d, p, gi, x, y);
  const float gx = gp.x, gy = gp.y;
  if (s == 0) {
    d.nvl[2 * p] = (vx * d.scale_x) * d.dt;
    d.nvl[2 * p + 1] = (vy * d.scale_y) * d.dt;
  }
  const int half = (K - 1) / 2;
  const float hw = (float)K / 2.0f;
  const float sx = floorf(gx) - (float)half, sy = floorf(gy) - (float)half;
  const int a = s / K, b = s - (s / K) * K;
  const bool act = s < K2;
  const float rx = fabsf((sx + (float)a) - gx) / hw;
  const float ry = fabsf((sy + (float)b) - gy) / hw;
  const float wxa = rx <= 2.0f ? 0.25f * (1.0f + cosf((MC_PI_F * rx) / 2.0f)) : 0.0f;
  const float wyb = ry <= 2.0f ? 0.25f * (1.0f + cosf((MC_PI_F * ry) / 2.0f)) : 0.0f;
  const float w = wxa * wyb;
  float sum = 0.0f;
  for (int q = 0; q < K2; ++q) sum = sum + __shfl_sync(gmask, w, q, 16);
  const float den = sum + MC_EPSIL;
  if (!act) return;
  const int cx = imod_floor((int)(sx + (float)a), d.lW);
  const int cy = imod_floor((int)(sy + (float)b), d.lH);
  const int k = p * K2 + s;
  d.ib_cell[k] = cy * d.lW + cx;
  d.ib_w[k] = w / den;
  const int tile = (cy / kBinTile) * d.lntile_x + cx / kBinTile;
  const unsigned active = __activemask();
  const unsigned group = __match_any_sync(active, tile);
  const int leader = __ffs(group) - 1;
  int base = 0;
  if (lane == leader) {
    base = atomicAdd(d.ib_tcount + tile, __popc(group));
    if (base == 0) d.wl_ib[atomicAdd(d.wl_ctl, 1)] = make_int2(d.ridx, tile);
  }
  base = __shfl_sync(group, base, leader);
  const int pos = base + __popc(group & ((1u << lane) - 1u));
  if (pos < d.ib_cap) {
    d.ib_store[(size_t)tile * d.ib_cap + pos] = bin_entry(cy, cx, k);
  } else {
    d.ib_ovf[atomicAdd(d.ib_ctl, 1)] = k;
  }
}

// The prediction displaced by the steric force (simulate.py:55-65), written to the node
// positions the rod kernels start from.
__global__ void __launch_bounds__(256) k_steric(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int gi = (blockIdx.x - off[r]) * blockDim.x + threadIdx.x;
  if (gi >= d.N) return;
  const float2 s = node_start(d, gi);
  d.pos[2 * gi] = s.x;
  d.pos[2 * gi + 1] = s.y;
}

// ---------------------------------------------------------------- chains: warp per rod
// Lane l owns nodes/edges/pairs j = l*P + q (q < P).  In a chain, edge j = (node j, node
// j+1) and pair j = (edge j, edge j+1); the scatter-adds reduce to
//   theta_j += ((0 + c_j) + (-c_{j-1})) / deg_j * 1.8,   x_j += ((0 + f_j) + (-f_{j-1})) / deg_j
// with the terms that exist, in the reference's order (e_in / src updates first).
template <int P>
__device__ __forceinline__ void shift_next(const float (&v)[P], float (&nx)[P]) {
  const float first_next = __shfl_down_sync(0xffffffffu, v[0], 1);
#pragma unroll
  for (int q = 0; q < P - 1; ++q) nx[q] = v[q + 1];
  nx[P - 1] = first_next;
}
template <int P>
__device__ __forceinline__ void shift_prev(const float (&v)[P], float (&pv)[P]) {
  const float last_prev = __shfl_up_sync(0xffffffffu, v[P - 1], 1);
#pragma unroll
  for (int q = P - 1; q > 0; --q) pv[q] = v[q - 1];
  pv[0] = last_prev;
}

// Stable-Cosserat iterations of one chain rod (solver/stable_cosserat.py:13-119), same
// lane layout as the PBD loop below.  Phase 1: the bending pass without over-relaxation,
// then theta += wrap(atan2(r) - theta) * 0.05 with r the segment's min-image vector.
// Phase 2: x += (w (y0 - x) + f_j - f_{j-1}) / ((w + H_j) + H_{j-1}), f = (k_s/l)(r/l - d),
// H = k_s/l^2, y0 the inertial prediction (the positions the kernel started from).
template <int P>
__device__ __forceinline__ void cosserat_chain(const RDesc& d, int lane, int nn, int ne, int nb, float (&x)[P],
                                               float (&y)[P], float (&th)[P], const float (&l0)[P],
                                               const float (&ra)[P], const float (&kb)[P], const float (&edg)[P]) {
  const float W = (float)d.W, H = (float)d.H;
  const float ks = d.k_stretch, w = d.cos_w;
  float x0[P], y0[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    x0[q] = x[q];
    y0[q] = y[q];
  }
  for (int it = 0; it < d.cycles; ++it) {
    float nx[P], pv[P], c[P], xn[P], yn[P];
    shift_next<P>(th, nx);
#pragma unroll
    for (int q = 0; q < P; ++q) c[q] = (lane * P + q < nb) ? bend_corr(th[q], nx[q], ra[q], kb[q]) : 0.0f;
    shift_prev<P>(c, pv);
    shift_next<P>(x, xn);
    shift_next<P>(y, yn);
    float fx[P], fy[P], he[P], fxp[P], fyp[P], hep[P];
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const int j = lane * P + q;
      fx[q] = fy[q] = he[q] = 0.0f;
      if (j < ne) {
        float acc = 0.0f;
        if (j < nb) acc = acc + c[q];
        if (j >= 1 && j - 1 < nb) acc = acc + (-pv[q]);
        const float2 r = min_image(xn[q], yn[q], x[q], y[q], W, H);
        th[q] = cos_pull(th[q] + acc * edg[q], r.x, r.y);
        float sn, cs;
        sincosf(th[q], &sn, &cs);
        const float kl = ks / l0[q];
        fx[q] = kl * (r.x / l0[q] - cs);
        fy[q] = kl * (r.y / l0[q] - sn);
        he[q] = ks / (l0[q] * l0[q]);
      }
    }
    shift_prev<P>(fx, fxp);
    shift_prev<P>(fy, fyp);
    shift_prev<P>(he, hep);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const int j = lane * P + q;
      if (j < nn) {
        float ax = w * (x0[q] - x[q]), ay = w * (y0[q] - y[q]), hh = w;
        if (j < ne) {
          ax = ax + fx[q];
          ay = ay + fy[q];
          hh = hh + he[q];
        }
        if (j >= 1) {
          ax = ax + (-fxp[q]);
          ay = ay + (-fyp[q]);
          hh = hh + hep[q];
        }
        x[q] = x[q] + ax / hh;
        y[q] = y[q] + ay / hh;
      }
    }
  }
}

template <int P>
__global__ void __launch_bounds__(128) k_chain(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                                               const int* __restrict__ tdev) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ci = (blockIdx.x - off[r]) * kChainWarps + warp;
  if (ci >= d.nchain) return;  // the whole warp leaves together
  const int comp = d.chain_comp[ci];
  const int n0 = d.comp_n[comp], nn = d.comp_n[comp + 1] - n0;
  const int e0 = d.comp_e[comp], ne = nn - 1;
  const int b0 = d.comp_b[comp], nb = nn > 2 ? nn - 2 : 0;
  const int t = *tdev;
  float x[P], y[P], th[P], l0[P], ra[P], kb[P], edg[P], ndg[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int j = lane * P + q;
    x[q] = y[q] = th[q] = l0[q] = ra[q] = kb[q] = 0.0f;
    if (j < nn) {
      x[q] = d.pos[2 * (n0 + j)];
      y[q] = d.pos[2 * (n0 + j) + 1];
    }
    if (j < ne) {
      th[q] = d.theta[e0 + j];
      l0[q] = d.rest_len[e0 + j];
    }
    if (j < nb) {
      ra[q] = rest_angle(d, b0 + j, t);
      kb[q] = d.kb[b0 + j];
    }
    // chain degrees are 1 or 2, so x / deg == x * (1 / deg) exactly
    edg[q] = ((j < nb) + (j >= 1 && j - 1 < nb)) == 2 ? 0.5f : 1.0f;
    ndg[q] = ((j < ne) + (j >= 1 && j - 1 < ne)) == 2 ? 0.5f : 1.0f;
  }
  const int cycles = d.cycles;
  if (d.solver == 1) {
    cosserat_chain<P>(d, lane, nn, ne, nb, x, y, th, l0, ra, kb, edg);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const int j = lane * P + q;
      if (j < ne) d.theta[e0 + j] = th[q];
      if (j < nn) {
        d.pos[2 * (n0 + j)] = x[q];
        d.pos[2 * (n0 + j) + 1] = y[q];
      }
    }
    return;
  }
  // descriptor values the iterations use, held in registers for the whole loop
  const float Wf = (float)d.W, Hf = (float)d.H, ksh = d.k_shear, kst = d.k_stretch;
  for (int it = 0; it < cycles; ++it) {
    // The part of each edge force that depends only on the positions (min-image segment,
    // length, stretch term: edge_force's first half) is taken before the bending pass, whose
    // chain of shuffles and angle updates it then overlaps; the angle-dependent half follows
    // it.  Same expressions as edge_force, so the same bits.
    float xn[P], yn[P], sgx[P], sgy[P], stx[P], sty[P];
    shift_next<P>(x, xn);
    shift_next<P>(y, yn);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const float2 cur = min_image(xn[q], yn[q], x[q], y[q], Wf, Hf);
      const float L = sqrtf(cur.x * cur.x + cur.y * cur.y);
      const float Lc = max_prop(L, 1e-8f);
      sgx[q] = cur.x;
      sgy[q] = cur.y;
      stx[q] = (cur.x / Lc) * (L - l0[q]);
      sty[q] = (cur.y / Lc) * (L - l0[q]);
    }
    float nx[P], pv[P], c[P];
    shift_next<P>(th, nx);
#pragma unroll
    for (int q = 0; q < P; ++q) c[q] = (lane * P + q < nb) ? bend_corr(th[q], nx[q], ra[q], kb[q]) : 0.0f;
    shift_prev<P>(c, pv);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const int j = lane * P + q;
      if (j < ne) {
        float acc = 0.0f;
        if (j < nb) acc = acc + c[q];
        if (j >= 1 && j - 1 < nb) acc = acc + (-pv[q]);
        th[q] = th[q] + (acc * edg[q]) * 1.8f;
      }
    }
    float fx[P], fy[P], fxp[P], fyp[P];
#pragma unroll
    for (int q = 0; q < P; ++q) {
      fx[q] = fy[q] = 0.0f;
      if (lane * P + q < ne) {
        float sn, cs;
        sincosf(th[q], &sn, &cs);
        const float tx = cs * l0[q], ty = sn * l0[q];
        const float shx = (sgx[q] - tx) - stx[q], shy = (sgy[q] - ty) - sty[q];
        fx[q] = ((stx[q] + shx * ksh) * kst) * 0.5f;
        fy[q] = ((sty[q] + shy * ksh) * kst) * 0.5f;
      }
    }
    shift_prev<P>(fx, fxp);
    shift_prev<P>(fy, fyp);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const int j = lane * P + q;
      if (j < nn) {
        float ax = 0.0f, ay = 0.0f;
        if (j < ne) {
          ax = ax + fx[q];
          ay = ay + fy[q];
        }
        if (j >= 1) {
          ax = ax + (-fxp[q]);
          ay = ay + (-fyp[q]);
        }
        x[q] = x[q] + ax * ndg[q];
        y[q] = y[q] + ay * ndg[q];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int j = lane * P + q;
    if (j < ne) d.theta[e0 + j] = th[q];
    if (j < nn) {
      d.pos[2 * (n0 + j)] = x[q];
      d.pos[2 * (n0 + j) + 1] = y[q];
    }
  }
}

// ---------------------------------------------------------------- general rods: CTA per rod
__global__ void k_node(const RDesc* __restrict__ D, const int* __restrict__ off, int n,
                       const int* __restrict__ tdev) {
  extern __shared__ float sm[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int comp = d.generic_comp[blockIdx.x - off[r]];
  const int n0 = d.comp_n[comp], nn = d.comp_n[comp + 1] - n0;
  const int e0 = d.comp_e[comp], ne = d.comp_e[comp + 1] - e0;
  const int b0 = d.comp_b[comp], nb = d.comp_b[comp + 1] - b0;
  float* px = sm;
  float* py = px + d.max_comp_nodes;
  float* th = py + d.max_comp_nodes;
  float* l0 = th + d.max_comp_edges;
  float* fx = l0 + d.max_comp_edges;
  float* fy = fx + d.max_comp_edges;
  float* corr = fy + d.max_comp_edges;
  float* ra = corr + d.max_comp_pairs;
  float* kb = ra + d.max_comp_pairs;
  const int tid = threadIdx.x, bd = blockDim.x;
  const int t = *tdev;

  for (int b = tid; b < nb; b += bd) {
    ra[b] = rest_angle(d, b0 + b, t);
    kb[b] = d.kb[b0 + b];
  }
  for (int e = tid; e < ne; e += bd) {
    th[e] = d.theta[e0 + e];
    l0[e] = d.rest_len[e0 + e];
  }
  for (int i = tid; i < nn; i += bd) {
    px[i] = d.pos[2 * (n0 + i)];
    py[i] = d.pos[2 * (n0 + i) + 1];
  }
  __syncthreads();

  const bool cosserat = d.solver == 1;
  for (int it = 0; it < d.cycles; ++it) {
    // theta pass over bending pairs (pbd.py:23-49; stable_cosserat.py:55-82)
    for (int b = tid; b < nb; b += bd) {
      const int ein = d.bpairs[2 * (b0 + b)] - e0, eout = d.bpairs[2 * (b0 + b) + 1] - e0;
      corr[b] = bend_corr(th[ein], th[eout], ra[b], kb[b]);
    }
    __syncthreads();
    for (int e = tid; e < ne; e += bd) {
      const int ge = e0 + e;
      float acc = 0.0f;
      for (int j = d.ep_off[ge]; j < d.ep_off[ge + 1]; ++j) {
        const int code = d.ep_idx[j];
        const float c = corr[(code >> 1) - b0];
        acc = (code & 1) ? acc + (-c) : acc + c;
      }
      if (cosserat) {
        const int s = d.pairs[2 * ge] - n0, g = d.pairs[2 * ge + 1] - n0;
        const float2 r = min_image(px[g], py[g], px[s], py[s], (float)d.W, (float)d.H);
        th[e] = cos_pull(th[e] + acc / d.edeg[ge], r.x, r.y);
      } else {
        th[e] = th[e] + (acc / d.edeg[ge]) * 1.8f;
      }
    }
    __syncthreads();
    // position pass over edges (pbd.py:51-89; stable_cosserat.py:84-119)
    for (int e = tid; e < ne; e += bd) {
      const int s = d.pairs[2 * (e0 + e)] - n0, g = d.pairs[2 * (e0 + e) + 1] - n0;
      if (cosserat) {
        const float2 r = min_image(px[g], py[g], px[s], py[s], (float)d.W, (float)d.H);
        float sn, cs;
        sincosf(th[e], &sn, &cs);
        const float kl = d.k_stretch / l0[e];
        fx[e] = kl * (r.x / l0[e] - cs);
        fy[e] = kl * (r.y / l0[e] - sn);
      } else {
        const float2 f = edge_force(d, th[e], l0[e], px[s], py[s], px[g], py[g]);
        fx[e] = f.x;
        fy[e] = f.y;
      }
    }
    __syncthreads();
    if (cosserat) {
      // implicit update with inertia: per node (w (y0 - x) + sum +-f_e) / (w + sum k_s/l_e^2),
      // y0 = the positions this kernel started from (still in global memory)
      const float w = d.cos_w;
      for (int i = tid; i < nn; i += bd) {
        const int gi = n0 + i;
        float ax = w * (d.pos[2 * gi] - px[i]), ay = w * (d.pos[2 * gi + 1] - py[i]), hh = w;
        for (int j = d.ne_off[gi]; j < d.ne_off[gi + 1]; ++j) {
          const int code = d.ne_idx[j];
          const int e = (code >> 1) - e0;
          if (code & 1) {
            ax = ax + (-fx[e]);
            ay = ay + (-fy[e]);
          } else {
            ax = ax + fx[e];
            ay = ay + fy[e];
          }
          hh = hh + d.k_stretch / (l0[e] * l0[e]);
        }
        px[i] = px[i] + ax / hh;
        py[i] = py[i] + ay / hh;
      }
      __syncthreads();
      continue;
    }
    for (int i = tid; i < nn; i += bd) {
      const int gi = n0 + i;
      float ax = 0.0f, ay = 0.0f;
      for (int j = d.ne_off[gi]; j < d.ne_off[gi + 1]; ++j) {
        const int code = d.ne_idx[j];
        const int e = (code >> 1) - e0;
        if (code & 1) {
          ax = ax + (-fx[e]);
          ay = ay + (-fy[e]);
        } else {
          ax = ax + fx[e];
          ay = ay + fy[e];
        }
      }
      const float dg = d.ndeg[gi];
      px[i] = px[i] + ax / dg;
      py[i] = py[i] + ay / dg;
    }
    __syncthreads();
  }

  for (int e = tid; e < ne; e += bd) d.theta[e0 + e] = th[e];
  for (int i = tid; i < nn; i += bd) {
    d.pos[2 * (n0 + i)] = px[i];
    d.pos[2 * (n0 + i) + 1] = py[i];
  }
}

void launch_predict(const Launch& L) { k_predict<<<L.grid, kNodeThreads, 0, L.s>>>(L.d, L.off, L.n); }
void launch_steric(const Launch& L) { k_steric<<<L.grid, kNodeThreads, 0, L.s>>>(L.d, L.off, L.n); }
void launch_stencil(const Launch& L) { k_stencil<<<L.grid, kNodeThreads, 0, L.s>>>(L.d, L.off, L.n); }
// 8 IB points (16 lanes each) per 128-thread CTA (measured 0.5% faster steps than 16 per 256)
void launch_stencil16(const Launch& L) { k_stencil16<<<L.grid, 128, 0, L.s>>>(L.d, L.off, L.n); }
void launch_node(const Launch& L, const int* tdev, size_t smem, int bs) {
  k_node<<<L.grid, bs, smem, L.s>>>(L.d, L.off, L.n, tdev);
}
void launch_chain(const Launch& L, const int* tdev, int slots) {
  switch (slots) {
    case 1: k_chain<1><<<L.grid, 32 * kChainWarps, 0, L.s>>>(L.d, L.off, L.n, tdev); break;
    case 2: k_chain<2><<<L.grid, 32 * kChainWarps, 0, L.s>>>(L.d, L.off, L.n, tdev); break;
    case 4: k_chain<4><<<L.grid, 32 * kChainWarps, 0, L.s>>>(L.d, L.off, L.n, tdev); break;
    default: k_chain<8><<<L.grid, 32 * kChainWarps, 0, L.s>>>(L.d, L.off, L.n, tdev); break;
  }
}
cudaError_t node_set_smem(size_t bytes) {
  return cudaFuncSetAttribute(k_node, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace mc
