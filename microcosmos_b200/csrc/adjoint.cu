// Reverse-mode derivative of a rollout (the gradient path behind the autograd bindings).
//
// A gradient plan wraps one forward plan (the same kernels as mc_rollout) and adds:
//   * checkpoints of the state every S steps during the forward rollout (S ~ sqrt(T));
//   * per segment, a recompute of its S step inputs with the forward plan;
//   * per step, in reverse, a "tape" recompute of the step's intermediates (steric-corrected
//     prediction, the PBD iterates, the IB stencils and multi-direct forcing iterates) and
//     the adjoint kernels of stream+collide, IB, PBD and steric.
//
// Derivative conventions are those jax.grad applies to the reference: the Peskin stencil
// positions are stop_gradient-ed (src/microcosmos/solver/fluid.py:237-239), floor has
// derivative 0, mod derivative 1, max/min pass the cotangent to the selected argument and
// split it on ties.  Every scatter-add of the adjoint (IB spread, node reaction, steric
// sample weights) goes through a cell-sorted list (CSR) whose entries are ordered by their
// flat index, so sums are taken in a fixed order and gradients are reproducible bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/microcosmos_b200.h"
#include "lbm_cell.cuh"
#include "mc_internal.cuh"

namespace mc {
// Inside a rollout of a one-rollout plan: the current populations in fields.f_grid layout
// written to dst, the rollout left as it is (runtime.cu).
mc_status rollout_snapshot_f(mc_plan* p, float* dst, cudaStream_t s);
}  // namespace mc

namespace {

constexpr int kMaxKK = 64;       // stencil entries per node (kernel size <= 8)
constexpr int kScanChunk = 4096;  // cells per scan block (1024 threads x 4)
constexpr int kPbdThreads = 128;  // threads per rod component in the PBD kernels

// Per-step inputs of one reverse step, read on the device so that the same CUDA graph
// replays every step of a segment (sa[*jp], jp counts down).
struct StepArgs {
  int t;
  const float* pos;
  const float* vel;
  const float* th;
  const float* f;
  const float* V;
  float* lf_in;
  float* lf_out;
};

struct AD {
  int H, W, N, E, B, HW, C, iters, K, KK, steric, fluid, nskip, has_act;
  int lH, lW, lHW;  // the fluid lattice (f_grid (9, lH, lW)); H, W, HW: the domain grid
  int solver;  // MC_SOLVER_PBD or MC_SOLVER_COSSERAT
  int force_clamp;  // enable_force_clamp: F = F_raw * clamp factor of F_raw
  int NI;      // IB points: N, or 2N with synthetic pairs (point p < N: node p, + side; else node p - N, - side)
  float syn_w, syn_ms;  // synthetic_node_width and the mean lattice scale it is multiplied by
  float dt, damp, st_strength, sigma, scatter, kstretch, kshear, vmax, relax, mass, wp, wm, cp, cm;
  float cos_w;  // stable-Cosserat inertia weight 1 / solver_dt^2
  float scx, scy, sdtx, sdty;
  // topology
  const int2* pairs;
  const int2* bpairs;
  const int* n_start;  // node -> incident edges: entry = e * 2 + role (0: src, 1: tgt)
  const int* n_list;
  const int* e_start;  // edge -> incident bending pairs: entry = b * 2 + role (0: e_in, 1: e_out)
  const int* e_list;
  // rod components (connected by edges): their nodes, edges and bending pairs, ascending
  int ncomp;
  const int* c_nstart;
  const int* c_nodes;
  const int* c_estart;
  const int* c_edges;
  const int* c_bstart;
  const int* c_bps;
  // per-step inputs of the reverse step being replayed
  const StepArgs* sa;
  int* jp;
  const float* ndeg;
  const float* edeg;
  const float* rest_len;
  const float* kb;
  const float* rest_static;
  const float* act_c;
  const float* act_amp;
  const float* act_om;
  const float* act_ph;
  // tape
  float* rest;   // (B) rest angles of the current step
  float2* pred0;  // (N)
  float2* pp;     // (C+1) x N PBD iterates
  float* tt;      // (C+1) x E
  int* ib_idx;    // NI x KK
  float* ib_w;    // NI x KK
  float2* sraw;   // iters x NI
  float2* s_tmp;  // NI
  float* uc;      // 2 x lHW
  float* inv;     // lHW
  // CSR over cells
  int* cnt;    // max(HW, lHW) (all zero between builds)
  int* start;  // max(HW, lHW) + 1
  int* bsum;   // scan block sums
  int* ent;    // entries
  int* touched;   // cells with at least one entry (any order), M entries at most
  int* ntouched;  // their count
  int max_entries;
  // adjoint
  float* lf0p;   // 9 x lHW
  float* lv;     // 2 x lHW
  float* lrho;   // lHW
  float* luc;    // 2 x lHW
  float2* lnv;   // NI
  float2* lprev;  // N
  float2* lpos;   // N   (state cotangent)
  float2* lvel;   // N
  float* lth;     // E
  float2* lp[2];  // N
  float* lt[2];   // E
  float2* lcur;   // E
  float* lthn;    // E
  float* gb;      // B
  float2* ly;     // N  stable-Cosserat: cotangent of the prediction the iterations pull toward
  float2* lfn;    // N  stable-Cosserat: cotangent of a node's summed force
  float* lhn;     // N  stable-Cosserat: cotangent of a node's summed stiffness
  float* rest_acc;  // B (this step)
  float* d_c;
  float* d_amp;
  float* d_ph;
  float* d_om;
  float* d_rest;
  float* d_len;
  float* d_kb;
  // steric
  int* st_cell;    // 16 N
  float* st_val;   // 16 N
  float2* lpred1;  // N
  float2* lpred0p;  // N
  float* lV;       // HW
  float* ctmp;     // HW
  float* ldep;     // HW
};

__device__ __forceinline__ float dmaxf(float x, float c) { return x > c ? 1.0f : (x == c ? 0.5f : 0.0f); }

// cotangent of (x, y) through (x c, y c), c = min(1, vmax / (sqrt(x^2+y^2+eps)+eps))
__device__ __forceinline__ float2 clamp_vjp(float x, float y, float vmax, float gx, float gy) {
  const float mag = sqrtf((x * x + y * y) + MC_EPSIL);
  const float a = vmax / (mag + MC_EPSIL);
  const float c = mc::min_prop(1.0f, a);
  const float sel = a < 1.0f ? 1.0f : (a == 1.0f ? 0.5f : 0.0f);
  const float gc = x * gx + y * gy;
  const float da = -vmax / ((mag + MC_EPSIL) * (mag + MC_EPSIL));
  const float k = ((gc * sel) * da) / mag;
  return make_float2(c * gx + k * x, c * gy + k * y);
}

__device__ __forceinline__ int cell_of(int y, int x, int H, int W) { return mc::imod_floor(y, H) * W + mc::imod_floor(x, W); }

// map_coordinates(order=1, mode="wrap") of field V at (yy, xx)
__device__ __forceinline__ float sample_wrap(const float* V, int H, int W, float yy, float xx) {
  const float ly = floorf(yy), lx = floorf(xx);
  const float ty = yy - ly, tx = xx - lx;
  const float wy0 = 1.0f - ty, wx0 = 1.0f - tx;
  const int iy = (int)ly, ix = (int)lx;
  const int y0 = mc::imod_floor(iy, H), y1 = mc::imod_floor(iy + 1, H);
  const int x0 = mc::imod_floor(ix, W), x1 = mc::imod_floor(ix + 1, W);
  float acc = (wy0 * wx0) * V[y0 * W + x0];
  acc = acc + (wy0 * tx) * V[y0 * W + x1];
  acc = acc + (ty * wx0) * V[y1 * W + x0];
  acc = acc + (ty * tx) * V[y1 * W + x1];
  return acc;
}

// ------------------------------------------------------------------ tape: prediction + steric
__global__ void k_rest(AD d) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.B) return;
  const int t = d.sa[*d.jp].t;
  float r;
  if (d.has_act) {
    const float arg = d.act_om[b] * (float)t + d.act_ph[b];
    r = d.act_c[b] + d.act_amp[b] * sinf(arg);
  } else {
    r = d.rest_static[b];
  }
  d.rest[b] = r;
  d.rest_acc[b] = 0.0f;
}

__global__ void k_pred(AD d) {
  const StepArgs a = d.sa[*d.jp];
  const float2* __restrict__ pos = reinterpret_cast<const float2*>(a.pos);
  const float2* __restrict__ vel = reinterpret_cast<const float2*>(a.vel);
  const float* __restrict__ theta = a.th;
  const float* __restrict__ V = a.V;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.E) d.tt[i] = theta[i];
  if (i >= d.N) return;
  const float2 p = pos[i], v = vel[i];
  float2 q = make_float2(p.x + (v.x * d.damp) * d.dt, p.y + (v.y * d.damp) * d.dt);
  d.pred0[i] = q;
  if (d.steric) {
    const float Wf = (float)d.W, Hf = (float)d.H;
    const float x = mc::fmod_floor(q.x, Wf), y = mc::fmod_floor(q.y, Hf);
    const float e = 0.5f, den = 1.0f;
    const float gx = (sample_wrap(V, d.H, d.W, y, x + e) - sample_wrap(V, d.H, d.W, y, x - e)) / den;
    const float gy = (sample_wrap(V, d.H, d.W, y + e, x) - sample_wrap(V, d.H, d.W, y - e, x)) / den;
    float fx = -gx, fy = -gy;
    if (d.nskip > 0) {
      const float inv2s2 = 2.0f * d.sigma * d.sigma;
      const float norm = (float)(2.0 * M_PI) * d.sigma * d.sigma;
      float ax = 0.0f, ay = 0.0f;
      // the neighbours' wrapped predictions, recomputed from their positions and velocities
      for (int o = -d.nskip; o <= d.nskip; ++o) {
        const int j = i + o;
        if (j < 0 || j >= d.N) continue;
        const float2 pj0 = pos[j], vj = vel[j];
        const float qx = pj0.x + (vj.x * d.damp) * d.dt, qy = pj0.y + (vj.y * d.damp) * d.dt;
        const float2 r = mc::min_image(x, y, mc::fmod_floor(qx, Wf), mc::fmod_floor(qy, Hf), Wf, Hf);
        const float d2 = r.x * r.x + r.y * r.y;
        const float K = expf(-d2 / inv2s2) / norm;
        ax = ax + K * r.x;
        ay = ay + K * r.y;
      }
      const float pre = d.scatter / (d.sigma * d.sigma);
      fx = fx - pre * ax;
      fy = fy - pre * ay;
    }
    q.x = q.x + (fx * d.st_strength) * d.dt;
    q.y = q.y + (fy * d.st_strength) * d.dt;
  }
  d.pp[i] = q;
}

// ------------------------------------------------------------------ tape: PBD iterates (one CTA)
// bending correction of pair (e_in, e_out) from the angles th_in = theta[e_in], th_out = theta[e_out]
__device__ __forceinline__ float bend_corr_v(float th_in, float th_out, float rest, float kb) {
  const float pi = (float)M_PI;
  const float diff = mc::fmod_floor((th_out - th_in) + pi, (float)(2.0 * M_PI)) - pi;
  return ((diff - rest) * kb) * 0.5f;
}

__device__ __forceinline__ float bend_corr(const AD& d, const float* th, int b) {
  const int2 bp = d.bpairs[b];
  return bend_corr_v(th[bp.x], th[bp.y], d.rest[b], d.kb[b]);
}

// stretch + shear force of an edge from its endpoints a = p[src], b = p[tgt], its new angle
// and its rest length
__device__ __forceinline__ float2 edge_force_v(const AD& d, float2 a, float2 b, float thn, float L0) {
  const float tx = cosf(thn) * L0, ty = sinf(thn) * L0;
  const float2 cur = mc::min_image(b.x, b.y, a.x, a.y, (float)d.W, (float)d.H);
  const float L = sqrtf(cur.x * cur.x + cur.y * cur.y);
  const float m = mc::max_prop(L, 1e-8f);
  const float sx = (cur.x / m) * (L - L0), sy = (cur.y / m) * (L - L0);
  const float shx = (cur.x - tx) - sx, shy = (cur.y - ty) - sy;
  return make_float2(((sx + shx * d.kshear) * d.kstretch) * 0.5f, ((sy + shy * d.kshear) * d.kstretch) * 0.5f);
}

__device__ __forceinline__ float2 edge_force(const AD& d, const float2* p, float thn, int e) {
  const int2 pr = d.pairs[e];
  return edge_force_v(d, p[pr.x], p[pr.y], thn, d.rest_len[e]);
}

// Rod components whose edges, nodes and bending pairs fit one per thread, with at most
// kPbdGather incidences each (chains: 2), keep their topology in registers for all C
// iterations: each phase of an iteration then waits for one round of independent loads of
// the iterates instead of a chain of index loads.  Same operands and summation order as the
// general loops below, so the same bits.
constexpr int kPbdGather = 4;

struct PbdEdgeReg {  // an edge and its bending pairs (edge pass of the forward)
  int e = -1, nb = 0;
  int2 bp[kPbdGather];
  float rest[kPbdGather], kb[kPbdGather];
  bool neg[kPbdGather];
  float edeg = 1.0f;
};

struct PbdNodeReg {  // a node and its incident edges
  int n = -1, ne = 0;
  int e[kPbdGather];
  int2 pr[kPbdGather];
  float L0[kPbdGather];
  bool neg[kPbdGather];
  float ndeg = 1.0f;
};

// loads thread t's edge / node of component c; false when a list is too long for registers
__device__ __forceinline__ bool pbd_load_edge(const AD& d, int ie, int eb, PbdEdgeReg& r) {
  if (ie >= eb) return true;
  r.e = d.c_edges[ie];
  const int qa = d.e_start[r.e], qb = d.e_start[r.e + 1];
  r.nb = qb - qa;
  if (r.nb > kPbdGather) return false;
#pragma unroll
  for (int q = 0; q < kPbdGather; ++q)
    if (q < r.nb) {
      const int en = d.e_list[qa + q];
      r.bp[q] = d.bpairs[en >> 1];
      r.rest[q] = d.rest[en >> 1];
      r.kb[q] = d.kb[en >> 1];
      r.neg[q] = en & 1;
    }
  r.edeg = d.edeg[r.e];
  return true;
}

__device__ __forceinline__ bool pbd_load_node(const AD& d, int in, int nb, PbdNodeReg& r) {
  if (in >= nb) return true;
  r.n = d.c_nodes[in];
  const int qa = d.n_start[r.n], qb = d.n_start[r.n + 1];
  r.ne = qb - qa;
  if (r.ne > kPbdGather) return false;
#pragma unroll
  for (int q = 0; q < kPbdGather; ++q)
    if (q < r.ne) {
      const int en = d.n_list[qa + q];
      r.e[q] = en >> 1;
      r.pr[q] = d.pairs[en >> 1];
      r.L0[q] = d.rest_len[en >> 1];
      r.neg[q] = en & 1;
    }
  r.ndeg = d.ndeg[r.n];
  return true;
}

// one CTA per rod component: the components never interact in the PBD passes
__global__ void __launch_bounds__(kPbdThreads) k_pbd_fwd(AD d) {
  const int c = blockIdx.x;
  const int ea = d.c_estart[c], eb = d.c_estart[c + 1], na = d.c_nstart[c], nb = d.c_nstart[c + 1];
  {
    PbdEdgeReg re;
    PbdNodeReg rn;
    bool ok = eb - ea <= (int)blockDim.x && nb - na <= (int)blockDim.x;
    if (ok) ok = pbd_load_edge(d, ea + threadIdx.x, eb, re) && pbd_load_node(d, na + threadIdx.x, nb, rn);
    if (__syncthreads_and(ok)) {
      for (int k = 0; k < d.C; ++k) {
        const float* th = d.tt + (size_t)k * d.E;
        float* thn = d.tt + (size_t)(k + 1) * d.E;
        if (re.e >= 0) {
          float tin[kPbdGather], tout[kPbdGather];
#pragma unroll
          for (int q = 0; q < kPbdGather; ++q)
            if (q < re.nb) {
              tin[q] = th[re.bp[q].x];
              tout[q] = th[re.bp[q].y];
            }
          const float th_e = th[re.e];
          float acc = 0.0f;
#pragma unroll
          for (int q = 0; q < kPbdGather; ++q)
            if (q < re.nb) {
              const float cr = bend_corr_v(tin[q], tout[q], re.rest[q], re.kb[q]);
              acc = acc + (re.neg[q] ? -cr : cr);
            }
          thn[re.e] = th_e + (acc / re.edeg) * 1.8f;
        }
        __syncthreads();
        const float2* p = d.pp + (size_t)k * d.N;
        float2* pn = d.pp + (size_t)(k + 1) * d.N;
        if (rn.n >= 0) {
          float2 pa[kPbdGather], pb[kPbdGather];
          float tq[kPbdGather];
#pragma unroll
          for (int q = 0; q < kPbdGather; ++q)
            if (q < rn.ne) {
              pa[q] = p[rn.pr[q].x];
              pb[q] = p[rn.pr[q].y];
              tq[q] = thn[rn.e[q]];
            }
          const float2 self = p[rn.n];
          float ax = 0.0f, ay = 0.0f;
#pragma unroll
          for (int q = 0; q < kPbdGather; ++q)
            if (q < rn.ne) {
              const float2 f = edge_force_v(d, pa[q], pb[q], tq[q], rn.L0[q]);
              if (rn.neg[q]) {
                ax = ax + (-f.x);
                ay = ay + (-f.y);
              } else {
                ax = ax + f.x;
                ay = ay + f.y;
              }
            }
          pn[rn.n] = make_float2(self.x + ax / rn.ndeg, self.y + ay / rn.ndeg);
        }
        __syncthreads();
      }
      return;
    }
  }
  for (int k = 0; k < d.C; ++k) {
    const float* th = d.tt + (size_t)k * d.E;
    float* thn = d.tt + (size_t)(k + 1) * d.E;
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      float acc = 0.0f;
      for (int q = d.e_start[e]; q < d.e_start[e + 1]; ++q) {
        const int en = d.e_list[q];
        const float c = bend_corr(d, th, en >> 1);
        acc = acc + ((en & 1) ? -c : c);
      }
      thn[e] = th[e] + (acc / d.edeg[e]) * 1.8f;
    }
    __syncthreads();
    const float2* p = d.pp + (size_t)k * d.N;
    float2* pn = d.pp + (size_t)(k + 1) * d.N;
    for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
      const int n = d.c_nodes[in];
      float ax = 0.0f, ay = 0.0f;
      for (int q = d.n_start[n]; q < d.n_start[n + 1]; ++q) {
        const int en = d.n_list[q];
        const int e = en >> 1;
        const float2 f = edge_force(d, p, thn[e], e);
        if (en & 1) {
          ax = ax + (-f.x);
          ay = ay + (-f.y);
        } else {
          ax = ax + f.x;
          ay = ay + f.y;
        }
      }
      const float dg = d.ndeg[n];
      pn[n] = make_float2(p[n].x + ax / dg, p[n].y + ay / dg);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ tape: IB stencils
// The stencil of IB point n at the step's final PBD positions; with synthetic pairs the
// point is offset by +-syn_w * syn_ms along the normal of its node's chain tangent (the sum
// of its edges' min-image vectors, src roles first, as the forward computes it).  The
// positions are stop_gradient-ed: constants of the derivative.
__global__ void k_ib_weights(AD d) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.NI) return;
  const int gi = n < d.N ? n : n - d.N;
  const float2* pc = d.pp + (size_t)d.C * d.N;
  const float2 p = pc[gi];
  float x = p.x * d.scx, y = p.y * d.scy;
  if (d.NI > d.N) {
    float tx = 0.0f, ty = 0.0f;
    for (int q = d.n_start[gi]; q < d.n_start[gi + 1]; ++q) {
      const int2 pr = d.pairs[d.n_list[q] >> 1];
      const float2 ev = mc::min_image(pc[pr.y].x, pc[pr.y].y, pc[pr.x].x, pc[pr.x].y, (float)d.W, (float)d.H);
      tx = tx + ev.x;
      ty = ty + ev.y;
    }
    const float nrm = sqrtf((tx * tx + ty * ty) + MC_EPSIL);
    const float ux = tx / nrm, uy = ty / nrm;
    const float ox = (d.syn_w * (-uy)) * d.syn_ms, oy = (d.syn_w * ux) * d.syn_ms;
    if (n < d.N) {
      x = x + ox;
      y = y + oy;
    } else {
      x = x - ox;
      y = y - oy;
    }
  }
  const int K = d.K;
  const float half = (float)((K - 1) / 2);
  const float hw = (float)K / 2.0f;
  const float sx = floorf(x) - half, sy = floorf(y) - half;
  float w[kMaxKK];
  float s = 0.0f;
  for (int a = 0; a < K; ++a) {
    for (int b = 0; b < K; ++b) {
      const float nx = sx + (float)a, ny = sy + (float)b;
      const float rx = fabsf(nx - x) / hw, ry = fabsf(ny - y) / hw;
      const float px = rx <= 2.0f ? 0.25f * (1.0f + cosf(((float)M_PI * rx) / 2.0f)) : 0.0f;
      const float py = ry <= 2.0f ? 0.25f * (1.0f + cosf(((float)M_PI * ry) / 2.0f)) : 0.0f;
      const int q = a * K + b;
      w[q] = px * py;
      s = s + w[q];
      d.ib_idx[(size_t)n * d.KK + q] = cell_of((int)ny, (int)nx, d.lH, d.lW);
    }
  }
  for (int q = 0; q < d.KK; ++q) d.ib_w[(size_t)n * d.KK + q] = w[q] / (s + MC_EPSIL);
}

// ------------------------------------------------------------------ CSR over cells
__global__ void k_csr_count(const int* __restrict__ cells, int M, int* cnt) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < M) atomicAdd(cnt + cells[e], 1);
}

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem[lane] = w;
  }
  __syncthreads();
  const int before = (wid > 0 ? smem[wid - 1] : 0) + x - v;
  total = smem[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(1024) k_scan1(const int* __restrict__ cnt, int n, int* start, int* bsum) {
  __shared__ int smem[32];
  const int base = blockIdx.x * kScanChunk + threadIdx.x * 4;
  int v[4];
  int s = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    v[j] = base + j < n ? cnt[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, smem, total);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < n) start[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan2(int* bsum, int nb) {
  __shared__ int smem[32];
  const int base = threadIdx.x * 4;
  int v[4];
  int s = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    v[j] = base + j < nb ? bsum[base + j] : 0;
    s += v[j];
  }
  int total;
  int run = block_exclusive_scan(s, smem, total);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < nb) bsum[base + j] = run;
    run += v[j];
  }
}

__global__ void k_scan3(int* start, const int* __restrict__ bsum, int n, int M) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) start[i] += bsum[i / kScanChunk];
  if (i == 0) start[n] = M;
}

__global__ void k_csr_fill(const int* __restrict__ cells, int M, const int* __restrict__ start, int* cnt, int* ent) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M) return;
  const int c = cells[e];
  const int slot = start[c] + atomicSub(cnt + c, 1) - 1;  // leaves cnt at zero
  ent[slot] = e;
}

// entries of each cell in increasing flat index (the order np.add.at applies them)
// the cells that received entries, compacted (their order does not matter: every
// per-cell kernel below writes only its own cell)
__global__ void k_csr_touched(const int* __restrict__ start, int n, int* touched, int* ntouched) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n || start[c + 1] == start[c]) return;
  touched[atomicAdd(ntouched, 1)] = c;
}

__global__ void k_csr_sort(const int* __restrict__ start, const int* __restrict__ touched,
                           const int* __restrict__ ntouched, int* ent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *ntouched) return;
  const int c = touched[i];
  const int a = start[c], b = start[c + 1];
  for (int i = a + 1; i < b; ++i) {
    const int v = ent[i];
    int j = i - 1;
    while (j >= a && ent[j] > v) {
      ent[j + 1] = ent[j];
      --j;
    }
    ent[j + 1] = v;
  }
}

// ------------------------------------------------------------------ tape: macroscopic + IB iterations
__global__ void k_macro(AD d) {
  const float* __restrict__ f = d.sa[*d.jp].f;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.lHW) return;
  float r = mc::max_prop(f[c], MC_EPSIL);
  float fv[9];
  fv[0] = r;
#pragma unroll
  for (int i = 1; i < 9; ++i) {
    fv[i] = mc::max_prop(f[(size_t)i * d.lHW + c], MC_EPSIL);
    r = r + fv[i];
  }
  const float rho = mc::max_prop(r, 0.1f);
  const float ux = (((((fv[1] - fv[3]) + fv[5]) - fv[6]) - fv[7]) + fv[8]) / rho;
  const float uy = (((((fv[2] - fv[4]) + fv[5]) + fv[6]) - fv[7]) - fv[8]) / rho;
  const float c1 = mc::clamp_factor(ux, uy, d.vmax);
  d.uc[c] = ux * c1;
  d.uc[d.lHW + c] = uy * c1;
  float cov = 0.0f;
  for (int q = d.start[c]; q < d.start[c + 1]; ++q) cov = cov + d.ib_w[d.ent[q]];
  d.inv[c] = 1.0f / mc::max_prop(cov, 1.0f);
}

__global__ void k_ib_interp(AD d, int it) {
  const float2* __restrict__ prev = reinterpret_cast<const float2*>(d.sa[*d.jp].pos);
  int n = blockIdx.x * blockDim.x + threadIdx.x;  // IB point
  if (n >= d.NI) return;
  const int gi = n < d.N ? n : n - d.N;
  float ix = 0.0f, iy = 0.0f;
  for (int q = 0; q < d.KK; ++q) {
    const int c = d.ib_idx[(size_t)n * d.KK + q];
    const float w = d.ib_w[(size_t)n * d.KK + q];
    ix = ix + d.uc[c] * w;
    iy = iy + d.uc[d.lHW + c] * w;
  }
  const float2 pc = d.pp[(size_t)d.C * d.N + gi], p0 = prev[gi];
  const float v1x = (pc.x - p0.x) / d.dt, v1y = (pc.y - p0.y) / d.dt;
  const float nvx = (v1x * d.scx) * d.dt, nvy = (v1y * d.scy) * d.dt;
  const float sx = (nvx - ix) * d.relax, sy = (nvy - iy) * d.relax;
  d.sraw[(size_t)it * d.NI + n] = make_float2(sx, sy);
  const float cf = mc::clamp_factor(sx, sy, d.vmax);
  d.s_tmp[n] = make_float2(sx * cf, sy * cf);
}

__global__ void k_ib_spread(AD d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *d.ntouched) return;
  const int c = d.touched[i];
  const int a = d.start[c], b = d.start[c + 1];
  float ax = 0.0f, ay = 0.0f;
  for (int q = a; q < b; ++q) {
    const int e = d.ent[q];
    const float w = d.ib_w[e];
    const float2 s = d.s_tmp[e / d.KK];
    ax = ax + s.x * w;
    ay = ay + s.y * w;
  }
  const float iv = d.inv[c];
  d.uc[c] = d.uc[c] + ax * iv;
  d.uc[d.lHW + c] = d.uc[d.lHW + c] + ay * iv;
}

// ------------------------------------------------------------------ adjoint: stream + collide + F
__constant__ float kW9[9] = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                             1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
// opposite D2Q9 direction {0, 3, 4, 1, 2, 7, 8, 5, 6} as a compile-time function: in the
// unrolled population loops the index folds to a constant and the per-cell arrays stay in
// registers (a table lookup would put them in local memory)
__device__ __forceinline__ constexpr int opp9(int i) { return i == 0 ? 0 : (i <= 4 ? (i + 1) % 4 + 1 : (i - 3) % 4 + 5); }

__global__ void k_lbm_adj1(AD d) {
  const StepArgs a = d.sa[*d.jp];
  const float* __restrict__ f = a.f;
  const float* __restrict__ lfn = a.lf_in;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.lHW) return;
  const int y = c / d.lW, x = c - y * d.lW;
  float f0[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) f0[i] = mc::max_prop(f[(size_t)i * d.lHW + c], MC_EPSIL);
  float rr = f0[0];
#pragma unroll
  for (int i = 1; i < 9; ++i) rr = rr + f0[i];
  const float rho = mc::max_prop(rr, 0.1f);
  const float ux = ((((f0[1] - f0[3]) + f0[5]) - f0[6]) - f0[7]) + f0[8];
  const float uy = ((((f0[2] - f0[4]) + f0[5]) + f0[6]) - f0[7]) - f0[8];
  const float c1 = mc::clamp_factor(ux / rho, uy / rho, d.vmax);
  const float vx = (ux / rho) * c1, vy = (uy / rho) * c1;
  const float u5x = d.uc[c], u5y = d.uc[d.lHW + c];
  const float c2 = mc::clamp_factor(u5x, u5y, d.vmax);
  const float ucx = u5x * c2, ucy = u5y * c2;
  const float Frx = (ucx - vx) * rho, Fry = (ucy - vy) * rho;
  float Fx = Frx, Fy = Fry;
  if (d.force_clamp) {
    const float c3 = mc::clamp_factor(Frx, Fry, d.vmax);
    Fx = Frx * c3;
    Fy = Fry * c3;
  }
  // forward collide for the floor masks
  float post[9], us_x, us_y;
  mc::collide(f0, rho, vx, vy, Fx, Fy, d.wp, d.wm, d.cp, d.cm, post, us_x, us_y);
  // recompute the unfloored collide output for the first mask
  const float half = 0.5f;
  const float usx = vx + half * Fx / rho, usy = vy + half * Fy / rho;
  const float usq = usx * usx + usy * usy;
  const float udF = usx * Fx + usy * Fy;
  float eu[9], eF[9], feq[9], raw[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    eu[i] = (float)mc::kEx[i] * usx + (float)mc::kEy[i] * usy;
    eF[i] = (float)mc::kEx[i] * Fx + (float)mc::kEy[i] * Fy;
    feq[i] = (rho * kW9[i]) * (((1.0f + 3.0f * eu[i]) + 4.5f * (eu[i] * eu[i])) - 1.5f * usq);
    raw[i] = kW9[i] * (3.0f * (eF[i] - udF) + (9.0f * eu[i]) * eF[i]);
  }
  float g[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int o = opp9(i);
    const float pr = f0[i] - d.wp * (half * (f0[i] + f0[o]) - half * (feq[i] + feq[o])) -
                     d.wm * (half * (f0[i] - f0[o]) - half * (feq[i] - feq[o]));
    const float src = d.cp * (half * (raw[i] + raw[o])) + d.cm * (half * (raw[i] - raw[o]));
    const int xn = x + mc::kEx[i], yn = y + mc::kEy[i];
    const float lin = lfn[(size_t)i * d.lHW + cell_of(yn, xn, d.lH, d.lW)];
    g[i] = (lin * dmaxf(post[i], MC_EPSIL)) * dmaxf(pr + src, MC_EPSIL);
  }
  float lf0[9];
  float lrho = 0.0f, lusx = 0.0f, lusy = 0.0f, lFx = 0.0f, lFy = 0.0f;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int o = opp9(i);
    const float gp = half * (g[i] + g[o]), gm = half * (g[i] - g[o]);
    lf0[i] = g[i] - d.wp * gp - d.wm * gm;
    const float lfeq = d.wp * gp + d.wm * gm;
    const float lraw = (1.0f - half * d.wp) * gp + (1.0f - half * d.wm) * gm;
    const float ex = (float)mc::kEx[i], ey = (float)mc::kEy[i];
    lrho += lfeq * kW9[i] * (1.0f + 3.0f * eu[i] + 4.5f * eu[i] * eu[i] - 1.5f * usq);
    const float a = lfeq * rho * kW9[i];
    lusx += a * (3.0f * ex + 9.0f * eu[i] * ex - 3.0f * usx);
    lusy += a * (3.0f * ey + 9.0f * eu[i] * ey - 3.0f * usy);
    const float b = lraw * kW9[i];
    lusx += b * (-3.0f * Fx + 9.0f * eF[i] * ex);
    lusy += b * (-3.0f * Fy + 9.0f * eF[i] * ey);
    lFx += b * (3.0f * ex - 3.0f * usx + 9.0f * eu[i] * ex);
    lFy += b * (3.0f * ey - 3.0f * usy + 9.0f * eu[i] * ey);
  }
  float lvx = lusx, lvy = lusy;
  lFx += half * lusx / rho;
  lFy += half * lusy / rho;
  lrho -= half * (lusx * Fx + lusy * Fy) / (rho * rho);
  // node reaction: vel_out = vel1 - (nf / m) / sdt, nf = sum_s w F[idx] (with synthetic
  // pairs, nf of a node = 0.5 (nf of its + point + nf of its - point))
  const bool syn = d.NI > d.N;
  float rx = 0.0f, ry = 0.0f;
  for (int q = d.start[c]; q < d.start[c + 1]; ++q) {
    const int e = d.ent[q];
    const float w = d.ib_w[e];
    const int pt = e / d.KK;
    const float2 lv = d.lvel[pt < d.N ? pt : pt - d.N];
    float gx = (-lv.x / d.mass) / d.sdtx, gy = (-lv.y / d.mass) / d.sdty;
    if (syn) {
      gx = 0.5f * gx;
      gy = 0.5f * gy;
    }
    rx = rx + w * gx;
    ry = ry + w * gy;
  }
  lFx = rx + lFx;
  lFy = ry + lFy;
  if (d.force_clamp) {
    const float2 lr = clamp_vjp(Frx, Fry, d.vmax, lFx, lFy);
    lFx = lr.x;
    lFy = lr.y;
  }
  // F = (ucc - v) rho
  const float lccx = lFx * rho, lccy = lFy * rho;
  lvx -= lFx * rho;
  lvy -= lFy * rho;
  lrho += lFx * (ucx - vx) + lFy * (ucy - vy);  // through F_raw = (ucc - v) rho
  const float2 l5 = clamp_vjp(u5x, u5y, d.vmax, lccx, lccy);
  d.luc[c] = l5.x;
  d.luc[d.lHW + c] = l5.y;
  d.lv[c] = lvx;
  d.lv[d.lHW + c] = lvy;
  d.lrho[c] = lrho;
#pragma unroll
  for (int i = 0; i < 9; ++i) d.lf0p[(size_t)i * d.lHW + c] = lf0[i];
}

__global__ void k_ib_rev_node(AD d, int it) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;  // IB point
  if (n >= d.NI) return;
  float sx = 0.0f, sy = 0.0f;
  for (int q = 0; q < d.KK; ++q) {
    const int c = d.ib_idx[(size_t)n * d.KK + q];
    const float w = d.ib_w[(size_t)n * d.KK + q];
    const float iv = d.inv[c];
    sx = sx + (iv * d.luc[c]) * w;
    sy = sy + (iv * d.luc[d.lHW + c]) * w;
  }
  const float2 r = d.sraw[(size_t)it * d.NI + n];
  const float2 lr = clamp_vjp(r.x, r.y, d.vmax, sx, sy);
  float2 a = d.lnv[n];
  a.x += d.relax * lr.x;
  a.y += d.relax * lr.y;
  d.lnv[n] = a;
  d.s_tmp[n] = make_float2(-d.relax * lr.x, -d.relax * lr.y);
}

__global__ void k_ib_rev_cell(AD d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *d.ntouched) return;
  const int c = d.touched[i];
  const int a = d.start[c], b = d.start[c + 1];
  float ax = 0.0f, ay = 0.0f;
  for (int q = a; q < b; ++q) {
    const int e = d.ent[q];
    const float w = d.ib_w[e];
    const float2 s = d.s_tmp[e / d.KK];
    ax = ax + s.x * w;
    ay = ay + s.y * w;
  }
  d.luc[c] = d.luc[c] + ax;
  d.luc[d.lHW + c] = d.luc[d.lHW + c] + ay;
}

__global__ void k_lbm_adj2(AD d) {
  const StepArgs a = d.sa[*d.jp];
  const float* __restrict__ f = a.f;
  float* __restrict__ lf_out = a.lf_out;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.lHW) return;
  float f0[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) f0[i] = mc::max_prop(f[(size_t)i * d.lHW + c], MC_EPSIL);
  float rr = f0[0];
#pragma unroll
  for (int i = 1; i < 9; ++i) rr = rr + f0[i];
  const float rho = mc::max_prop(rr, 0.1f);
  const float ux = (((((f0[1] - f0[3]) + f0[5]) - f0[6]) - f0[7]) + f0[8]) / rho;
  const float uy = (((((f0[2] - f0[4]) + f0[5]) + f0[6]) - f0[7]) - f0[8]) / rho;
  const float lvx = d.lv[c] + d.luc[c], lvy = d.lv[d.lHW + c] + d.luc[d.lHW + c];
  const float2 lu = clamp_vjp(ux, uy, d.vmax, lvx, lvy);
  const float lrho = d.lrho[c] - (lu.x * ux + lu.y * uy) / rho;
  const float lraw = lrho * dmaxf(rr, 0.1f);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float l0 = d.lf0p[(size_t)i * d.lHW + c] + lraw + ((float)mc::kEx[i] * lu.x + (float)mc::kEy[i] * lu.y) / rho;
    lf_out[(size_t)i * d.lHW + c] = l0 * dmaxf(f[(size_t)i * d.lHW + c], MC_EPSIL);
  }
}

// ------------------------------------------------------------------ adjoint: node velocity / position
__global__ void k_node_adj(AD d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.E) d.lt[0][i] = d.lth[i];
  if (i >= d.N) return;
  float2 lv1 = d.lvel[i];
  if (d.fluid) {
    float2 a = d.lnv[i];
    if (d.NI > d.N) {  // both synthetic points carry the node's velocity
      const float2 b = d.lnv[i + d.N];
      a.x = a.x + b.x;
      a.y = a.y + b.y;
    }
    lv1.x = lv1.x + (a.x * d.scx) * d.dt;
    lv1.y = lv1.y + (a.y * d.scy) * d.dt;
  }
  const float2 lp = d.lpos[i];
  d.lp[0][i] = make_float2(lp.x + lv1.x / d.dt, lp.y + lv1.y / d.dt);
  d.lprev[i] = make_float2(-lv1.x / d.dt, -lv1.y / d.dt);
}

// ------------------------------------------------------------------ adjoint: PBD iterations (one CTA per rod component)
// The reverse iterations of a component whose edges, nodes and bending pairs fit one per
// thread (kPbdGather incidences at most): topology in registers, the accumulated cotangents
// of the owned edge / pair (d_len, rest_acc, d_kb) in registers and written once.  Same
// arithmetic and order as the general loops of k_pbd_rev.  All threads of the CTA call it;
// false (nothing done) when the component does not fit.
__device__ __forceinline__ bool pbd_rev_fast(const AD& d, int ea, int eb, int na, int nb, int ba, int bb, float ks,
                                             float kst) {
  const int tid = threadIdx.x;
  PbdNodeReg rn;
  int e = -1, ne3 = 0, b = -1;
  int2 pr = make_int2(0, 0), bp = make_int2(0, 0);
  float ns = 1.0f, nt = 1.0f, L0 = 0.0f, ed_x = 1.0f, ed_y = 1.0f, kbb = 0.0f, rst = 0.0f;
  int bq[kPbdGather];
  bool negq[kPbdGather];
  bool ok = eb - ea <= (int)blockDim.x && nb - na <= (int)blockDim.x && bb - ba <= (int)blockDim.x;
  if (ok) ok = pbd_load_node(d, na + tid, nb, rn);
  if (ok && ea + tid < eb) {
    e = d.c_edges[ea + tid];
    pr = d.pairs[e];
    ns = d.ndeg[pr.x];
    nt = d.ndeg[pr.y];
    L0 = d.rest_len[e];
    const int qa = d.e_start[e];
    ne3 = d.e_start[e + 1] - qa;
    if (ne3 > kPbdGather) ok = false;
#pragma unroll
    for (int q = 0; q < kPbdGather; ++q)
      if (q < ne3) {
        const int en = d.e_list[qa + q];
        bq[q] = en >> 1;
        negq[q] = en & 1;
      }
  }
  if (ok && ba + tid < bb) {
    b = d.c_bps[ba + tid];
    bp = d.bpairs[b];
    ed_x = d.edeg[bp.x];
    ed_y = d.edeg[bp.y];
    kbb = d.kb[b];
    rst = d.rest[b];
  }
  if (!__syncthreads_and(ok)) return false;
  float acc_len = e >= 0 ? d.d_len[e] : 0.0f;
  float acc_rest = b >= 0 ? d.rest_acc[b] : 0.0f;
  float acc_kb = b >= 0 ? d.d_kb[b] : 0.0f;
  int cur = 0;
  for (int k = d.C - 1; k >= 0; --k) {
    const float2* p = d.pp + (size_t)k * d.N;
    const float* th = d.tt + (size_t)k * d.E;
    const float* thn = d.tt + (size_t)(k + 1) * d.E;
    const float2* lpi = d.lp[cur];
    float2* lpo = d.lp[cur ^ 1];
    const float* lti = d.lt[cur];
    float* lto = d.lt[cur ^ 1];
    // position pass
    if (e >= 0) {
      const float2 la = lpi[pr.x], lb = lpi[pr.y], pa = p[pr.x], pb = p[pr.y];
      const float th_n = thn[e], lt_e = lti[e];
      const float hx = ((la.x / ns - lb.x / nt) * kst) * 0.5f;
      const float hy = ((la.y / ns - lb.y / nt) * kst) * 0.5f;
      const float2 cur_v = mc::min_image(pb.x, pb.y, pa.x, pa.y, (float)d.W, (float)d.H);
      const float L = sqrtf(cur_v.x * cur_v.x + cur_v.y * cur_v.y);
      const float m = mc::max_prop(L, 1e-8f);
      const float a = (L - L0) / m;
      const float da = (1.0f / m - (L - L0) * dmaxf(L, 1e-8f) / (m * m)) / L;
      const float lsx = (1.0f - ks) * hx, lsy = (1.0f - ks) * hy;
      const float sdot = cur_v.x * lsx + cur_v.y * lsy;
      const float lcx = ks * hx + a * lsx + (sdot * da) * cur_v.x;
      const float lcy = ks * hy + a * lsy + (sdot * da) * cur_v.y;
      const float ltx = -ks * hx, lty = -ks * hy;
      float cs, sn;
      sincosf(th_n, &sn, &cs);
      acc_len += -sdot / m + (cs * ltx + sn * lty);
      d.lthn[e] = lt_e + L0 * (-sn * ltx + cs * lty);
      d.lcur[e] = make_float2(lcx, lcy);
    }
    __syncthreads();
    if (rn.n >= 0) {
      float2 lc[kPbdGather];
#pragma unroll
      for (int q = 0; q < kPbdGather; ++q)
        if (q < rn.ne) lc[q] = d.lcur[rn.e[q]];
      float ax = lpi[rn.n].x, ay = lpi[rn.n].y;
#pragma unroll
      for (int q = 0; q < kPbdGather; ++q)
        if (q < rn.ne) {
          if (rn.neg[q]) {
            ax += lc[q].x;
            ay += lc[q].y;
          } else {
            ax -= lc[q].x;
            ay -= lc[q].y;
          }
        }
      lpo[rn.n] = make_float2(ax, ay);
    }
    if (b >= 0) {
      const float lx = d.lthn[bp.x], ly = d.lthn[bp.y], tx = th[bp.x], ty = th[bp.y];
      const float lcorr = 1.8f * (lx / ed_x - ly / ed_y);
      const float g = lcorr * kbb * 0.5f;
      d.gb[b] = g;
      acc_rest -= g;
      const float pi = (float)M_PI;
      const float diff = mc::fmod_floor((ty - tx) + pi, (float)(2.0 * M_PI)) - pi;
      acc_kb += lcorr * (diff - rst) * 0.5f;
    }
    __syncthreads();
    if (e >= 0) {
      float gq[kPbdGather];
#pragma unroll
      for (int q = 0; q < kPbdGather; ++q)
        if (q < ne3) gq[q] = d.gb[bq[q]];
      float a = d.lthn[e];
#pragma unroll
      for (int q = 0; q < kPbdGather; ++q)
        if (q < ne3) a += negq[q] ? gq[q] : -gq[q];
      lto[e] = a;
    }
    __syncthreads();
    cur ^= 1;
  }
  if (e >= 0) d.d_len[e] = acc_len;
  if (b >= 0) {
    d.rest_acc[b] = acc_rest;
    d.d_kb[b] = acc_kb;
  }
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(kPbdThreads) k_pbd_rev(AD d) {
  const int t = d.sa[*d.jp].t;
  const int c = blockIdx.x;
  const int ea = d.c_estart[c], eb = d.c_estart[c + 1], na = d.c_nstart[c], nb = d.c_nstart[c + 1];
  const int ba = d.c_bstart[c], bb = d.c_bstart[c + 1];
  int cur = 0;
  const float ks = d.kshear, kst = d.kstretch;
  if (pbd_rev_fast(d, ea, eb, na, nb, ba, bb, ks, kst))
    cur = d.C & 1;
  else
  for (int k = d.C - 1; k >= 0; --k) {
    const float2* p = d.pp + (size_t)k * d.N;
    const float* th = d.tt + (size_t)k * d.E;
    const float* thn = d.tt + (size_t)(k + 1) * d.E;
    const float2* lpi = d.lp[cur];
    float2* lpo = d.lp[cur ^ 1];
    const float* lti = d.lt[cur];
    float* lto = d.lt[cur ^ 1];
    // position pass
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      const int2 pr = d.pairs[e];
      const float ns = d.ndeg[pr.x], nt = d.ndeg[pr.y];
      const float hx = ((lpi[pr.x].x / ns - lpi[pr.y].x / nt) * kst) * 0.5f;
      const float hy = ((lpi[pr.x].y / ns - lpi[pr.y].y / nt) * kst) * 0.5f;
      const float2 cur_v = mc::min_image(p[pr.y].x, p[pr.y].y, p[pr.x].x, p[pr.x].y, (float)d.W, (float)d.H);
      const float L = sqrtf(cur_v.x * cur_v.x + cur_v.y * cur_v.y);
      const float L0 = d.rest_len[e];
      const float m = mc::max_prop(L, 1e-8f);
      const float a = (L - L0) / m;
      const float da = (1.0f / m - (L - L0) * dmaxf(L, 1e-8f) / (m * m)) / L;
      const float lsx = (1.0f - ks) * hx, lsy = (1.0f - ks) * hy;
      const float sdot = cur_v.x * lsx + cur_v.y * lsy;
      const float lcx = ks * hx + a * lsx + (sdot * da) * cur_v.x;
      const float lcy = ks * hy + a * lsy + (sdot * da) * cur_v.y;
      const float ltx = -ks * hx, lty = -ks * hy;
      float cs, sn;
      sincosf(thn[e], &sn, &cs);
      d.d_len[e] += -sdot / m + (cs * ltx + sn * lty);
      d.lthn[e] = lti[e] + L0 * (-sn * ltx + cs * lty);
      d.lcur[e] = make_float2(lcx, lcy);
    }
    __syncthreads();
    for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
      const int n = d.c_nodes[in];
      float ax = lpi[n].x, ay = lpi[n].y;
      for (int q = d.n_start[n]; q < d.n_start[n + 1]; ++q) {
        const int en = d.n_list[q];
        const float2 lc = d.lcur[en >> 1];
        if (en & 1) {
          ax += lc.x;
          ay += lc.y;
        } else {
          ax -= lc.x;
          ay -= lc.y;
        }
      }
      lpo[n] = make_float2(ax, ay);
    }
    for (int ib = ba + threadIdx.x; ib < bb; ib += blockDim.x) {
      const int b = d.c_bps[ib];
      const int2 bp = d.bpairs[b];
      const float lcorr = 1.8f * (d.lthn[bp.x] / d.edeg[bp.x] - d.lthn[bp.y] / d.edeg[bp.y]);
      const float g = lcorr * d.kb[b] * 0.5f;
      d.gb[b] = g;
      d.rest_acc[b] -= g;
      const float pi = (float)M_PI;
      const float diff = mc::fmod_floor((th[bp.y] - th[bp.x]) + pi, (float)(2.0 * M_PI)) - pi;
      d.d_kb[b] += lcorr * (diff - d.rest[b]) * 0.5f;
    }
    __syncthreads();
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      float a = d.lthn[e];
      for (int q = d.e_start[e]; q < d.e_start[e + 1]; ++q) {
        const int en = d.e_list[q];
        const float g = d.gb[en >> 1];
        a += (en & 1) ? g : -g;
      }
      lto[e] = a;
    }
    __syncthreads();
    cur ^= 1;
  }
  for (int in = na + threadIdx.x; in < nb; in += blockDim.x) d.lpred1[d.c_nodes[in]] = d.lp[cur][d.c_nodes[in]];
  for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) d.lth[d.c_edges[ie]] = d.lt[cur][d.c_edges[ie]];
  for (int ib = ba + threadIdx.x; ib < bb; ib += blockDim.x) {
    const int b = d.c_bps[ib];
    const float G = d.rest_acc[b];
    if (d.has_act) {
      const float arg = d.act_om[b] * (float)t + d.act_ph[b];
      float sn, cs;
      sincosf(arg, &sn, &cs);
      d.d_c[b] += G;
      d.d_amp[b] += G * sn;
      d.d_ph[b] += G * d.act_amp[b] * cs;
      d.d_om[b] += G * d.act_amp[b] * cs * (float)t;
    } else {
      d.d_rest[b] += G;
    }
  }
}

// ------------------------------------------------------------------ stable-Cosserat iterations
// (solver/stable_cosserat.py:13-119), one CTA per rod component like the PBD kernels.
// Iteration k: theta' = pull(theta + sum(+-corr) / edeg) toward the segment direction,
// then x' = x + (w (y - x) + sum(+-f_e)) / (w + sum k_s / l_e^2) with
// f_e = (k_s / l_e)(r_e / l_e - (cos theta'_e, sin theta'_e)), r_e the min-image segment,
// y the prediction (pp[0]).  Same arithmetic and sum order as the forward rod kernels.
__device__ __forceinline__ float2 cos_force(const AD& d, const float2* p, float thn, int e) {
  const int2 pr = d.pairs[e];
  const float L0 = d.rest_len[e];
  const float2 r = mc::min_image(p[pr.y].x, p[pr.y].y, p[pr.x].x, p[pr.x].y, (float)d.W, (float)d.H);
  float sn, cs;
  sincosf(thn, &sn, &cs);
  const float kl = d.kstretch / L0;
  return make_float2(kl * (r.x / L0 - cs), kl * (r.y / L0 - sn));
}

// the summed force and stiffness of node n at iterate p, angles thn
__device__ __forceinline__ void cos_node_sum(const AD& d, const float2* p, const float* thn, int n, float& ax,
                                             float& ay, float& hh) {
  const float w = d.cos_w;
  ax = w * (d.pp[n].x - p[n].x);
  ay = w * (d.pp[n].y - p[n].y);
  hh = w;
  for (int q = d.n_start[n]; q < d.n_start[n + 1]; ++q) {
    const int en = d.n_list[q];
    const int e = en >> 1;
    const float2 f = cos_force(d, p, thn[e], e);
    if (en & 1) {
      ax = ax + (-f.x);
      ay = ay + (-f.y);
    } else {
      ax = ax + f.x;
      ay = ay + f.y;
    }
    const float L0 = d.rest_len[e];
    hh = hh + d.kstretch / (L0 * L0);
  }
}

__global__ void __launch_bounds__(kPbdThreads) k_cos_fwd(AD d) {
  const int c = blockIdx.x;
  const int ea = d.c_estart[c], eb = d.c_estart[c + 1], na = d.c_nstart[c], nb = d.c_nstart[c + 1];
  for (int k = 0; k < d.C; ++k) {
    const float* th = d.tt + (size_t)k * d.E;
    float* thn = d.tt + (size_t)(k + 1) * d.E;
    const float2* p = d.pp + (size_t)k * d.N;
    float2* pn = d.pp + (size_t)(k + 1) * d.N;
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      float acc = 0.0f;
      for (int q = d.e_start[e]; q < d.e_start[e + 1]; ++q) {
        const int en = d.e_list[q];
        const float cr = bend_corr(d, th, en >> 1);
        acc = acc + ((en & 1) ? -cr : cr);
      }
      const int2 pr = d.pairs[e];
      const float2 r = mc::min_image(p[pr.y].x, p[pr.y].y, p[pr.x].x, p[pr.x].y, (float)d.W, (float)d.H);
      thn[e] = mc::cos_pull(th[e] + acc / d.edeg[e], r.x, r.y);
    }
    __syncthreads();
    for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
      const int n = d.c_nodes[in];
      float ax, ay, hh;
      cos_node_sum(d, p, thn, n, ax, ay, hh);
      pn[n] = make_float2(p[n].x + ax / hh, p[n].y + ay / hh);
    }
    __syncthreads();
  }
}

// Reverse of k_cos_fwd.  mod passes its cotangent through (derivative 1) and
// d atan2(r_y, r_x) = (r_x dr_y - r_y dr_x) / |r|^2.
__global__ void __launch_bounds__(kPbdThreads) k_cos_rev(AD d) {
  const int t = d.sa[*d.jp].t;
  const int c = blockIdx.x;
  const int ea = d.c_estart[c], eb = d.c_estart[c + 1], na = d.c_nstart[c], nb = d.c_nstart[c + 1];
  const int ba = d.c_bstart[c], bb = d.c_bstart[c + 1];
  const float ks = d.kstretch, w = d.cos_w;
  int cur = 0;
  for (int in = na + threadIdx.x; in < nb; in += blockDim.x) d.ly[d.c_nodes[in]] = make_float2(0.0f, 0.0f);
  for (int k = d.C - 1; k >= 0; --k) {
    const float2* p = d.pp + (size_t)k * d.N;
    const float* th = d.tt + (size_t)k * d.E;
    const float* thn = d.tt + (size_t)(k + 1) * d.E;
    const float2* lpi = d.lp[cur];
    float2* lpo = d.lp[cur ^ 1];
    const float* lti = d.lt[cur];
    float* lto = d.lt[cur ^ 1];
    // x' = x + F / h: cotangents of F, h, y and the direct part of x
    for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
      const int n = d.c_nodes[in];
      float ax, ay, hh;
      cos_node_sum(d, p, thn, n, ax, ay, hh);
      const float2 lx = lpi[n];
      const float lfx = lx.x / hh, lfy = lx.y / hh;
      d.lfn[n] = make_float2(lfx, lfy);
      d.lhn[n] = -(lx.x * ax + lx.y * ay) / (hh * hh);
      const float2 yy = d.ly[n];
      d.ly[n] = make_float2(yy.x + w * lfx, yy.y + w * lfy);
      lpo[n] = make_float2(lx.x - w * lfx, lx.y - w * lfy);
    }
    __syncthreads();
    // per edge: f_e and h_e -> segment, angle, rest length; then the pull
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      const int2 pr = d.pairs[e];
      const float L0 = d.rest_len[e];
      const float2 r = mc::min_image(p[pr.y].x, p[pr.y].y, p[pr.x].x, p[pr.x].y, (float)d.W, (float)d.H);
      float sn, cs;
      sincosf(thn[e], &sn, &cs);
      const float2 a = d.lfn[pr.x], b = d.lfn[pr.y];
      const float lfx = a.x - b.x, lfy = a.y - b.y;
      const float kl = ks / L0;
      float lrx = (kl / L0) * lfx, lry = (kl / L0) * lfy;
      const float lthn = lti[e] + kl * (lfx * sn - lfy * cs);
      const float cx = r.x / L0 - cs, cy = r.y / L0 - sn;
      d.d_len[e] += -(kl / L0) * (lfx * cx + lfy * cy) - (kl / (L0 * L0)) * (lfx * r.x + lfy * r.y) +
                    (d.lhn[pr.x] + d.lhn[pr.y]) * (-2.0f * ks / (L0 * L0 * L0));
      const float la = 0.05f * lthn;
      const float r2 = r.x * r.x + r.y * r.y;
      lrx += -r.y * la / r2;
      lry += r.x * la / r2;
      d.lcur[e] = make_float2(lrx, lry);
      d.lthn[e] = lthn - 0.05f * lthn;  // cotangent of the angle before the pull
    }
    __syncthreads();
    for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
      const int n = d.c_nodes[in];
      float ax = lpo[n].x, ay = lpo[n].y;
      for (int q = d.n_start[n]; q < d.n_start[n + 1]; ++q) {
        const int en = d.n_list[q];
        const float2 lc = d.lcur[en >> 1];
        if (en & 1) {
          ax += lc.x;
          ay += lc.y;
        } else {
          ax -= lc.x;
          ay -= lc.y;
        }
      }
      lpo[n] = make_float2(ax, ay);
    }
    for (int ib = ba + threadIdx.x; ib < bb; ib += blockDim.x) {
      const int b = d.c_bps[ib];
      const int2 bp = d.bpairs[b];
      const float lcorr = d.lthn[bp.x] / d.edeg[bp.x] - d.lthn[bp.y] / d.edeg[bp.y];
      const float g = lcorr * d.kb[b] * 0.5f;
      d.gb[b] = g;
      d.rest_acc[b] -= g;
      const float pi = (float)M_PI;
      const float diff = mc::fmod_floor((th[bp.y] - th[bp.x]) + pi, (float)(2.0 * M_PI)) - pi;
      d.d_kb[b] += lcorr * (diff - d.rest[b]) * 0.5f;
    }
    __syncthreads();
    for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) {
      const int e = d.c_edges[ie];
      float a = d.lthn[e];
      for (int q = d.e_start[e]; q < d.e_start[e + 1]; ++q) {
        const int en = d.e_list[q];
        const float g = d.gb[en >> 1];
        a += (en & 1) ? g : -g;
      }
      lto[e] = a;
    }
    __syncthreads();
    cur ^= 1;
  }
  // the iterations start from the prediction and are pulled toward it
  for (int in = na + threadIdx.x; in < nb; in += blockDim.x) {
    const int n = d.c_nodes[in];
    const float2 a = d.lp[cur][n], yy = d.ly[n];
    d.lpred1[n] = make_float2(a.x + yy.x, a.y + yy.y);
  }
  for (int ie = ea + threadIdx.x; ie < eb; ie += blockDim.x) d.lth[d.c_edges[ie]] = d.lt[cur][d.c_edges[ie]];
  for (int ib = ba + threadIdx.x; ib < bb; ib += blockDim.x) {
    const int b = d.c_bps[ib];
    const float G = d.rest_acc[b];
    if (d.has_act) {
      const float arg = d.act_om[b] * (float)t + d.act_ph[b];
      float sn, cs;
      sincosf(arg, &sn, &cs);
      d.d_c[b] += G;
      d.d_amp[b] += G * sn;
      d.d_ph[b] += G * d.act_amp[b] * cs;
      d.d_om[b] += G * d.act_amp[b] * cs * (float)t;
    } else {
      d.d_rest[b] += G;
    }
  }
}

// ------------------------------------------------------------------ adjoint: steric
__device__ __forceinline__ void sample_adj(const AD& d, const float* V, float yy, float xx, float coef, int n, int qs,
                                           float& lpx, float& lpy) {
  const float ly = floorf(yy), lx = floorf(xx);
  const float ty = yy - ly, tx = xx - lx;
  const int iy = (int)ly, ix = (int)lx;
  const int y0 = mc::imod_floor(iy, d.H), y1 = mc::imod_floor(iy + 1, d.H);
  const int x0 = mc::imod_floor(ix, d.W), x1 = mc::imod_floor(ix + 1, d.W);
  const float v00 = V[y0 * d.W + x0], v01 = V[y0 * d.W + x1], v10 = V[y1 * d.W + x0], v11 = V[y1 * d.W + x1];
  lpx += coef * ((1.0f - ty) * (v01 - v00) + ty * (v11 - v10));
  lpy += coef * ((1.0f - tx) * (v10 - v00) + tx * (v11 - v01));
  const size_t base = (size_t)n * 16 + qs * 4;
  d.st_cell[base + 0] = y0 * d.W + x0;
  d.st_val[base + 0] = coef * ((1.0f - ty) * (1.0f - tx));
  d.st_cell[base + 1] = y0 * d.W + x1;
  d.st_val[base + 1] = coef * ((1.0f - ty) * tx);
  d.st_cell[base + 2] = y1 * d.W + x0;
  d.st_val[base + 2] = coef * (ty * (1.0f - tx));
  d.st_cell[base + 3] = y1 * d.W + x1;
  d.st_val[base + 3] = coef * (ty * tx);
}

__global__ void k_steric_adj_node(AD d) {
  const float* __restrict__ V = d.sa[*d.jp].V;
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  const float Wf = (float)d.W, Hf = (float)d.H;
  const float2 lp1 = d.lpred1[n];
  const float lfx = (lp1.x * d.st_strength) * d.dt, lfy = (lp1.y * d.st_strength) * d.dt;
  const float2 q = d.pred0[n];
  const float x = mc::fmod_floor(q.x, Wf), y = mc::fmod_floor(q.y, Hf);
  const float e = 0.5f;
  float lpx = 0.0f, lpy = 0.0f;
  sample_adj(d, V, y, x + e, -lfx, n, 0, lpx, lpy);
  sample_adj(d, V, y, x - e, lfx, n, 1, lpx, lpy);
  sample_adj(d, V, y + e, x, -lfy, n, 2, lpx, lpy);
  sample_adj(d, V, y - e, x, lfy, n, 3, lpx, lpy);
  if (d.nskip > 0) {
    const float s2 = d.sigma * d.sigma;
    const float inv2s2 = 2.0f * d.sigma * d.sigma;
    const float norm = (float)(2.0 * M_PI) * d.sigma * d.sigma;
    const float pre = d.scatter / (d.sigma * d.sigma);
    for (int o = -d.nskip; o <= d.nskip; ++o) {
      const int j = n + o;
      if (o == 0 || j < 0 || j >= d.N) continue;
      const float2 qj = d.pred0[j];
      const float2 r = mc::min_image(x, y, mc::fmod_floor(qj.x, Wf), mc::fmod_floor(qj.y, Hf), Wf, Hf);
      const float d2 = r.x * r.x + r.y * r.y;
      const float K = expf(-d2 / inv2s2) / norm;
      const float2 lpj = d.lpred1[j];
      const float ljx = (lpj.x * d.st_strength) * d.dt, ljy = (lpj.y * d.st_strength) * d.dt;
      // J(r) (g_n - g_j) with g = -pre * lf and J = K (I - r r^T / sigma^2)
      const float gx = -pre * (lfx - ljx), gy = -pre * (lfy - ljy);
      const float rg = (r.x * gx + r.y * gy) / s2;
      lpx += K * (gx - r.x * rg);
      lpy += K * (gy - r.y * rg);
    }
  }
  d.lpred0p[n] = make_float2(lp1.x + lpx, lp1.y + lpy);
}

// out must be zero outside the touched cells
__global__ void k_gather_field(AD d, const float* __restrict__ val, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *d.ntouched) return;
  const int c = d.touched[i];
  float a = 0.0f;
  for (int q = d.start[c]; q < d.start[c + 1]; ++q) a = a + val[d.ent[q]];
  out[c] = a;
}

__global__ void k_steric_adj_cic(AD d) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= d.N) return;
  float2 l0 = d.lpred0p[n];
  if (d.steric) {
    const float Wf = (float)d.W, Hf = (float)d.H;
    const float2 q = d.pred0[n];
    const float x = mc::fmod_floor(q.x, Wf), y = mc::fmod_floor(q.y, Hf);
    const float fx = floorf(x), fy = floorf(y);
    const int x0 = mc::imod_floor((int)fx, d.W), y0 = mc::imod_floor((int)fy, d.H);
    const int x1 = (x0 + 1) % d.W, y1 = (y0 + 1) % d.H;
    const float dx = x - fx, dy = y - fy;
    const float d00 = d.ldep[y0 * d.W + x0], d10 = d.ldep[y0 * d.W + x1];
    const float d01 = d.ldep[y1 * d.W + x0], d11 = d.ldep[y1 * d.W + x1];
    const float s = d.scatter;
    l0.x += s * (-(1.0f - dy) * d00 + (1.0f - dy) * d10 - dy * d01 + dy * d11);
    l0.y += s * (-(1.0f - dx) * d00 - dx * d10 + (1.0f - dx) * d01 + dx * d11);
  }
  const float2 lpv = d.lprev[n];
  d.lpos[n] = make_float2(lpv.x + l0.x, lpv.y + l0.y);
  d.lvel[n] = make_float2((l0.x * d.damp) * d.dt, (l0.y * d.damp) * d.dt);
}

__global__ void k_step_next(AD d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *d.jp -= 1;
}

__global__ void k_copy_lpred(AD d) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < d.N) d.lpred0p[n] = d.lpred1[n];
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------------ host plan
struct mc_grad_plan {
  mc_dims dims{};
  mc_config cfg{};
  float dt = 0.f;
  int T = 0, S = 1, nseg = 0;
  std::vector<int> pairs, bpairs, n_start, n_list, e_start, e_list;
  std::vector<float> ndeg, edeg;
  mc_plan* fwd = nullptr;
  size_t fwd_bytes = 0, total = 0;
  unsigned char* ws = nullptr;
  bool bound = false, have_forward = false, has_act = false;
  // region offsets
  struct R {
    size_t off = 0, bytes = 0;
  };
  R r_fwd, r_pairs, r_bpairs, r_nst, r_nl, r_est, r_el, r_ndeg, r_edeg, r_len, r_kb, r_rst, r_ac, r_aa, r_ao, r_ap,
      r_fdesc;
  bool filter_ready = false;
  R r_wpos, r_wvel, r_wth, r_wra, r_wst, r_wfu, r_wf, r_ck, r_seg, r_segV;
  R r_rest, r_pred0, r_pp, r_tt, r_ibidx, r_ibw, r_sraw, r_stmp, r_uc, r_inv, r_cnt, r_start, r_bsum, r_ent, r_touch;
  R r_lf0p, r_lv, r_lrho, r_luc, r_lnv, r_lprev, r_lpos, r_lvel, r_lth, r_lp0, r_lp1, r_lt0, r_lt1, r_lcur, r_lthn,
      r_gb, r_racc, r_dc, r_da, r_dp, r_do, r_dr, r_dl, r_dk, r_stc, r_stv, r_lpred1, r_lpred0p, r_lV, r_ctmp, r_ldep, r_lf0,
      r_lf1;
  size_t state_ck_bytes = 0;  // one checkpoint: pos, vel, theta, f
  AD ad{};
  std::vector<int> c_nstart, c_nodes, c_estart, c_edges, c_bstart, c_bps;  // rod components
  R r_cns, r_cn, r_ces, r_ce, r_cbs, r_cb, r_sargs, r_jp;
  R r_ly, r_lfn, r_lhn;
  std::vector<StepArgs> sargs;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t rev_graph = nullptr;  // one reverse step, replayed per step
  int rev_graph_act = -1;               // has_act the graph was captured with
};

namespace {

thread_local std::string g_gerr;

mc_status gfail(mc_status s, const std::string& m) {
  mc::set_last_error(m.c_str());
  return s;
}

#define GC(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return gfail(MC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

size_t al(size_t x) { return (x + 255) / 256 * 256; }

template <typename T>
T* at(unsigned char* ws, const mc_grad_plan::R& r) {
  return reinterpret_cast<T*>(ws + r.off);
}

// CSR of M entries over ncells cells (the lattice for the IB stencils, the domain grid for
// the steric samples)
void csr_build(const AD& d, const int* cells, int M, int ncells, cudaStream_t s) {
  const int nb = nblk(ncells, kScanChunk);
  if (M > 0) k_csr_count<<<nblk(M, 256), 256, 0, s>>>(cells, M, d.cnt);
  k_scan1<<<nb, 1024, 0, s>>>(d.cnt, ncells, d.start, d.bsum);
  k_scan2<<<1, 1024, 0, s>>>(d.bsum, nb);
  k_scan3<<<nblk(ncells, 256), 256, 0, s>>>(d.start, d.bsum, ncells, M);
  if (M > 0) k_csr_fill<<<nblk(M, 256), 256, 0, s>>>(cells, M, d.start, d.cnt, d.ent);
  cudaMemsetAsync(d.ntouched, 0, sizeof(int), s);
  k_csr_touched<<<nblk(ncells, 256), 256, 0, s>>>(d.start, ncells, d.touched, d.ntouched);
  k_csr_sort<<<nblk(std::max(M, 1), 256), 256, 0, s>>>(d.start, d.touched, d.ntouched, d.ent);
}

mc_status copy_state_to(mc_grad_plan* p, float* pos, float* vel, float* th, float* f, const float* spos, const float* svel,
                        const float* sth, const float* sf, cudaStream_t s) {
  const mc_dims& D = p->dims;
  const size_t HW = (size_t)p->ad.lHW;  // f_grid lives on the fluid lattice
  GC(cudaMemcpyAsync(pos, spos, (size_t)D.N * 8, cudaMemcpyDeviceToDevice, s));
  GC(cudaMemcpyAsync(vel, svel, (size_t)D.N * 8, cudaMemcpyDeviceToDevice, s));
  if (D.E) GC(cudaMemcpyAsync(th, sth, (size_t)D.E * 4, cudaMemcpyDeviceToDevice, s));
  GC(cudaMemcpyAsync(f, sf, 9 * HW * 4, cudaMemcpyDeviceToDevice, s));
  return MC_OK;
}

// checkpoint / segment slot layout: pos (2N), vel (2N), theta (E), f (9 lHW), each 256-aligned
struct Slot {
  float *pos, *vel, *th, *f;
};
Slot slot(mc_grad_plan* p, const mc_grad_plan::R& r, int k) {
  const mc_dims& D = p->dims;
  unsigned char* b = p->ws + r.off + (size_t)k * p->state_ck_bytes;
  Slot s;
  s.pos = reinterpret_cast<float*>(b);
  b += al((size_t)D.N * 8);
  s.vel = reinterpret_cast<float*>(b);
  b += al((size_t)D.N * 8);
  s.th = reinterpret_cast<float*>(b);
  b += al((size_t)std::max(D.E, 1) * 4);
  s.f = reinterpret_cast<float*>(b);
  return s;
}

mc_state working_state(mc_grad_plan* p) {
  mc_state w{};
  w.position = at<float>(p->ws, p->r_wpos);
  w.velocity = at<float>(p->ws, p->r_wvel);
  w.theta = at<float>(p->ws, p->r_wth);
  w.rest_lengths = at<float>(p->ws, p->r_len);
  w.bending_rest_angles = at<float>(p->ws, p->r_wra);
  w.bending_stiffness = at<float>(p->ws, p->r_kb);
  w.steric = at<float>(p->ws, p->r_wst);
  w.fluid_velocity = at<float>(p->ws, p->r_wfu);
  w.f_grid = at<float>(p->ws, p->r_wf);
  return w;
}

// Open a rollout of the forward plan on the working state, actuated from step t0 (the
// static rest angles restored first when there is no actuation).
mc_status begin_fwd(mc_grad_plan* p, int t0, cudaStream_t s) {
  mc_state w = working_state(p);
  mc_actuation a{};
  const mc_actuation* ap = nullptr;
  if (p->has_act) {
    a.c = at<float>(p->ws, p->r_ac);
    a.amp = at<float>(p->ws, p->r_aa);
    a.omega = at<float>(p->ws, p->r_ao);
    a.phase = at<float>(p->ws, p->r_ap);
    a.t0 = t0;
    ap = &a;
  } else if (p->dims.B) {
    GC(cudaMemcpyAsync(w.bending_rest_angles, at<float>(p->ws, p->r_rst), (size_t)p->dims.B * 4,
                       cudaMemcpyDeviceToDevice, s));
  }
  const mc_actuation* const acts[1] = {ap};
  return mc_rollout_begin(p->fwd, &w, acts, nullptr, s);
}

mc_status run_fwd(mc_grad_plan* p, int steps, int t0, cudaStream_t s) {
  mc_state w = working_state(p);
  mc_actuation a{};
  const mc_actuation* ap = nullptr;
  if (p->has_act) {
    a.c = at<float>(p->ws, p->r_ac);
    a.amp = at<float>(p->ws, p->r_aa);
    a.omega = at<float>(p->ws, p->r_ao);
    a.phase = at<float>(p->ws, p->r_ap);
    a.t0 = t0;
    ap = &a;
  } else if (p->dims.B) {
    // the static rest angles (the actuation, when used, overwrites this copy)
    GC(cudaMemcpyAsync(w.bending_rest_angles, at<float>(p->ws, p->r_rst), (size_t)p->dims.B * 4,
                       cudaMemcpyDeviceToDevice, s));
  }
  const mc_actuation* const acts[1] = {ap};
  return mc_rollout(p->fwd, &w, steps, acts, nullptr, 1, s);
}

// The kernels of one reverse step; its per-step inputs come from sa[*jp], and the last
// kernel moves jp to the previous step, so one captured graph replays a whole segment.
void reverse_step(mc_grad_plan* p, cudaStream_t s) {
  AD& d = p->ad;
  const int TB = 256;
  const int nNE = std::max(d.N, d.E);
  k_rest<<<nblk(std::max(d.B, 1), TB), TB, 0, s>>>(d);
  k_pred<<<nblk(nNE, TB), TB, 0, s>>>(d);
  if (d.solver == MC_SOLVER_COSSERAT)
    k_cos_fwd<<<d.ncomp, kPbdThreads, 0, s>>>(d);
  else
    k_pbd_fwd<<<d.ncomp, kPbdThreads, 0, s>>>(d);
  if (d.fluid) {
    k_ib_weights<<<nblk(d.NI, TB), TB, 0, s>>>(d);
    csr_build(d, d.ib_idx, d.NI * d.KK, d.lHW, s);
    k_macro<<<nblk(d.lHW, TB), TB, 0, s>>>(d);
    for (int it = 0; it < d.iters; ++it) {
      k_ib_interp<<<nblk(d.NI, TB), TB, 0, s>>>(d, it);
      k_ib_spread<<<nblk(d.NI * d.KK, TB), TB, 0, s>>>(d);
    }
    k_lbm_adj1<<<nblk(d.lHW, TB), TB, 0, s>>>(d);
    cudaMemsetAsync(d.lnv, 0, (size_t)d.NI * 8, s);
    for (int it = d.iters - 1; it >= 0; --it) {
      k_ib_rev_node<<<nblk(d.NI, TB), TB, 0, s>>>(d, it);
      k_ib_rev_cell<<<nblk(d.NI * d.KK, TB), TB, 0, s>>>(d);
    }
    k_lbm_adj2<<<nblk(d.lHW, TB), TB, 0, s>>>(d);
  }
  k_node_adj<<<nblk(nNE, TB), TB, 0, s>>>(d);
  if (d.solver == MC_SOLVER_COSSERAT)
    k_cos_rev<<<d.ncomp, kPbdThreads, 0, s>>>(d);
  else
    k_pbd_rev<<<d.ncomp, kPbdThreads, 0, s>>>(d);
  if (d.steric) {
    k_steric_adj_node<<<nblk(d.N, TB), TB, 0, s>>>(d);
    csr_build(d, d.st_cell, d.N * 16, d.HW, s);
    cudaMemsetAsync(d.lV, 0, (size_t)d.HW * 4, s);
    k_gather_field<<<nblk(d.N * 16, TB), TB, 0, s>>>(d, d.st_val, d.lV);
    // the spectral filter is real and even, so it is its own adjoint: the forward plan's
    // filter kernels map the sample cotangent lV to the deposit cotangent ldep
    mc::filter_launch(p->fwd, p->ws + p->r_fdesc.off, s);
  } else {
    k_copy_lpred<<<nblk(d.N, TB), TB, 0, s>>>(d);
  }
  k_steric_adj_cic<<<nblk(d.N, TB), TB, 0, s>>>(d);
  k_step_next<<<1, 32, 0, s>>>(d);
}

}  // namespace

extern "C" {

mc_status mc_grad_plan_create(const mc_dims* dims, const mc_config* cfg, float dt, const int32_t* pairs,
                              const int32_t* bending_pairs, int32_t num_steps, int32_t checkpoint_every,
                              mc_grad_plan** out) {
  mc::set_last_error("");
  if (!dims || !cfg || !out) return gfail(MC_ERR_INVALID, "null argument");
  *out = nullptr;
  const mc_dims D = *dims;
  if (D.N < 1 || D.E < 0 || D.B < 0 || D.H < 4 || D.W < 4) return gfail(MC_ERR_INVALID, "bad dims");
  if ((D.E && !pairs) || (D.B && !bending_pairs)) return gfail(MC_ERR_INVALID, "null topology");
  if (num_steps < 0) return gfail(MC_ERR_INVALID, "negative num_steps");
  if ((long long)D.H * D.W > (long long)kScanChunk * 4096) return gfail(MC_ERR_UNSUPPORTED, "grid too large for the gradient path");
  if (cfg->ibm_kernel_size < 1 || cfg->ibm_kernel_size * cfg->ibm_kernel_size > kMaxKK)
    return gfail(MC_ERR_UNSUPPORTED, "ibm_kernel_size outside 1..8");
  if (cfg->synthetic_node_width < 0.0f) return gfail(MC_ERR_INVALID, "synthetic_node_width must be >= 0");
  if ((D.fluid_H > 0) != (D.fluid_W > 0) || D.fluid_H < 0 || D.fluid_W < 0)
    return gfail(MC_ERR_INVALID, "fluid_H and fluid_W must both be 0 (the domain grid) or both > 0");
  if ((long long)std::max(D.fluid_H, 0) * std::max(D.fluid_W, 0) > (long long)kScanChunk * 4096)
    return gfail(MC_ERR_UNSUPPORTED, "fluid lattice too large for the gradient path");
  if (cfg->solver_type != MC_SOLVER_PBD && cfg->solver_type != MC_SOLVER_COSSERAT)
    return gfail(MC_ERR_INVALID, "solver_type must be MC_SOLVER_PBD or MC_SOLVER_COSSERAT");
  if (cfg->solver_type == MC_SOLVER_COSSERAT && !(cfg->solver_dt > 0.0))
    return gfail(MC_ERR_INVALID, "the stable-Cosserat solver needs solver_dt > 0");
  mc_grad_plan* p = new mc_grad_plan();
  p->dims = D;
  p->cfg = *cfg;
  p->dt = dt;
  p->T = num_steps;
  int S = checkpoint_every;
  if (S <= 0) S = std::max(1, (int)std::ceil(std::sqrt((double)std::max(num_steps, 1))));
  p->S = S;
  p->nseg = (num_steps + S - 1) / S;
  p->pairs.assign(pairs, pairs + 2 * (size_t)D.E);
  p->bpairs.assign(bending_pairs, bending_pairs + 2 * (size_t)D.B);
  for (int e = 0; e < D.E; ++e)
    for (int j = 0; j < 2; ++j)
      if (p->pairs[2 * e + j] < 0 || p->pairs[2 * e + j] >= D.N) {
        delete p;
        return gfail(MC_ERR_INVALID, "pairs index out of range");
      }
  for (int b = 0; b < D.B; ++b)
    for (int j = 0; j < 2; ++j)
      if (p->bpairs[2 * b + j] < 0 || p->bpairs[2 * b + j] >= D.E) {
        delete p;
        return gfail(MC_ERR_INVALID, "bending_pairs index out of range");
      }
  // gather lists in scatter order: sources first (in edge order), then targets
  p->n_start.assign(D.N + 1, 0);
  std::vector<std::vector<int>> nl(D.N);
  for (int e = 0; e < D.E; ++e) nl[p->pairs[2 * e]].push_back(e * 2);
  for (int e = 0; e < D.E; ++e) nl[p->pairs[2 * e + 1]].push_back(e * 2 + 1);
  p->ndeg.resize(D.N);
  for (int n = 0; n < D.N; ++n) {
    p->n_start[n + 1] = p->n_start[n] + (int)nl[n].size();
    p->n_list.insert(p->n_list.end(), nl[n].begin(), nl[n].end());
    p->ndeg[n] = std::max((float)nl[n].size(), 1.0f);
  }
  p->e_start.assign(D.E + 1, 0);
  std::vector<std::vector<int>> el(D.E);
  for (int b = 0; b < D.B; ++b) el[p->bpairs[2 * b]].push_back(b * 2);
  for (int b = 0; b < D.B; ++b) el[p->bpairs[2 * b + 1]].push_back(b * 2 + 1);
  p->edeg.resize(D.E);
  for (int e = 0; e < D.E; ++e) {
    p->e_start[e + 1] = p->e_start[e] + (int)el[e].size();
    p->e_list.insert(p->e_list.end(), el[e].begin(), el[e].end());
    p->edeg[e] = std::max((float)el[e].size(), 1.0f);
  }
  {
    // rod components: union-find over the edges; members listed in ascending order
    std::vector<int> par(D.N);
    for (int n = 0; n < D.N; ++n) par[n] = n;
    auto find = [&](int x) {
      while (par[x] != x) {
        par[x] = par[par[x]];
        x = par[x];
      }
      return x;
    };
    for (int e = 0; e < D.E; ++e) {
      const int a = find(p->pairs[2 * e]), b = find(p->pairs[2 * e + 1]);
      if (a != b) par[std::max(a, b)] = std::min(a, b);
    }
    std::vector<int> cid(D.N, -1);
    int nc = 0;
    for (int n = 0; n < D.N; ++n) {
      const int r = find(n);
      if (cid[r] < 0) cid[r] = nc++;
      cid[n] = cid[r];
    }
    std::vector<std::vector<int>> cn(nc), ce(nc), cb(nc);
    for (int n = 0; n < D.N; ++n) cn[cid[n]].push_back(n);
    for (int e = 0; e < D.E; ++e) ce[cid[p->pairs[2 * e]]].push_back(e);
    for (int b = 0; b < D.B; ++b) cb[cid[p->pairs[2 * p->bpairs[2 * b]]]].push_back(b);
    p->c_nstart.assign(1, 0);
    p->c_estart.assign(1, 0);
    p->c_bstart.assign(1, 0);
    for (int c = 0; c < nc; ++c) {
      p->c_nodes.insert(p->c_nodes.end(), cn[c].begin(), cn[c].end());
      p->c_edges.insert(p->c_edges.end(), ce[c].begin(), ce[c].end());
      p->c_bps.insert(p->c_bps.end(), cb[c].begin(), cb[c].end());
      p->c_nstart.push_back((int)p->c_nodes.size());
      p->c_estart.push_back((int)p->c_edges.size());
      p->c_bstart.push_back((int)p->c_bps.size());
    }
  }
  // forward plan (same kernels as mc_rollout)
  const int32_t* pp[1] = {pairs};
  const int32_t* bb[1] = {bending_pairs};
  mc_status st = mc_plan_create(1, &D, cfg, &dt, pp, bb, &p->fwd);
  if (st != MC_OK) {
    delete p;
    return st;
  }
  p->fwd_bytes = mc_plan_workspace_bytes(p->fwd);
  // layout
  const size_t N = D.N, E = std::max(D.E, 1), B = std::max(D.B, 1), HW = (size_t)D.H * D.W;
  const size_t LHW = D.fluid_H > 0 ? (size_t)D.fluid_H * D.fluid_W : HW;  // fluid lattice cells
  const size_t CHW = std::max(HW, LHW);                                    // CSR cells
  const size_t NI = N * (cfg->enable_fluid && cfg->synthetic_node_width > 0.0f ? 2 : 1);  // IB points
  const int C = cfg->cycles_per_step, KK = cfg->ibm_kernel_size * cfg->ibm_kernel_size;
  const int iters = std::max(cfg->ibm_iterations, 1);
  size_t o = 0;
  auto take = [&](mc_grad_plan::R& r, size_t bytes) {
    r.off = o;
    r.bytes = bytes;
    o += al(std::max<size_t>(bytes, 4));
  };
  take(p->r_fwd, p->fwd_bytes);
  take(p->r_pairs, E * 8);
  take(p->r_bpairs, B * 8);
  take(p->r_nst, (N + 1) * 4);
  take(p->r_nl, std::max<size_t>(p->n_list.size(), 1) * 4);
  take(p->r_est, (E + 1) * 4);
  take(p->r_el, std::max<size_t>(p->e_list.size(), 1) * 4);
  take(p->r_ndeg, N * 4);
  take(p->r_edeg, E * 4);
  take(p->r_len, E * 4);
  take(p->r_kb, B * 4);
  take(p->r_rst, B * 4);
  take(p->r_ac, B * 4);
  take(p->r_aa, B * 4);
  take(p->r_ao, B * 4);
  take(p->r_ap, B * 4);
  take(p->r_wpos, N * 8);
  take(p->r_wvel, N * 8);
  take(p->r_wth, E * 4);
  take(p->r_wra, B * 4);
  take(p->r_wst, HW * 4);
  take(p->r_wfu, 2 * LHW * 4);
  take(p->r_wf, 9 * LHW * 4);
  p->state_ck_bytes = al(N * 8) * 2 + al(E * 4) + al(9 * LHW * 4);
  take(p->r_ck, std::max(p->nseg, 1) * p->state_ck_bytes);
  take(p->r_seg, (size_t)S * p->state_ck_bytes);
  take(p->r_segV, (size_t)S * al(HW * 4));
  take(p->r_rest, B * 4);
  take(p->r_pred0, N * 8);
  take(p->r_pp, (size_t)(C + 1) * N * 8);
  take(p->r_tt, (size_t)(C + 1) * E * 4);
  take(p->r_ibidx, NI * KK * 4);
  take(p->r_ibw, NI * KK * 4);
  take(p->r_sraw, (size_t)iters * NI * 8);
  take(p->r_stmp, NI * 8);
  take(p->r_uc, 2 * LHW * 4);
  take(p->r_inv, LHW * 4);
  take(p->r_cnt, CHW * 4);
  take(p->r_start, (CHW + 1) * 4);
  take(p->r_bsum, 4096 * 4);
  take(p->r_ent, std::max<size_t>(NI * KK, 16 * N) * 4);
  take(p->r_touch, std::max<size_t>(NI * KK, 16 * N) * 4 + 256);
  take(p->r_lf0p, 9 * LHW * 4);
  take(p->r_lv, 2 * LHW * 4);
  take(p->r_lrho, LHW * 4);
  take(p->r_luc, 2 * LHW * 4);
  take(p->r_lnv, NI * 8);
  take(p->r_lprev, N * 8);
  take(p->r_lpos, N * 8);
  take(p->r_lvel, N * 8);
  take(p->r_lth, E * 4);
  take(p->r_lp0, N * 8);
  take(p->r_lp1, N * 8);
  take(p->r_lt0, E * 4);
  take(p->r_lt1, E * 4);
  take(p->r_lcur, E * 8);
  take(p->r_lthn, E * 4);
  take(p->r_gb, B * 4);
  take(p->r_ly, N * 8);
  take(p->r_lfn, N * 8);
  take(p->r_lhn, N * 4);
  take(p->r_racc, B * 4);
  take(p->r_dc, B * 4);
  take(p->r_da, B * 4);
  take(p->r_dp, B * 4);
  take(p->r_do, B * 4);
  take(p->r_dr, B * 4);
  take(p->r_dl, E * 4);
  take(p->r_dk, B * 4);
  take(p->r_stc, 16 * N * 4);
  take(p->r_stv, 16 * N * 4);
  take(p->r_lpred1, N * 8);
  take(p->r_lpred0p, N * 8);
  take(p->r_lV, HW * 4);
  take(p->r_ctmp, HW * 4);
  take(p->r_ldep, HW * 4);
  take(p->r_lf0, 9 * LHW * 4);
  take(p->r_lf1, 9 * LHW * 4);
  take(p->r_cns, p->c_nstart.size() * 4);
  take(p->r_cn, std::max<size_t>(p->c_nodes.size(), 1) * 4);
  take(p->r_ces, p->c_estart.size() * 4);
  take(p->r_ce, std::max<size_t>(p->c_edges.size(), 1) * 4);
  take(p->r_cbs, p->c_bstart.size() * 4);
  take(p->r_cb, std::max<size_t>(p->c_bps.size(), 1) * 4);
  take(p->r_sargs, (size_t)S * sizeof(StepArgs));
  take(p->r_fdesc, mc::filter_desc_bytes());
  take(p->r_jp, 4);
  p->total = o;
  *out = p;
  return MC_OK;
}

void mc_grad_plan_destroy(mc_grad_plan* p) {
  if (!p) return;
  if (p->rev_graph) cudaGraphExecDestroy(p->rev_graph);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  if (p->fwd) mc_plan_destroy(p->fwd);
  delete p;
}

size_t mc_grad_plan_workspace_bytes(const mc_grad_plan* p) { return p ? p->total : 0; }

int32_t mc_grad_plan_checkpoint_every(const mc_grad_plan* p) { return p ? p->S : 0; }

mc_status mc_grad_plan_bind(mc_grad_plan* p, void* workspace, size_t bytes, void* stream) {
  mc::set_last_error("");
  if (!p) return gfail(MC_ERR_INVALID, "null plan");
  if (!workspace || bytes < p->total || ((uintptr_t)workspace & 255))
    return gfail(MC_ERR_WORKSPACE, "workspace missing, too small or not 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  p->ws = (unsigned char*)workspace;
  mc_status st = mc_plan_bind(p->fwd, p->ws + p->r_fwd.off, p->fwd_bytes, stream);
  if (st != MC_OK) return st;
  std::vector<mc::Upload> ups;
  auto up = [&](const mc_grad_plan::R& r, const void* src, size_t n) -> cudaError_t {
    if (n) ups.push_back({p->ws + r.off, src, n});
    return cudaSuccess;
  };
  GC(up(p->r_pairs, p->pairs.data(), p->pairs.size() * 4));
  GC(up(p->r_bpairs, p->bpairs.data(), p->bpairs.size() * 4));
  GC(up(p->r_nst, p->n_start.data(), p->n_start.size() * 4));
  GC(up(p->r_nl, p->n_list.data(), p->n_list.size() * 4));
  GC(up(p->r_est, p->e_start.data(), p->e_start.size() * 4));
  GC(up(p->r_el, p->e_list.data(), p->e_list.size() * 4));
  GC(up(p->r_ndeg, p->ndeg.data(), p->ndeg.size() * 4));
  GC(up(p->r_edeg, p->edeg.data(), p->edeg.size() * 4));
  GC(up(p->r_cns, p->c_nstart.data(), p->c_nstart.size() * 4));
  GC(up(p->r_cn, p->c_nodes.data(), p->c_nodes.size() * 4));
  GC(up(p->r_ces, p->c_estart.data(), p->c_estart.size() * 4));
  GC(up(p->r_ce, p->c_edges.data(), p->c_edges.size() * 4));
  GC(up(p->r_cbs, p->c_bstart.data(), p->c_bstart.size() * 4));
  GC(up(p->r_cb, p->c_bps.data(), p->c_bps.size() * 4));
  GC(mc::stage_uploads(ups.data(), (int)ups.size(), s));
  if (p->rev_graph) {
    cudaGraphExecDestroy(p->rev_graph);
    p->rev_graph = nullptr;
  }
  p->filter_ready = false;
  if (!p->cap_stream) GC(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
  GC(cudaMemsetAsync(p->ws + p->r_cnt.off, 0, p->r_cnt.bytes, s));
  const mc_config& c = p->cfg;
  const mc_dims& D = p->dims;
  AD& d = p->ad;
  d = AD{};
  d.H = D.H;
  d.W = D.W;
  d.N = D.N;
  d.E = D.E;
  d.B = D.B;
  d.HW = D.H * D.W;
  d.lH = D.fluid_H > 0 ? D.fluid_H : D.H;
  d.lW = D.fluid_W > 0 ? D.fluid_W : D.W;
  d.lHW = d.lH * d.lW;
  d.C = c.cycles_per_step;
  d.iters = c.ibm_iterations;
  d.K = c.ibm_kernel_size;
  d.KK = d.K * d.K;
  d.steric = c.enable_steric;
  d.fluid = c.enable_fluid;
  d.nskip = c.steric_neighbor_skip;
  d.dt = p->dt;
  d.damp = c.damping;
  d.st_strength = c.steric_strength;
  d.sigma = c.steric_sigma;
  d.scatter = c.steric_scatter_value;
  d.kstretch = c.stiffness_stretch;
  d.kshear = c.stiffness_shear;
  d.solver = c.solver_type;
  d.force_clamp = c.enable_force_clamp;
  d.NI = D.N * (c.enable_fluid && c.synthetic_node_width > 0.0f ? 2 : 1);
  d.syn_w = c.synthetic_node_width;
  // scale = (lW / H, lH / W): the reference's axis order (fluid.py:222-226)
  const double sxd = (double)d.lW / (double)D.H, syd = (double)d.lH / (double)D.W;
  d.syn_ms = (float)(0.5 * (sxd + syd));
  d.cos_w = c.solver_type == MC_SOLVER_COSSERAT ? (float)(1.0 / (c.solver_dt * c.solver_dt)) : 0.0f;
  const float scx = (float)sxd, scy = (float)syd;
  d.scx = scx;
  d.scy = scy;
  d.vmax = (float)((double)c.max_fluid_velocity * (0.5 * (sxd + syd)));
  d.relax = c.ibm_relaxation;
  d.mass = c.node_mass;
  {
    // omega+ = clip(1/(3 nu + 0.5), 0, 1.9); omega- from the magic parameter (fluid.py:155-161)
    const float wp = std::min(std::max((float)(1.0 / (3.0 * c.viscosity + 0.5)), 0.0f), 1.9f);
    const float eps = 1.1920928955078125e-07f;
    const float off = 1.0f / std::max(wp, eps) - 0.5f;
    const float wm = 1.0f / (c.lambda_trt / std::max(off, eps) + 0.5f);
    d.wp = wp;
    d.wm = wm;
    d.cp = 1.0f - 0.5f * wp;
    d.cm = 1.0f - 0.5f * wm;
  }
  d.sdtx = scx * p->dt;
  d.sdty = scy * p->dt;
  unsigned char* w = p->ws;
  d.pairs = at<int2>(w, p->r_pairs);
  d.bpairs = at<int2>(w, p->r_bpairs);
  d.n_start = at<int>(w, p->r_nst);
  d.n_list = at<int>(w, p->r_nl);
  d.e_start = at<int>(w, p->r_est);
  d.e_list = at<int>(w, p->r_el);
  d.ndeg = at<float>(w, p->r_ndeg);
  d.edeg = at<float>(w, p->r_edeg);
  d.rest_len = at<float>(w, p->r_len);
  d.kb = at<float>(w, p->r_kb);
  d.rest_static = at<float>(w, p->r_rst);
  d.act_c = at<float>(w, p->r_ac);
  d.act_amp = at<float>(w, p->r_aa);
  d.act_om = at<float>(w, p->r_ao);
  d.act_ph = at<float>(w, p->r_ap);
  d.rest = at<float>(w, p->r_rest);
  d.pred0 = at<float2>(w, p->r_pred0);
  d.pp = at<float2>(w, p->r_pp);
  d.tt = at<float>(w, p->r_tt);
  d.ib_idx = at<int>(w, p->r_ibidx);
  d.ib_w = at<float>(w, p->r_ibw);
  d.sraw = at<float2>(w, p->r_sraw);
  d.s_tmp = at<float2>(w, p->r_stmp);
  d.uc = at<float>(w, p->r_uc);
  d.inv = at<float>(w, p->r_inv);
  d.cnt = at<int>(w, p->r_cnt);
  d.start = at<int>(w, p->r_start);
  d.bsum = at<int>(w, p->r_bsum);
  d.ent = at<int>(w, p->r_ent);
  d.ntouched = at<int>(w, p->r_touch);
  d.touched = d.ntouched + 64;
  d.lf0p = at<float>(w, p->r_lf0p);
  d.lv = at<float>(w, p->r_lv);
  d.lrho = at<float>(w, p->r_lrho);
  d.luc = at<float>(w, p->r_luc);
  d.lnv = at<float2>(w, p->r_lnv);
  d.lprev = at<float2>(w, p->r_lprev);
  d.lpos = at<float2>(w, p->r_lpos);
  d.lvel = at<float2>(w, p->r_lvel);
  d.lth = at<float>(w, p->r_lth);
  d.lp[0] = at<float2>(w, p->r_lp0);
  d.lp[1] = at<float2>(w, p->r_lp1);
  d.lt[0] = at<float>(w, p->r_lt0);
  d.lt[1] = at<float>(w, p->r_lt1);
  d.lcur = at<float2>(w, p->r_lcur);
  d.lthn = at<float>(w, p->r_lthn);
  d.gb = at<float>(w, p->r_gb);
  d.ly = at<float2>(w, p->r_ly);
  d.lfn = at<float2>(w, p->r_lfn);
  d.lhn = at<float>(w, p->r_lhn);
  d.rest_acc = at<float>(w, p->r_racc);
  d.d_c = at<float>(w, p->r_dc);
  d.d_amp = at<float>(w, p->r_da);
  d.d_ph = at<float>(w, p->r_dp);
  d.d_om = at<float>(w, p->r_do);
  d.d_rest = at<float>(w, p->r_dr);
  d.d_len = at<float>(w, p->r_dl);
  d.d_kb = at<float>(w, p->r_dk);
  d.st_cell = at<int>(w, p->r_stc);
  d.st_val = at<float>(w, p->r_stv);
  d.lpred1 = at<float2>(w, p->r_lpred1);
  d.lpred0p = at<float2>(w, p->r_lpred0p);
  d.lV = at<float>(w, p->r_lV);
  d.ctmp = at<float>(w, p->r_ctmp);
  d.ldep = at<float>(w, p->r_ldep);
  d.ncomp = (int)p->c_nstart.size() - 1;
  d.c_nstart = at<int>(w, p->r_cns);
  d.c_nodes = at<int>(w, p->r_cn);
  d.c_estart = at<int>(w, p->r_ces);
  d.c_edges = at<int>(w, p->r_ce);
  d.c_bstart = at<int>(w, p->r_cbs);
  d.c_bps = at<int>(w, p->r_cb);
  d.sa = at<StepArgs>(w, p->r_sargs);
  d.jp = at<int>(w, p->r_jp);
  p->bound = true;
  return MC_OK;
}

mc_status mc_grad_forward(mc_grad_plan* p, const mc_state* state, const mc_actuation* act, void* stream) {
  mc::set_last_error("");
  if (!p || !state) return gfail(MC_ERR_INVALID, "null argument");
  if (!p->bound) return gfail(MC_ERR_NOT_BOUND, "mc_grad_plan_bind() was not called");
  cudaStream_t s = (cudaStream_t)stream;
  const mc_dims& D = p->dims;
  const size_t HW = (size_t)D.H * D.W;
  const size_t LHW = (size_t)p->ad.lHW;  // fluid lattice cells
  unsigned char* w = p->ws;
  auto cp = [&](const mc_grad_plan::R& r, const void* src, size_t n) -> cudaError_t {
    if (n == 0 || !src) return cudaSuccess;
    return cudaMemcpyAsync(w + r.off, src, n, cudaMemcpyDeviceToDevice, s);
  };
  if (!state->position || !state->velocity || !state->f_grid || (D.E && (!state->theta || !state->rest_lengths)) ||
      (D.B && (!state->bending_rest_angles || !state->bending_stiffness)))
    return gfail(MC_ERR_INVALID, "null state array");
  GC(cp(p->r_wpos, state->position, (size_t)D.N * 8));
  GC(cp(p->r_wvel, state->velocity, (size_t)D.N * 8));
  GC(cp(p->r_wth, state->theta, (size_t)D.E * 4));
  GC(cp(p->r_len, state->rest_lengths, (size_t)D.E * 4));
  GC(cp(p->r_kb, state->bending_stiffness, (size_t)D.B * 4));
  GC(cp(p->r_rst, state->bending_rest_angles, (size_t)D.B * 4));
  GC(cp(p->r_wra, state->bending_rest_angles, (size_t)D.B * 4));
  if (state->steric) GC(cp(p->r_wst, state->steric, HW * 4));
  else GC(cudaMemsetAsync(w + p->r_wst.off, 0, HW * 4, s));
  if (state->fluid_velocity) GC(cp(p->r_wfu, state->fluid_velocity, 2 * LHW * 4));
  else GC(cudaMemsetAsync(w + p->r_wfu.off, 0, 2 * LHW * 4, s));
  GC(cp(p->r_wf, state->f_grid, 9 * LHW * 4));
  p->has_act = act != nullptr;
  if (act) {
    if (D.B && (!act->c || !act->amp || !act->omega || !act->phase)) return gfail(MC_ERR_INVALID, "null actuation array");
    if (act->t0 != 0) return gfail(MC_ERR_UNSUPPORTED, "the gradient path starts its actuation clock at t0 = 0");
    GC(cp(p->r_ac, act->c, (size_t)D.B * 4));
    GC(cp(p->r_aa, act->amp, (size_t)D.B * 4));
    GC(cp(p->r_ao, act->omega, (size_t)D.B * 4));
    GC(cp(p->r_ap, act->phase, (size_t)D.B * 4));
  }
  p->ad.has_act = p->has_act ? 1 : 0;
  for (int k = 0; k < p->nseg; ++k) {
    Slot ck = slot(p, p->r_ck, k);
    mc_status st = copy_state_to(p, ck.pos, ck.vel, ck.th, ck.f, at<float>(w, p->r_wpos), at<float>(w, p->r_wvel),
                                 at<float>(w, p->r_wth), at<float>(w, p->r_wf), s);
    if (st != MC_OK) return st;
    const int len = std::min(p->S, p->T - k * p->S);
    st = run_fwd(p, len, k * p->S, s);
    if (st != MC_OK) return st;
  }
  // final state back to the caller
  auto back = [&](void* dst, const mc_grad_plan::R& r, size_t n) -> cudaError_t {
    if (!dst || n == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, w + r.off, n, cudaMemcpyDeviceToDevice, s);
  };
  GC(back(state->position, p->r_wpos, (size_t)D.N * 8));
  GC(back(state->velocity, p->r_wvel, (size_t)D.N * 8));
  GC(back(state->theta, p->r_wth, (size_t)D.E * 4));
  GC(back(state->bending_rest_angles, p->r_wra, (size_t)D.B * 4));
  GC(back(state->steric, p->r_wst, HW * 4));
  GC(back(state->fluid_velocity, p->r_wfu, 2 * LHW * 4));
  GC(back(state->f_grid, p->r_wf, 9 * LHW * 4));
  GC(cudaGetLastError());
  p->have_forward = true;
  return MC_OK;
}

mc_status mc_grad_backward(mc_grad_plan* p, const mc_state_cot* final_cot, mc_state_cot* initial_cot,
                           mc_param_grads* grads, void* stream) {
  mc::set_last_error("");
  if (!p || !final_cot || !initial_cot) return gfail(MC_ERR_INVALID, "null argument");
  if (!p->bound) return gfail(MC_ERR_NOT_BOUND, "mc_grad_plan_bind() was not called");
  if (!p->have_forward) return gfail(MC_ERR_INVALID, "mc_grad_forward() has not run on this plan");
  cudaStream_t s = (cudaStream_t)stream;
  const mc_dims& D = p->dims;
  const size_t HW = (size_t)D.H * D.W;
  const size_t LHW = (size_t)p->ad.lHW;  // fluid lattice cells
  unsigned char* w = p->ws;
  AD& d = p->ad;
  auto seed = [&](const mc_grad_plan::R& r, const float* src, size_t n) -> cudaError_t {
    if (n == 0) return cudaSuccess;
    if (!src) return cudaMemsetAsync(w + r.off, 0, n, s);
    return cudaMemcpyAsync(w + r.off, src, n, cudaMemcpyDeviceToDevice, s);
  };
  GC(seed(p->r_lpos, final_cot->position, (size_t)D.N * 8));
  GC(seed(p->r_lvel, final_cot->velocity, (size_t)D.N * 8));
  GC(seed(p->r_lth, final_cot->theta, (size_t)D.E * 4));
  GC(seed(p->r_lf0, final_cot->f_grid, 9 * LHW * 4));
  for (const mc_grad_plan::R* r : {&p->r_dc, &p->r_da, &p->r_dp, &p->r_do, &p->r_dr, &p->r_dl, &p->r_dk})
    GC(cudaMemsetAsync(w + r->off, 0, r->bytes, s));
  if (d.steric && !p->filter_ready) {
    // the forward plan's descriptor exists once mc_grad_forward has run a rollout call
    GC(mc::filter_prepare(p->fwd, w + p->r_fdesc.off, d.lV, d.ctmp, d.ldep, s));
    p->filter_ready = true;
  }
  int lfcur = 0;
  for (int k = p->nseg - 1; k >= 0; --k) {
    const int t0 = k * p->S;
    const int len = std::min(p->S, p->T - t0);
    Slot ck = slot(p, p->r_ck, k);
    mc_status st = copy_state_to(p, at<float>(w, p->r_wpos), at<float>(w, p->r_wvel), at<float>(w, p->r_wth),
                                 at<float>(w, p->r_wf), ck.pos, ck.vel, ck.th, ck.f, s);
    if (st != MC_OK) return st;
    // the segment's step inputs: one rollout over the segment, the populations of every
    // step's input snapshot from the open rollout (no per-step entry/exit conversion)
    st = begin_fwd(p, t0, s);
    if (st != MC_OK) return st;
    for (int j = 0; j < len; ++j) {
      Slot sj = slot(p, p->r_seg, j);
      GC(cudaMemcpyAsync(sj.pos, at<float>(w, p->r_wpos), (size_t)D.N * 8, cudaMemcpyDeviceToDevice, s));
      GC(cudaMemcpyAsync(sj.vel, at<float>(w, p->r_wvel), (size_t)D.N * 8, cudaMemcpyDeviceToDevice, s));
      if (D.E) GC(cudaMemcpyAsync(sj.th, at<float>(w, p->r_wth), (size_t)D.E * 4, cudaMemcpyDeviceToDevice, s));
      if (d.fluid) {
        st = mc::rollout_snapshot_f(p->fwd, sj.f, s);
        if (st != MC_OK) return st;
      } else {
        GC(cudaMemcpyAsync(sj.f, at<float>(w, p->r_wf), 9 * LHW * 4, cudaMemcpyDeviceToDevice, s));
      }
      st = mc_rollout_advance(p->fwd, 1, 1, 1, s);
      if (st != MC_OK) return st;
      GC(cudaMemcpyAsync(w + p->r_segV.off + (size_t)j * al(HW * 4), w + p->r_wst.off, HW * 4,
                         cudaMemcpyDeviceToDevice, s));
    }
    st = mc_rollout_end(p->fwd, s);
    if (st != MC_OK) return st;
    // per-step inputs of the segment (the cotangent of f alternates between two buffers)
    p->sargs.assign(len, StepArgs{});
    for (int j = len - 1; j >= 0; --j) {
      Slot sj = slot(p, p->r_seg, j);
      StepArgs& a = p->sargs[j];
      a.t = t0 + j;
      a.pos = sj.pos;
      a.vel = sj.vel;
      a.th = sj.th;
      a.f = sj.f;
      a.V = reinterpret_cast<const float*>(w + p->r_segV.off + (size_t)j * al(HW * 4));
      a.lf_in = at<float>(w, lfcur ? p->r_lf1 : p->r_lf0);
      a.lf_out = at<float>(w, lfcur ? p->r_lf0 : p->r_lf1);
      if (d.fluid) lfcur ^= 1;
    }
    const int jlast = len - 1;
    {
      // staged: the host arrays may change once the call returns, and the host does not
      // wait here for the stream to reach these copies
      const mc::Upload u[2] = {{w + p->r_sargs.off, p->sargs.data(), len * sizeof(StepArgs)},
                               {w + p->r_jp.off, &jlast, sizeof(int)}};
      GC(mc::stage_uploads(u, 2, s));
    }
    if (!p->rev_graph || p->rev_graph_act != d.has_act) {
      if (p->rev_graph) {
        cudaGraphExecDestroy(p->rev_graph);
        p->rev_graph = nullptr;
      }
      cudaGraph_t g;
      GC(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
      reverse_step(p, p->cap_stream);
      cudaError_t e = cudaStreamEndCapture(p->cap_stream, &g);
      if (e != cudaSuccess) return gfail(MC_ERR_CUDA, std::string("capture of the reverse step: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&p->rev_graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        p->rev_graph = nullptr;
        return gfail(MC_ERR_CUDA, std::string("instantiating the reverse step: ") + cudaGetErrorString(e));
      }
      p->rev_graph_act = d.has_act;
    }
    for (int j = len - 1; j >= 0; --j) GC(cudaGraphLaunch(p->rev_graph, s));
    GC(cudaGetLastError());
  }
  (void)d;
  auto out = [&](float* dst, const mc_grad_plan::R& r, size_t n) -> cudaError_t {
    if (!dst || n == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, w + r.off, n, cudaMemcpyDeviceToDevice, s);
  };
  GC(out(initial_cot->position, p->r_lpos, (size_t)D.N * 8));
  GC(out(initial_cot->velocity, p->r_lvel, (size_t)D.N * 8));
  GC(out(initial_cot->theta, p->r_lth, (size_t)D.E * 4));
  GC(out(initial_cot->f_grid, lfcur ? p->r_lf1 : p->r_lf0, 9 * LHW * 4));
  if (grads) {
    GC(out(grads->act_c, p->r_dc, (size_t)D.B * 4));
    GC(out(grads->act_amp, p->r_da, (size_t)D.B * 4));
    GC(out(grads->act_phase, p->r_dp, (size_t)D.B * 4));
    GC(out(grads->act_omega, p->r_do, (size_t)D.B * 4));
    GC(out(grads->rest_angles, p->r_dr, (size_t)D.B * 4));
    GC(out(grads->rest_lengths, p->r_dl, (size_t)D.E * 4));
    GC(out(grads->bending_stiffness, p->r_dk, (size_t)D.B * 4));
  }
  GC(cudaGetLastError());
  return MC_OK;
}

}  // extern "C"
