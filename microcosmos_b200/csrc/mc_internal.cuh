// Internal declarations shared by the kernels and the host runtime.
//
// Every kernel takes the plan's rollout descriptor table (RDesc[n], device memory)
// and a per-kernel CTA offset table cta_off[n+1]: CTA b works for rollout
// r = max{r : cta_off[r] <= b} on its local block b - cta_off[r].  A single
// rollout is the batch of one, so the plain and batched paths share every kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define MC_EPSIL 1.1920928955078125e-07f  // float32 eps (src/microcosmos/utils.py:9)
#define MC_PI_F 3.14159265358979323846f
#define MC_2PI_F 6.28318530717958647692f

namespace mc {

constexpr int kBinTile = 16;       // binning tile edge for the deterministic reductions
// threads per CTA of the per-node / per-IB-point kernels and of the per-touched-cell IB
// kernels: 128 spreads the 1024² workload's 16,384 nodes over 128 SMs instead of 64
// (measured: 0.1733 → 0.1720 ms per step; batch 1.990 → 1.982 ms; 64 is no better)
constexpr int kNodeThreads = 128;
// chain rods (one warp each) per CTA of the chain kernel: one spreads the rods over the most
// SMs (measured per batch step: 1.963 ms with 1, 1.965 with 2, 1.973 with 4)
constexpr int kChainWarps = 1;
constexpr int kHeadThreads = 128;
constexpr int kLbmTileX = 128;     // dense LBM CTA tile: 32 lanes x 4 cells
constexpr int kStageCells = 1024;  // staged dense pass: lattice cells per item (a band of whole rows)
constexpr int kStagedThreads = 256;  // ... and threads per CTA (4 cells each)
constexpr int kConvTile = 32;     // steric direct convolution: 32 x 32 outputs per CTA
constexpr int kConvMaxR = 24;     // largest tap radius of the direct convolution       //                    8 rows
constexpr int kIbCap = 1024;       // minimum IB bin capacity per 16x16 tile (grown with node density)
constexpr int kCicCap = 512;       // minimum CIC bin capacity per tile
constexpr int kMaxBinCap = 8192;   // largest bin capacity (the tile sort keeps 4 x cap words in shared memory)
constexpr int kFftMaxN = 4096;     // largest FFT length (shared memory)
constexpr int kFftMaxFactors = 16;
constexpr int kFftColsPerCta = 2;  // complex columns per column-pass CTA (4 real columns)

// Per-rollout descriptor.  All pointers are device pointers.
struct RDesc {
  // sizes
  int H, W, N, E, B, K;  // H, W: the domain grid (positions, steric field); K = ibm_kernel_size
  int lH, lW;            // the fluid lattice (f_grid, IB stencils, force overlay)
  int ncomp;             // rod components
  int NI;                // IB points: N, or 2N with synthetic node pairs
  int M;                 // IB contributions = NI*K*K
  int ntile_x, ntile_y;  // binning tiles (kBinTile) of the domain grid (cloud-in-cell deposit)
  int lntile_x, lntile_y;  // binning tiles of the lattice (IB contributions)
  float rs_inv_y, rs_ks_y, rs_inv_x, rs_ks_x;  // lattice -> domain resize of the recorded u*: 1/scale, kernel width
  int lbm_tx, lbm_ty;    // LBM tiles
  int lbm_tw;            // LBM tile width in cells (32 * cells per lane)
  int lbm_th;            // LBM tile height in rows (threads per CTA = 32 * lbm_th)
  int max_comp_nodes, max_comp_edges, max_comp_pairs;
  // configuration
  float dt, damping, k_stretch, k_shear, vmax, relax, node_mass, wp, wm;
  int solver;       // 0 = PBD rod constraint, 1 = stable Cosserat (projective dynamics)
  float cos_w;      // Cosserat inertia weight 1 / dt_config^2 (float32 of the double value)
  float syn_w;      // synthetic_node_width (0: the IB points are the nodes)
  float syn_ms;     // mean of the two grid scales (float32), multiplies the synthetic offset
  float vmax_q4;  // (vmax / 2)^2 rounded down: below it every velocity clamp factor is exactly 1
  float st_strength, st_sigma, st_scatter;
  float st_2s2, st_norm, st_coef;  // 2 sigma^2, 2 pi sigma^2, scatter / sigma^2 (float32 of the double values)
  int st_skip, ib_iters, cycles, enable_fluid, enable_steric, force_clamp;
  float scale_x, scale_y;   // fluid grid / domain grid, reference axis order
  float sdt_x, sdt_y;       // scale * dt (float32)
  // FFT plans (steric filter)
  int fftW_nf, fftH_nf;
  // power-of-two fast path: threads per transform, transforms per CTA, log2 of the length
  int fft_T_r, fft_tpc_r, fft_logW, fft_T_c, fft_tpc_c, fft_logH;
  int fftW_f[kFftMaxFactors], fftH_f[kFftMaxFactors];
  const float2* twW;  // W roots exp(-2 pi i k / W)
  const float2* twH;
  const float2* ptW;  // the register-radix passes' twiddles of length W, per pass (pass_twiddles)
  const float2* ptH;
  const float* gW;    // separable spectral Gaussian / W
  const float* gH;    // ... / H
  // direct-convolution form of the same filter: the periodic kernel of the spectral
  // Gaussian along x / y, taps for offsets -R..R (symmetric)
  const float* conv_gW;
  const float* conv_gH;
  int conv_RW, conv_RH, conv_ntx;
  // state (caller buffers)
  float* pos;
  float* vel;
  float* theta;
  const float* rest_len;
  float* rest_ang;
  const float* kb;
  float* steric;
  float* fluid_vel;
  float* f_grid;
  // actuation
  const float* act_c;
  const float* act_amp;
  const float* act_omega;
  const float* act_phase;
  int act_t0;
  // recording
  float* rec_pos;
  float* rec_vel;
  float* rec_steric;
  float* rec_fluid;
  int rec_every;
  // topology (workspace)
  const int* pairs;    // (E,2)
  const int* bpairs;   // (B,2)
  const int* comp_n;   // (ncomp+1) node offsets
  const int* comp_e;   // (ncomp+1) edge offsets
  const int* comp_b;   // (ncomp+1) pair offsets
  const int* ep_off;   // (E+1) edge -> bending pairs, (pair<<1)|neg
  const int* ep_idx;
  const int* ne_off;   // (N+1) node -> edges, (edge<<1)|neg
  const int* ne_idx;
  const float* edeg;   // (E,) max(bending degree, 1)
  const float* ndeg;   // (N,) max(node degree, 1)
  // workspace
  float* h[2];         // pull-scheme post-collision populations (9,lH,lW)
  float* dep;          // (H,W) CIC deposit (kept zero between steps)
  float* tmp;          // (H,W) FFT row-pass output
  float* prev;         // (N,2)
  float* pred;         // (N,2)
  float* predw;        // (N,2) prediction wrapped into the domain (steric sampling)
  float* nvl;          // (NI,2) IB point velocity in lattice units
  float* delta;        // (NI,2) IB per-iteration correction
  // Deterministic scatter-add bins.  Contribution k goes to bin tile t at
  // store[t * cap + atomic position]; a tile that fills up spills into the overflow list.
  // store[ntiles * cap ...] is an arena for sorting tiles with more than cap entries.
  // ctl[0] = overflow count, ctl[1] = arena use, ctl[2] = touched-cell (head) count,
  // ctl[3], ctl[4] = arrival count and generation of the fused IB kernel's barrier,
  // ctl[5] = the head count saved by the finalize step for k_collide_heads.
  int ib_cap;
  int* ib_cell;     // (M) cell of contribution k = n*K*K + s
  float* ib_w;      // (M) normalised stencil weight
  int* ib_store;    // (ntiles * ib_cap + 2 * M); after the tile sort: contributing node per run entry
  float* ib_store_w;  // same indexing: the run entry's weight
  int* ib_tcount;   // (ntiles)
  int* ib_ovf;      // (M)
  int* ib_ctl;      // (4)
  int* ib_slot;     // (M) contribution -> head slot of its cell
  // per touched cell ("head"), slots in [0, ctl[2])
  int* h_cell;
  int* h_start;     // position of the cell's sorted run in ib_store
  int* h_len;
  float* s_rho;
  float* s_vx;
  float* s_vy;
  float* s_inv;
  float* s_ucx;
  float* s_ucy;
  float* s_fx;
  float* s_fy;
  // CIC deposit contributions k = corner*N + n (4N)
  int c_cap;
  int* c_cell;
  float* c_w;
  int* c_store;     // (ntiles * c_cap + 8 * N)
  int* c_tcount;
  int* c_ovf;       // (4N)
  int* c_ctl;       // (4)
  // plan-wide lists of bin tiles that received contributions this step: (rollout, tile)
  int ridx;            // this rollout's index in the plan
  int2* wl_ib;
  int2* wl_cic;
  int* wl_ctl;         // [0] IB list length, [1] CIC list length, [2] / [3] their cursors
  // rod components: chains (warp kernel) and general graphs (CTA kernel)
  int nchain, ngeneric;
  const int* chain_comp;    // (nchain) component index
  const int* generic_comp;  // (ngeneric)
  unsigned* flags;  // MC_FLAG_* for this rollout
};

struct Batch {
  const RDesc* d;  // device descriptor table
  int n;
};

__device__ __forceinline__ int find_rollout(const int* __restrict__ off, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Floored float modulo, the semantics of jnp.mod / numpy.mod for floats (y > 0 here):
// r = fmodf(x, y); r += y if r is nonzero with the sign opposite to y.
// For |x| < 2y, fmodf(x, y) is x or x -/+ y, and both subtractions are exact (Sterbenz),
// so the shortcut below returns the same bits as the fmodf route.
__device__ __forceinline__ float fmod_floor(float x, float y) {
  if (fabsf(x) < 2.0f * y) {
    // both signs' results are formed and one is selected (no divergent branch)
    const float rp = (x >= y) ? x - y : x;
    float rn = (x <= -y) ? x + y : x;
    rn = (rn < 0.0f) ? rn + y : rn;
    return (x >= 0.0f) ? rp : rn;
  }
  float r = fmodf(x, y);
  if (r != 0.0f && ((r < 0.0f) != (y < 0.0f))) r += y;
  return r;
}

__device__ __forceinline__ int imod_floor(int x, int m) {
  int r = x % m;
  return r < 0 ? r + m : r;
}

// utils.displacement for one (x, y) pair, size (H, W) flipped to (W, H)
// (src/microcosmos/utils.py:18-23): mod(a - b + L/2, L) - L/2.
__device__ __forceinline__ float2 min_image(float ax, float ay, float bx, float by, float W, float H) {
  float hx = W / 2.0f, hy = H / 2.0f;
  return make_float2(fmod_floor((ax - bx) + hx, W) - hx, fmod_floor((ay - by) + hy, H) - hy);
}

// A bin entry: contribution index k (< 2^24) with its cell's position inside the 16 x 16
// bin tile in the top 8 bits, so the tile kernel sorts without looking the cell up.
__device__ __forceinline__ int bin_entry(int cy, int cx, int k) {
  return (int)((((unsigned)(cy % kBinTile) * kBinTile + (unsigned)(cx % kBinTile)) << 24) | (unsigned)k);
}

// Stable-Cosserat pull of an edge angle toward its segment's direction (sx, sy):
// th + wrap(atan2(sy, sx) - th) * 0.05 (solver/stable_cosserat.py:55-82)
__device__ __forceinline__ float cos_pull(float th, float sx, float sy) {
  const float alpha = atan2f(sy, sx);
  return th + (fmod_floor((alpha - th) + MC_PI_F, MC_2PI_F) - MC_PI_F) * 0.05f;
}

__device__ __forceinline__ float nan_f() { return __int_as_float(0x7fffffff); }
__device__ __forceinline__ bool is_sentinel(float v) { return __float_as_int(v) == 0x7fffffff; }

// ------------------------------------------------------------------ launch helpers
// (host) kernels launched by the runtime; each takes the descriptor table, the CTA
// offset table for its kind, and the number of rollouts.
struct Launch {
  const RDesc* d;
  const int* off;
  int n;
  int grid;
  cudaStream_t s;
};

void launch_predict(const Launch& L);
// wl_count: the list length; wl_count[2] is the cursor the CTAs take tiles from (reset to 0
// with the list)
void launch_bin_tiles(const Launch& L, const int2* wl, int* wl_count, int which, int parity, int capS,
                      int threads = 256);
cudaError_t tiles_blocks_per_sm(int threads, int capS, int* out);
cudaError_t tiles_set_smem(size_t bytes);
void launch_fft_rows(const Launch& L, size_t smem);
void launch_fft_cols(const Launch& L, size_t smem);
void launch_node(const Launch& L, const int* tdev, size_t smem, int bs);
void launch_chain(const Launch& L, const int* tdev, int slots);
void launch_steric(const Launch& L);
void launch_stencil(const Launch& L);
void launch_stencil16(const Launch& L);
void launch_ib_interp(const Launch& L, int it);
void launch_ib_spread(const Launch& L, int it, int fuse_finalize);
void launch_ib_finalize(const Launch& L, int parity);
cudaError_t launch_ib_coop(const Launch& L, int parity);
cudaError_t ib_coop_blocks_per_sm(int* out);
cudaError_t launch_ib_cluster(const RDesc* d, int n, int ctas, int threads, cudaStream_t s);
cudaError_t ib_cluster_allow_16();
void launch_lbm(const Launch& L, int parity, int write_u, int vec, int rows);
bool is_dense_pass_kernel(const void* f);
void launch_lbm_staged(const Launch& L, int parity, int write_u, int stages, int ctas);
size_t lbm_staged_smem(int stages);
cudaError_t lbm_staged_set_smem(size_t bytes);
cudaError_t lbm_staged_blocks_per_sm(int stages, int* out);
void launch_collide_heads(const Launch& L, int parity, int write_u);
void launch_steric_conv(const Launch& L, size_t smem);
void launch_fftreg_rows(const Launch& L, int values_per_thread);
void launch_fft12_rows(const Launch& L);
void launch_fft12_cols(const Launch& L);
void launch_fftreg_cols(const Launch& L, int values_per_thread, int values_per_cta);
void launch_reaction(const Launch& L, const int* tdev);
void launch_record_fields(const Launch& L, const int* tdev);
void launch_unstream(const Launch& L);
void launch_stream_out(const Launch& L, int parity, float* dst = nullptr);
void launch_clear_ws(const Launch& L);
void launch_tick(int* tdev, cudaStream_t s);
cudaError_t fft_set_smem(size_t rows, size_t cols);
void launch_fft_rows_p2(const Launch& L, size_t smem);
void launch_fft_cols_p2(const Launch& L, size_t smem);
cudaError_t fft_p2_set_smem(size_t bytes);
void set_last_error(const char* msg);  // text returned by mc_last_error() on this thread

// Host -> device copies staged through pinned host memory.  A cudaMemcpyAsync from
// pageable memory first waits for all earlier work of its stream, which would make plan
// construction and rollout set-up wait for the rollouts already running on that stream;
// staged copies are enqueued without waiting.  The source may be released on return.
struct Upload {
  void* dst;
  const void* src;
  size_t bytes;
};
cudaError_t stage_uploads(const Upload* items, int count, cudaStream_t s);

}  // namespace mc

struct mc_plan;

namespace mc {

// The steric filter of rollout 0 of a plan applied to other arrays (the gradient path uses
// it: the filter is its own adjoint).  filter_prepare writes a descriptor and CTA offset
// tables (filter_desc_bytes() bytes at `dev`) naming in -> tmp -> out; it needs the plan's
// descriptor of a rollout call (mc_rollout_begin has run once).  filter_launch enqueues
// the same row and column kernels as a step.
size_t filter_desc_bytes();
cudaError_t filter_prepare(mc_plan* p, void* dev, const float* in, float* tmp, float* out, cudaStream_t s);
void filter_launch(mc_plan* p, const void* dev, cudaStream_t s);
cudaError_t node_set_smem(size_t bytes);

}  // namespace mc
