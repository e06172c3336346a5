// Host runtime behind the C ABI (include/microcosmos_b200.h): plan construction
// (topology gather lists, FFT tables, workspace layout, CTA offset tables), workspace
// binding, and the per-step launch sequence with optional CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/microcosmos_b200.h"
#include "mc_internal.cuh"

using mc::RDesc;

namespace {

thread_local std::string g_err;

mc_status fail(mc_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

mc_status cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return MC_ERR_CUDA;
}

#define MC_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }


constexpr int kDefaultSortCap = 2048;  // contributions per tile sorted in shared memory by default
// largest plan (IB points over all rollouts) whose body force is computed by the last IB round
constexpr long long kFuseFinalizeMaxPoints = 65536;

enum Kind { K_NODES = 0, K_COMP, K_CHAIN, K_IB, K_TILES, K_LBM, K_CELLS, K_FFTR, K_FFTC, K_NODES16, K_IBCOOP, K_FFTR2, K_FFTC2, K_SCONV, K_FR16, K_FC16, K_FR12, K_FC12, K_COUNT };

// CTAs of the steric filter kernels for one rollout: the radix-16 register kernels for
// power-of-two sides >= 16, the mixed-radix Stockham kernels for the other FFT sides, or
// the direct convolution.
struct StericCtas {
  int fftr2 = 0, fftc2 = 0, sconv = 0, fr16 = 0, fc16 = 0, fr12 = 0, fc12 = 0;
};

// N = 3 * 2^a with 12 <= N <= 1536: the twelve-values-per-thread register kernels
bool three_pow2(int N) {
  if (N % 3 != 0 || N < 12 || N > 1536) return false;
  const int q = N / 3;
  return (q & (q - 1)) == 0;
}

struct Region {
  size_t off = 0;
  size_t bytes = 0;
};

struct HostRollout {
  mc_dims dims{};
  mc_config cfg{};
  float dt = 0.f;
  std::vector<int> pairs, bpairs;
  std::vector<int> comp_n, comp_e, comp_b, ep_off, ep_idx, ne_off, ne_idx;
  std::vector<float> edeg, ndeg;
  int ncomp = 0, max_cn = 0, max_ce = 0, max_cb = 0;
  std::vector<int> chain_comp, generic_comp;  // components by kernel
  int max_chain = 0;                          // longest chain (nodes)
  std::vector<int> fW, fH;
  std::vector<float2> twW, twH;
  std::vector<float2> ptW, ptH;  // the register-radix FFT's twiddles laid out per pass (bind time)
  std::vector<float> gW, gH;
  std::vector<float> cgW, cgH;  // direct-convolution taps of the steric filter
  int cRW = 0, cRH = 0;
  bool fft_ok = false, conv_ok = false, use_conv = false;
  Region r_cgW, r_cgH;
  int M = 0, ntx = 0, nty = 0, lbm_tx = 0, lbm_ty = 0, vec = 4, lbm_th = 4;
  int lH = 0, lW = 0;      // the fluid lattice (= dims.H, dims.W unless dims.fluid_H/W are set)
  int lntx = 0, lnty = 0;  // bin tiles of the lattice (IB); ntx, nty: of the domain grid (CIC)
  int ib_cap = 0, c_cap = 0;  // bin capacities (powers of two)
  int logW = -1, logH = -1;   // log2 of power-of-two grid sides (-1: mixed radix path)
  int T_r = 0, P_r = 0, T_c = 0, P_c = 0;
  // workspace regions (offsets relative to the workspace base)
  Region r_h0, r_h1, r_dep, r_tmp, r_prev, r_pred, r_predw, r_nvl, r_delta;
  Region r_ibcell, r_ibw, r_ibstore, r_ibstorew, r_ibtc, r_ibovf, r_ibctl, r_ibslot, r_hcell, r_hstart, r_hlen, r_srho, r_svx,
      r_svy, r_sinv, r_sucx, r_sucy, r_sfx, r_sfy;
  Region r_ccell, r_cw, r_cstore, r_ctc, r_covf, r_cctl, r_chain, r_generic;
  Region r_pairs, r_bpairs, r_compn, r_compe, r_compb, r_epo, r_epi, r_neo, r_nei, r_edeg, r_ndeg;
  Region r_twW, r_twH, r_ptW, r_ptH, r_gW, r_gH, r_flags;
};

}  // namespace

struct mc_plan {
  int n = 0;
  std::vector<HostRollout> R;
  size_t ws_bytes = 0;
  Region r_desc, r_tdev, r_wl_ib, r_wl_cic, r_wl_ctl;
  int tile_grid = 1;     // CTAs walking the tile lists (set at bind: as many as the GPU holds)
  int tile_grid_c = 1;   // the same for the cloud-in-cell tiles (their shared sort capacity differs)
  long long n_tiles = 0;  // bin tiles of all rollouts
  int bin_threads = 128;  // threads per CTA of the tile kernel
  int lbm_vec = 2, lbm_rows = 4;  // tile of the direct dense-pass kernel: cells per lane, rows per CTA
  int lbm_stages = 0;       // > 0: the staged dense-pass kernel, with that many bands in flight per CTA
  int lbm_staged_ctas = 0;  // its persistent grid (set at bind: as many CTAs as the GPU holds)
  int ib_capS = 0, c_capS = 0;  // largest bin capacity of the plan
  int ib_smem = 0, c_smem = 0;  // contributions a tile may hold to be sorted in shared memory
  Region r_off[K_COUNT];
  std::vector<int> off[K_COUNT];
  int grid[K_COUNT] = {};
  char* ws = nullptr;
  bool bound = false;
  int any_fluid = 0, any_steric = 0, max_iters = 0;
  size_t node_smem = 0, fftr_smem = 0, fftc_smem = 0, fftr2_smem = 0, fftc2_smem = 0, sconv_smem = 0;
  int node_bs = 32;
  int max_chain = 0, chain_slots = 1;
  int max_k = 0;  // largest IB kernel size of the plan
  int fft_e = 4;  // values per thread of the register-radix FFT kernels
  bool fuse_finalize = false;  // body force computed by the last IB spread round
  int fft_tv = 4096;  // values per CTA of the register-radix column pass (4096 or 2048)
  bool use_coop = false, coop_cap_checked = false;
  bool fused_ib = false;  // mc_plan_set_fused_ib (separate launches measured faster)
  int ib_cluster = 0;     // mc_plan_set_ib_cluster: CTAs per rollout cluster (0: separate launches)
  bool coop_possible = false;
  cudaError_t coop_err = cudaSuccess;
  std::vector<RDesc> desc;
  cudaStream_t cap_stream = nullptr;
  // CUDA graphs, keyed by [steps-1][parity][recording variant][write_u][runs next pipeline]
  cudaGraphExec_t graph[2][2][3][2][2] = {};
  int64_t graph_kernels[2][2][3][2][2] = {};
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t lbm_stream = nullptr;                  // the dense pass, beside the IB chain
  cudaEvent_t ev_lfork = nullptr, ev_ljoin = nullptr;
  bool pending_next = false;  // the next step's pipeline has already been launched
  int64_t last_launches = 0;
  // rollout in progress (mc_rollout_begin .. mc_rollout_end)
  bool active = false;
  int step = 0;
  int rec_fields = 0, rec_fluid = 0;
  // per-kernel CUDA-event profiling (direct launches only)
  bool profiling = false;
  struct Ev {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Ev> ev_pending;
  std::vector<cudaEvent_t> ev_pool;
  double prof_ms[32] = {};
  int64_t prof_n[32] = {};
};

namespace {

bool factorize(int N, std::vector<int>& f) {
  f.clear();
  while (N % 4 == 0) { f.push_back(4); N /= 4; }
  const int ps[] = {2, 3, 5, 7, 11, 13};
  for (int p : ps)
    while (N % p == 0) { f.push_back(p); N /= p; }
  return N == 1 && (int)f.size() <= mc::kFftMaxFactors;
}

// Periodic kernel of the spectral Gaussian exp(-2 pi^2 sigma^2 f^2) on N points (numpy
// fftfreq abscissae): g[k] = (1/N) sum_j kf_j cos(2 pi j k / N), even in k.  The filter is
// cut off at the Nyquist frequency, where it is still exp(-pi^2 sigma^2 / 2) (1.5e-5 for
// sigma = 1.5), so g has a slowly decaying tail of ~1e-6 g[0] beyond the Gaussian core.
// Returns the radius R = min(N/2, kConvMaxR) up to which taps are kept (or the radius where
// |g| first drops below 1e-10 g[0], if that is smaller) and the taps for offsets -R..R.
// Dropping the tail changes the filtered field by ~1e-6 relative (1.4e-6 rel-L2 measured
// for sigma = 1.5 at R = 12, 6e-7 at R = 24).
int conv_taps_compute(int N, double sigma, std::vector<float>& taps) {
  // only offsets up to kConvMaxR + 1 decide R and are kept; the spectrum is evaluated once
  const int kmax = std::min(N / 2, mc::kConvMaxR + 1);
  std::vector<double> spec(N);
  for (int j = 0; j < N; ++j) {
    const double f = (j < (N + 1) / 2 ? (double)j : (double)(j - N)) / (double)N;
    spec[j] = std::exp(-2.0 * M_PI * M_PI * sigma * sigma * f * f);
  }
  std::vector<double> g(kmax + 1);
  for (int k = 0; k <= kmax; ++k) {
    double s = 0.0;
    for (int j = 0; j < N; ++j) s += spec[j] * std::cos(2.0 * M_PI * (double)j * k / N);
    g[k] = s / N;
  }
  int R = 0;
  while (R + 1 <= N / 2 && R + 1 <= mc::kConvMaxR && std::fabs(g[R + 1]) > 1e-10 * std::fabs(g[0])) ++R;
  taps.clear();
  for (int k = -R; k <= R; ++k) taps.push_back((float)g[std::abs(k)]);
  return R;
}

// The steric tables depend only on (N, sigma): computed once per pair for the process and
// copied into each plan (a serving or batching loop builds many plans over the same sides).
struct StericTables {
  int R = 0;
  std::vector<float> taps;
  std::vector<float2> tw;
  std::vector<float> g;
};
std::mutex g_tables_mutex;
std::map<std::pair<int, double>, StericTables> g_tables;

void fft_tables_compute(int N, double sigma, std::vector<float2>& tw, std::vector<float>& g);

const StericTables& steric_tables(int N, double sigma) {
  std::lock_guard<std::mutex> lock(g_tables_mutex);
  auto key = std::make_pair(N, sigma);
  auto it = g_tables.find(key);
  if (it == g_tables.end()) {
    StericTables t;
    t.R = conv_taps_compute(N, sigma, t.taps);
    fft_tables_compute(N, sigma, t.tw, t.g);
    it = g_tables.emplace(key, std::move(t)).first;
  }
  return it->second;
}

int conv_taps(int N, double sigma, std::vector<float>& taps) {
  const StericTables& t = steric_tables(N, sigma);
  taps = t.taps;
  return t.R;
}

void fft_tables(int N, double sigma, std::vector<float2>& tw, std::vector<float>& g) {
  const StericTables& t = steric_tables(N, sigma);
  tw = t.tw;
  g = t.g;
}

void fft_tables_compute(int N, double sigma, std::vector<float2>& tw, std::vector<float>& g) {
  tw.resize(N);
  g.resize(N);
  for (int k = 0; k < N; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)N;
    tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    // numpy.fft.fftfreq abscissa
    const double f = (k < (N + 1) / 2 ? (double)k : (double)(k - N)) / (double)N;
    g[k] = (float)(std::exp(-2.0 * M_PI * M_PI * sigma * sigma * f * f) / (double)N);
  }
}

// The twiddles of the register-radix Stockham passes (steric.cu, pass_reg) for a
// power-of-two length N and E values per thread, laid out per pass: the pass with Ns
// (the product of the earlier radices) and radix R keeps, for each k < Ns, the R - 1
// factors tw[(m k) << (log N - log Ns - log R)], m = 1..R-1, at (Ns - 1) + k (R - 1) + m - 1
// (the passes' tables fill [0, N - 1) exactly).  The same values as the root table, so
// the transform's results are unchanged; a thread reads its factors from one base address.
void pass_twiddles(const std::vector<float2>& tw, int E, std::vector<float2>& pt) {
  const int N = (int)tw.size();
  pt.assign(N, make_float2(0.f, 0.f));
  if (N < 2 || (N & (N - 1))) return;
  int logN = 0;
  while ((1 << logN) < N) ++logN;
  const int LE = E == 4 ? 2 : E == 8 ? 3 : 4;
  int logNs = 0;
  while (logNs < logN) {
    const int LR = logNs + LE <= logN ? LE : logN - logNs;
    const int R = 1 << LR, Ns = 1 << logNs, tsh = logN - logNs - LR;
    for (int k = 0; k < Ns; ++k)
      for (int m = 1; m < R; ++m) pt[(Ns - 1) + k * (R - 1) + (m - 1)] = tw[(m * k) << tsh];
    logNs += LR;
  }
}

// Topology: rod components and the gather lists that reproduce the reference's in-order
// scatter-adds (pbd.py:26-47, 54-87).
mc_status build_topology(HostRollout& h) {
  const int N = h.dims.N, E = h.dims.E, B = h.dims.B;
  for (int e = 0; e < E; ++e)
    for (int j = 0; j < 2; ++j)
      if (h.pairs[2 * e + j] < 0 || h.pairs[2 * e + j] >= N)
        return fail(MC_ERR_INVALID, "edge " + std::to_string(e) + " references a node outside [0, N)");
  for (int b = 0; b < B; ++b)
    for (int j = 0; j < 2; ++j)
      if (h.bpairs[2 * b + j] < 0 || h.bpairs[2 * b + j] >= E)
        return fail(MC_ERR_INVALID, "bending pair " + std::to_string(b) + " references an edge outside [0, E)");
  // edge -> bending pairs: all pairs where it is e_in (ascending), then all where it is
  // e_out; node -> edges: edges where it is src (ascending), then edges where it is tgt.
  // Both are built as CSR lists by counting, then filling in index order.
  {
    std::vector<int> cin(E, 0), cout(E, 0);
    for (int b = 0; b < B; ++b) {
      cin[h.bpairs[2 * b]]++;
      cout[h.bpairs[2 * b + 1]]++;
    }
    h.ep_off.assign(E + 1, 0);
    h.edeg.assign(E, 1.f);
    for (int e = 0; e < E; ++e) {
      h.ep_off[e + 1] = h.ep_off[e] + cin[e] + cout[e];
      h.edeg[e] = (float)std::max(cin[e] + cout[e], 1);
    }
    h.ep_idx.assign(h.ep_off[E], 0);
    std::vector<int> fin(E, 0), fout(E, 0);
    for (int b = 0; b < B; ++b) {
      const int ei = h.bpairs[2 * b], eo = h.bpairs[2 * b + 1];
      h.ep_idx[h.ep_off[ei] + fin[ei]++] = b << 1;
      h.ep_idx[h.ep_off[eo] + cin[eo] + fout[eo]++] = (b << 1) | 1;
    }
  }
  {
    std::vector<int> csrc(N, 0), ctgt(N, 0);
    for (int e = 0; e < E; ++e) {
      csrc[h.pairs[2 * e]]++;
      ctgt[h.pairs[2 * e + 1]]++;
    }
    h.ne_off.assign(N + 1, 0);
    h.ndeg.assign(N, 1.f);
    for (int v = 0; v < N; ++v) {
      h.ne_off[v + 1] = h.ne_off[v] + csrc[v] + ctgt[v];
      h.ndeg[v] = (float)std::max(csrc[v] + ctgt[v], 1);
    }
    h.ne_idx.assign(h.ne_off[N], 0);
    std::vector<int> fs(N, 0), ft(N, 0);
    for (int e = 0; e < E; ++e) {
      const int a = h.pairs[2 * e], b = h.pairs[2 * e + 1];
      h.ne_idx[h.ne_off[a] + fs[a]++] = e << 1;
      h.ne_idx[h.ne_off[b] + csrc[b] + ft[b]++] = (e << 1) | 1;
    }
  }
  // connected components (union-find over edges)
  std::vector<int> par(N);
  for (int i = 0; i < N; ++i) par[i] = i;
  auto find = [&](int x) {
    while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
    return x;
  };
  for (int e = 0; e < E; ++e) {
    int a = find(h.pairs[2 * e]), b = find(h.pairs[2 * e + 1]);
    if (a != b) par[std::max(a, b)] = std::min(a, b);
  }
  // components must be contiguous node ranges whose edges and pairs are contiguous
  // ranges in the same order; otherwise the whole graph is one component
  std::vector<int> cid(N);
  std::vector<int> root_to_c(N, -1);
  bool ok = true;
  int nc = 0, last_root = -1;
  for (int i = 0; i < N; ++i) {
    int rt = find(i);
    if (rt != last_root) {
      if (root_to_c[rt] != -1) ok = false;
      root_to_c[rt] = nc++;
      last_root = rt;
    }
    cid[i] = root_to_c[rt];
  }
  std::vector<int> ce(nc + 1, 0), cb(nc + 1, 0), cn(nc + 1, 0);
  if (ok) {
    for (int i = 0; i < N; ++i) cn[cid[i] + 1]++;
    int prev = 0;
    for (int e = 0; e < E && ok; ++e) {
      int c = cid[h.pairs[2 * e]];
      if (c < prev) ok = false;
      prev = c;
      ce[c + 1]++;
    }
    prev = 0;
    for (int b = 0; b < B && ok; ++b) {
      int c = cid[h.pairs[2 * h.bpairs[2 * b]]];
      int c2 = cid[h.pairs[2 * h.bpairs[2 * b + 1]]];
      if (c != c2 || c < prev) ok = false;
      prev = c;
      cb[c + 1]++;
    }
  }
  if (ok && nc > 0) {
    for (int c = 0; c < nc; ++c) {
      cn[c + 1] += cn[c];
      ce[c + 1] += ce[c];
      cb[c + 1] += cb[c];
    }
    h.comp_n = cn;
    h.comp_e = ce;
    h.comp_b = cb;
    h.ncomp = nc;
  } else {
    h.comp_n = {0, N};
    h.comp_e = {0, E};
    h.comp_b = {0, B};
    h.ncomp = 1;
  }
  // chains (edge i = (n0+i, n0+i+1), pair i = (e0+i, e0+i+1), <= 256 nodes) run on the
  // warp kernel; every other component on the CTA kernel
  h.chain_comp.clear();
  h.generic_comp.clear();
  h.max_chain = 0;
  for (int c = 0; c < h.ncomp; ++c) {
    const int n0 = h.comp_n[c], nn = h.comp_n[c + 1] - n0;
    const int e0 = h.comp_e[c], ne = h.comp_e[c + 1] - e0;
    const int b0 = h.comp_b[c], nb = h.comp_b[c + 1] - b0;
    bool chain = nn >= 1 && nn <= 256 && ne == nn - 1 && nb == std::max(nn - 2, 0);
    for (int i = 0; chain && i < ne; ++i)
      chain = h.pairs[2 * (e0 + i)] == n0 + i && h.pairs[2 * (e0 + i) + 1] == n0 + i + 1;
    for (int i = 0; chain && i < nb; ++i)
      chain = h.bpairs[2 * (b0 + i)] == e0 + i && h.bpairs[2 * (b0 + i) + 1] == e0 + i + 1;
    if (chain) {
      h.chain_comp.push_back(c);
      h.max_chain = std::max(h.max_chain, nn);
    } else {
      h.generic_comp.push_back(c);
    }
  }
  h.max_cn = h.max_ce = h.max_cb = 1;
  for (int c = 0; c < h.ncomp; ++c) {
    h.max_cn = std::max(h.max_cn, h.comp_n[c + 1] - h.comp_n[c]);
    h.max_ce = std::max(h.max_ce, h.comp_e[c + 1] - h.comp_e[c]);
    h.max_cb = std::max(h.max_cb, h.comp_b[c + 1] - h.comp_b[c]);
  }
  return MC_OK;
}

struct Layout {
  size_t cur = 0;
  Region take(size_t bytes) {
    Region r;
    r.off = cur;
    r.bytes = bytes;
    cur = align_up(cur + std::max<size_t>(bytes, 1), 256);
    return r;
  }
};

int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

template <typename T>
T* at(char* base, const Region& r) {
  return reinterpret_cast<T*>(base + r.off);
}

void fill_desc(mc_plan* p, int i, const mc_state* st, const mc_actuation* act, const mc_record* rec) {
  HostRollout& h = p->R[i];
  RDesc d;
  std::memset(&d, 0, sizeof(d));
  char* b = p->ws;
  d.H = h.dims.H;
  d.W = h.dims.W;
  d.N = h.dims.N;
  d.E = h.dims.E;
  d.B = h.dims.B;
  d.K = h.cfg.ibm_kernel_size;
  d.ncomp = h.ncomp;
  d.M = h.M;
  d.NI = h.dims.N * (h.cfg.synthetic_node_width > 0.0f ? 2 : 1);
  d.ntile_x = h.ntx;
  d.ntile_y = h.nty;
  d.lH = h.lH;
  d.lW = h.lW;
  d.lntile_x = h.lntx;
  d.lntile_y = h.lnty;
  d.lbm_tx = h.lbm_tx;
  d.lbm_ty = h.lbm_ty;
  d.lbm_tw = 32 * h.vec;
  d.lbm_th = h.lbm_th;
  const mc_config& c = h.cfg;
  d.dt = h.dt;
  d.damping = c.damping;
  d.k_stretch = c.stiffness_stretch;
  d.k_shear = c.stiffness_shear;
  d.solver = c.solver_type;
  d.syn_w = c.synthetic_node_width;
  d.cos_w = (float)(1.0 / (c.solver_dt * c.solver_dt));
  // mean_scale = 1 (fluid grid == domain grid) but scale keeps the reference's axis order
  // scale = (w / grid_shape[0], h / grid_shape[1]) with (h, w) the lattice (fluid.py:222-226)
  const double sx = (double)h.lW / (double)h.dims.H, sy = (double)h.lH / (double)h.dims.W;
  {
    // linear resize of the recorded u* from the lattice to the domain grid: 1/scale and the
    // antialiasing kernel width max(1/scale, 1) per axis
    const double iy = 1.0 / ((double)h.dims.H / (double)h.lH), ix = 1.0 / ((double)h.dims.W / (double)h.lW);
    d.rs_inv_y = (float)iy;
    d.rs_inv_x = (float)ix;
    d.rs_ks_y = std::max((float)iy, 1.0f);
    d.rs_ks_x = std::max((float)ix, 1.0f);
  }
  d.scale_x = (float)sx;
  d.scale_y = (float)sy;
  d.syn_ms = (float)(0.5 * (sx + sy));
  d.vmax = (float)((double)c.max_fluid_velocity * (0.5 * (sx + sy)));
  d.vmax_q4 = std::nextafter((float)(0.25 * (double)d.vmax * (double)d.vmax), 0.0f);
  d.sdt_x = d.scale_x * h.dt;
  d.sdt_y = d.scale_y * h.dt;
  d.relax = c.ibm_relaxation;
  d.node_mass = c.node_mass;
  {
    // omega+ = clip(1/(3 nu + 0.5), 0, 1.9); omega- from Lambda (fluid.py:155-161, 342-344)
    double wpd = 1.0 / (3.0 * (double)c.viscosity + 0.5);
    wpd = std::min(std::max(wpd, 0.0), 1.9);
    const float eps = 1.1920928955078125e-07f;
    float wp = (float)wpd;
    float offs = 1.0f / std::max(wp, eps) - 0.5f;
    float wm = 1.0f / (c.lambda_trt / std::max(offs, eps) + 0.5f);
    d.wp = wp;
    d.wm = wm;
  }
  d.st_strength = c.steric_strength;
  d.st_sigma = c.steric_sigma;
  d.st_scatter = c.steric_scatter_value;
  const double sg = (double)c.steric_sigma;
  d.st_2s2 = (float)(2.0 * sg * sg);
  d.st_norm = (float)(2.0 * M_PI * sg * sg);
  d.st_coef = (float)((double)c.steric_scatter_value / (sg * sg));
  d.st_skip = c.steric_neighbor_skip;
  // a rollout without fluid has no IB contributions: the batch's IB iteration kernels
  // must not visit its nodes
  d.ib_iters = c.enable_fluid ? c.ibm_iterations : 0;
  d.cycles = c.cycles_per_step;
  d.enable_fluid = c.enable_fluid ? 1 : 0;
  d.enable_steric = c.enable_steric ? 1 : 0;
  d.force_clamp = c.enable_force_clamp ? 1 : 0;
  d.fft_T_r = h.T_r;
  d.fft_tpc_r = h.P_r;
  d.fft_logW = h.logW;
  d.fft_T_c = h.T_c;
  d.fft_tpc_c = h.P_c;
  d.fft_logH = h.logH;
  d.fftW_nf = (int)h.fW.size();
  d.fftH_nf = (int)h.fH.size();
  for (size_t k = 0; k < h.fW.size(); ++k) d.fftW_f[k] = h.fW[k];
  for (size_t k = 0; k < h.fH.size(); ++k) d.fftH_f[k] = h.fH[k];
  d.twW = at<float2>(b, h.r_twW);
  d.twH = at<float2>(b, h.r_twH);
  d.ptW = at<float2>(b, h.r_ptW);
  d.ptH = at<float2>(b, h.r_ptH);
  d.gW = at<float>(b, h.r_gW);
  d.gH = at<float>(b, h.r_gH);
  d.conv_gW = at<float>(b, h.r_cgW);
  d.conv_gH = at<float>(b, h.r_cgH);
  d.conv_RW = h.cRW;
  d.conv_RH = h.cRH;
  d.conv_ntx = div_up(h.dims.W, mc::kConvTile);
  if (st) {
    d.pos = st->position;
    d.vel = st->velocity;
    d.theta = st->theta;
    d.rest_len = st->rest_lengths;
    d.rest_ang = st->bending_rest_angles;
    d.kb = st->bending_stiffness;
    d.steric = st->steric;
    d.fluid_vel = st->fluid_velocity;
    d.f_grid = st->f_grid;
  }
  if (act) {
    d.act_c = act->c;
    d.act_amp = act->amp;
    d.act_omega = act->omega;
    d.act_phase = act->phase;
    d.act_t0 = act->t0;
  }
  if (rec) {
    d.rec_pos = rec->position;
    d.rec_vel = rec->velocity;
    d.rec_steric = rec->steric;
    d.rec_fluid = rec->fluid_velocity;
    d.rec_every = rec->every;
  }
  d.max_comp_nodes = 0;
  int mcn = 1, mce = 1, mcb = 1;
  for (auto& o : p->R) {
    if (o.generic_comp.empty()) continue;
    mcn = std::max(mcn, o.max_cn);
    mce = std::max(mce, o.max_ce);
    mcb = std::max(mcb, o.max_cb);
  }
  d.max_comp_nodes = mcn;
  d.max_comp_edges = mce;
  d.max_comp_pairs = mcb;
  d.pairs = at<int>(b, h.r_pairs);
  d.bpairs = at<int>(b, h.r_bpairs);
  d.comp_n = at<int>(b, h.r_compn);
  d.comp_e = at<int>(b, h.r_compe);
  d.comp_b = at<int>(b, h.r_compb);
  d.ep_off = at<int>(b, h.r_epo);
  d.ep_idx = at<int>(b, h.r_epi);
  d.ne_off = at<int>(b, h.r_neo);
  d.ne_idx = at<int>(b, h.r_nei);
  d.edeg = at<float>(b, h.r_edeg);
  d.ndeg = at<float>(b, h.r_ndeg);
  d.h[0] = at<float>(b, h.r_h0);
  d.h[1] = at<float>(b, h.r_h1);
  d.dep = at<float>(b, h.r_dep);
  d.tmp = at<float>(b, h.r_tmp);
  d.prev = at<float>(b, h.r_prev);
  d.pred = at<float>(b, h.r_pred);
  d.predw = at<float>(b, h.r_predw);
  d.nvl = at<float>(b, h.r_nvl);
  d.delta = at<float>(b, h.r_delta);
  d.ib_cap = h.ib_cap;
  d.ib_cell = at<int>(b, h.r_ibcell);
  d.ib_w = at<float>(b, h.r_ibw);
  d.ib_store = at<int>(b, h.r_ibstore);
  d.ib_store_w = at<float>(b, h.r_ibstorew);
  d.ib_tcount = at<int>(b, h.r_ibtc);
  d.ib_ovf = at<int>(b, h.r_ibovf);
  d.ib_ctl = at<int>(b, h.r_ibctl);
  d.ib_slot = at<int>(b, h.r_ibslot);
  d.h_cell = at<int>(b, h.r_hcell);
  d.h_start = at<int>(b, h.r_hstart);
  d.h_len = at<int>(b, h.r_hlen);
  d.s_rho = at<float>(b, h.r_srho);
  d.s_vx = at<float>(b, h.r_svx);
  d.s_vy = at<float>(b, h.r_svy);
  d.s_inv = at<float>(b, h.r_sinv);
  d.s_ucx = at<float>(b, h.r_sucx);
  d.s_ucy = at<float>(b, h.r_sucy);
  d.s_fx = at<float>(b, h.r_sfx);
  d.s_fy = at<float>(b, h.r_sfy);
  d.c_cap = h.c_cap;
  d.c_cell = at<int>(b, h.r_ccell);
  d.c_w = at<float>(b, h.r_cw);
  d.c_store = at<int>(b, h.r_cstore);
  d.c_tcount = at<int>(b, h.r_ctc);
  d.c_ovf = at<int>(b, h.r_covf);
  d.c_ctl = at<int>(b, h.r_cctl);
  d.ridx = i;
  d.wl_ib = at<int2>(b, p->r_wl_ib);
  d.wl_cic = at<int2>(b, p->r_wl_cic);
  d.wl_ctl = at<int>(b, p->r_wl_ctl);
  d.nchain = (int)h.chain_comp.size();
  d.ngeneric = (int)h.generic_comp.size();
  d.chain_comp = at<int>(b, h.r_chain);
  d.generic_comp = at<int>(b, h.r_generic);
  d.flags = at<unsigned>(b, h.r_flags);
  p->desc[i] = d;
}

// The staged dense pass copies whole 16-byte aligned rows of at most kStageCells cells.
bool lbm_staging_fits(const mc_plan* p) {
  for (const auto& h : p->R)
    if (h.cfg.enable_fluid && (h.lW % 4 != 0 || h.lW > mc::kStageCells)) return false;
  return true;
}

// The dense pass's work table for the plan's current kernel: tiles of lbm_vec * 32 columns x
// lbm_rows rows (direct kernel) or bands of whole rows of about kStageCells cells (staged
// kernel), per rollout, and the CTA / item offsets of K_LBM.
void lbm_tiles(mc_plan* p) {
  int prev = 0;
  for (int i = 0; i < p->n; ++i) {
    HostRollout& h = p->R[i];
    if (p->lbm_stages > 0) {
      h.vec = 4;
      h.lbm_th = std::min(h.lH, std::max(1, mc::kStageCells / h.lW));
      h.lbm_tx = 1;
    } else {
      h.vec = p->lbm_vec;
      h.lbm_th = p->lbm_rows;
      h.lbm_tx = div_up(h.lW, 32 * h.vec);
    }
    h.lbm_ty = div_up(h.lH, h.lbm_th);
    if (!p->off[K_LBM].empty()) {
      p->off[K_LBM][i] = prev;
      prev += h.cfg.enable_fluid ? h.lbm_tx * h.lbm_ty : 0;
    }
  }
  if (!p->off[K_LBM].empty()) {
    p->off[K_LBM][p->n] = prev;
    p->grid[K_LBM] = prev;
  }
}

mc::Launch L(mc_plan* p, Kind k, cudaStream_t s) {
  mc::Launch l;
  l.d = at<RDesc>(p->ws, p->r_desc);
  l.off = at<int>(p->ws, p->r_off[k]);
  l.n = p->n;
  l.grid = p->grid[k];
  l.s = s;
  return l;
}

const char* const kProfNames[] = {"predict", "cic_bins",  "fft_rows",    "fft_cols", "chain",
                                   "node",    "ib_bins",   "ib_interp",   "ib_spread", "ib_finalize",
                                   "lbm",     "reaction",  "record_fields", "tick",    "steric",
                                   "stencil", "ib_fused", "steric_conv", "collide_heads", "ib_cluster"};
constexpr int kNumProf = sizeof(kProfNames) / sizeof(kProfNames[0]);

cudaEvent_t take_event(mc_plan* p) {
  if (!p->ev_pool.empty()) {
    cudaEvent_t e = p->ev_pool.back();
    p->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

// Runs `launch` bracketed by two events when profiling (direct launches only).
template <typename F>
void timed(mc_plan* p, int kind, cudaStream_t s, bool capture, F&& launch) {
  if (!p->profiling || capture) {
    launch();
    return;
  }
  cudaEvent_t a = take_event(p), b = take_event(p);
  if (!a || !b) {
    launch();
    return;
  }
  cudaEventRecord(a, s);
  launch();
  cudaEventRecord(b, s);
  p->ev_pending.push_back({kind, a, b});
}

// One step (src/microcosmos/simulate.py:37-100) is launched as three pieces:
//   pipeline(t): predict, CIC deposit, steric filter, rod kernels      (simulate.py:41-84)
//   ib(t):       IB bins, multi-direct forcing iterations, body force   (fluid.py:268-339)
//   lbm(t):      the dense stream + collide pass                        (fluid.py:341-357)
//   tail(t):     node reaction, wrap, recording, step counter           (fluid.py:359-382)
// pipeline(t+1) depends only on tail(t), so it runs on a second stream concurrently with
// lbm(t); ib(t+1) joins both.  Per-step field recording needs lbm(t) before tail(t)'s
// field copy and before pipeline(t+1) rewrites the steric field, so it runs sequentially.
// e: values per thread of the register-radix kernels (4, 8 or 16); a side of length N takes
// them when it is a power of two with E <= N <= 256 E.  tv: values per column-pass CTA.
StericCtas steric_ctas(const HostRollout& h, int e, int tv) {
  StericCtas c;
  if (!h.cfg.enable_steric) return c;
  if (h.use_conv) {
    c.sconv = div_up(h.dims.W, mc::kConvTile) * div_up(h.dims.H, mc::kConvTile);
    return c;
  }
  const int W = h.dims.W, H = h.dims.H;
  if (h.logW >= 4 && W >= e && W <= 256 * e) c.fr16 = div_up(div_up(H, 2), 256 * e / W);
  else if (three_pow2(W)) c.fr12 = div_up(div_up(H, 2), 256 / (W / 12));
  else c.fftr2 = div_up(div_up(H, 2), h.P_r);
  if (h.logH >= 4 && H >= e && H <= 256 * e) c.fc16 = div_up(div_up(W, 2), tv / H);
  else if (three_pow2(H)) c.fc12 = div_up(div_up(W, 2), 384 / (H / 12));
  else c.fftc2 = div_up(W, 2 * h.P_c);
  return c;
}

// Values per thread of the register-radix FFT kernels for a plan: enough threads to fill
// the GPU (148 SMs x 1024) with the fewest instructions per value.
int default_fft_values(const std::vector<HostRollout>& R) {
  long long cplx = 0;
  for (auto& h : R)
    if (h.cfg.enable_steric && !h.use_conv) cplx += (long long)h.dims.H * h.dims.W / 2;
  const long long fill = 148LL * 1024;
  if (cplx >= 16 * fill) return 16;
  if (cplx >= 8 * fill) return 8;
  return 4;
}

// Values per CTA of the register-radix column pass: 4096, or 2048 when that many would give
// the plan fewer than two column CTAs per SM (148 SMs) and every such side fits 2048.
int default_fft_cols_tv(const std::vector<HostRollout>& R, int e) {
  long long ctas = 0;
  int maxH = 0;
  for (auto& h : R) {
    const StericCtas c = steric_ctas(h, e, 4096);
    if (c.fc16) {
      ctas += c.fc16;
      maxH = std::max(maxH, h.dims.H);
    }
  }
  return (ctas > 0 && ctas < 2 * 148 && maxH <= 2048) ? 2048 : 4096;
}

void recount_steric(mc_plan* p);

void recount_steric(mc_plan* p) {
  p->fft_tv = default_fft_cols_tv(p->R, p->fft_e);
  for (int k : {K_FFTR2, K_FFTC2, K_SCONV, K_FR16, K_FC16, K_FR12, K_FC12}) p->off[k][0] = 0;
  for (int i = 0; i < p->n; ++i) {
    const StericCtas c = steric_ctas(p->R[i], p->fft_e, p->fft_tv);
    p->off[K_FFTR2][i + 1] = p->off[K_FFTR2][i] + c.fftr2;
    p->off[K_FFTC2][i + 1] = p->off[K_FFTC2][i] + c.fftc2;
    p->off[K_SCONV][i + 1] = p->off[K_SCONV][i] + c.sconv;
    p->off[K_FR16][i + 1] = p->off[K_FR16][i] + c.fr16;
    p->off[K_FC16][i + 1] = p->off[K_FC16][i] + c.fc16;
    p->off[K_FR12][i + 1] = p->off[K_FR12][i] + c.fr12;
    p->off[K_FC12][i + 1] = p->off[K_FC12][i] + c.fc12;
  }
  for (int k : {K_FFTR2, K_FFTC2, K_SCONV, K_FR16, K_FC16, K_FR12, K_FC12}) p->grid[k] = p->off[k][p->n];
}

int64_t enqueue_pipeline(mc_plan* p, cudaStream_t s, bool capture) {
  int* tdev = at<int>(p->ws, p->r_tdev);
  int64_t k = 0;
  if (p->grid[K_NODES]) {
    timed(p, 0, s, capture, [&] { mc::launch_predict(L(p, K_NODES, s)); });
    ++k;
  }
  if (p->any_steric) {
    timed(p, 1, s, capture, [&] {
      mc::Launch l = L(p, K_TILES, s);
      l.grid = p->tile_grid_c;
      mc::launch_bin_tiles(l, at<int2>(p->ws, p->r_wl_cic), at<int>(p->ws, p->r_wl_ctl) + 1, 1, 0, p->c_smem,
                           p->bin_threads);
    });
    k += 1;
    if (p->grid[K_FR16]) {
      timed(p, 2, s, capture, [&] { mc::launch_fftreg_rows(L(p, K_FR16, s), p->fft_e); });
      ++k;
    }
    if (p->grid[K_FR12]) {
      timed(p, 2, s, capture, [&] { mc::launch_fft12_rows(L(p, K_FR12, s)); });
      ++k;
    }
    if (p->grid[K_FFTR2]) {
      timed(p, 2, s, capture, [&] { mc::launch_fft_rows_p2(L(p, K_FFTR2, s), p->fftr2_smem); });
      ++k;
    }
    if (p->grid[K_FFTR]) {
      timed(p, 2, s, capture, [&] { mc::launch_fft_rows(L(p, K_FFTR, s), p->fftr_smem); });
      ++k;
    }
    if (p->grid[K_FC16]) {
      timed(p, 3, s, capture, [&] { mc::launch_fftreg_cols(L(p, K_FC16, s), p->fft_e, p->fft_tv); });
      ++k;
    }
    if (p->grid[K_FC12]) {
      timed(p, 3, s, capture, [&] { mc::launch_fft12_cols(L(p, K_FC12, s)); });
      ++k;
    }
    if (p->grid[K_FFTC2]) {
      timed(p, 3, s, capture, [&] { mc::launch_fft_cols_p2(L(p, K_FFTC2, s), p->fftc2_smem); });
      ++k;
    }
    if (p->grid[K_FFTC]) {
      timed(p, 3, s, capture, [&] { mc::launch_fft_cols(L(p, K_FFTC, s), p->fftc_smem); });
      ++k;
    }
    if (p->grid[K_SCONV]) {
      timed(p, 17, s, capture, [&] { mc::launch_steric_conv(L(p, K_SCONV, s), p->sconv_smem); });
      ++k;
    }
  }
  if (p->grid[K_NODES]) {
    timed(p, 14, s, capture, [&] { mc::launch_steric(L(p, K_NODES, s)); });
    ++k;
  }
  if (p->grid[K_CHAIN]) {
    timed(p, 4, s, capture, [&] { mc::launch_chain(L(p, K_CHAIN, s), tdev, p->chain_slots); });
    ++k;
  }
  if (p->grid[K_COMP]) {
    timed(p, 5, s, capture, [&] { mc::launch_node(L(p, K_COMP, s), tdev, p->node_smem, p->node_bs); });
    ++k;
  }
  if (p->grid[K_NODES]) {
    if (p->max_k <= 4)
      timed(p, 15, s, capture, [&] { mc::launch_stencil16(L(p, K_NODES16, s)); });
    else
      timed(p, 15, s, capture, [&] { mc::launch_stencil(L(p, K_NODES, s)); });
    ++k;
  }
  return k;
}

int64_t enqueue_ib(mc_plan* p, int parity, cudaStream_t s, bool capture) {
  if (!p->any_fluid) return 0;
  int64_t k = 0;
  timed(p, 6, s, capture, [&] {
    mc::Launch l = L(p, K_TILES, s);
    l.grid = p->tile_grid;
    mc::launch_bin_tiles(l, at<int2>(p->ws, p->r_wl_ib), at<int>(p->ws, p->r_wl_ctl), 0, parity, p->ib_smem,
                         p->bin_threads);
  });
  ++k;
  if (p->ib_cluster > 0 && p->grid[K_NODES]) {
    timed(p, 19, s, capture, [&] {
      // a lone rollout needs all the threads a cluster can hold; a batch many small clusters
      p->coop_err = mc::launch_ib_cluster(at<RDesc>(p->ws, p->r_desc), p->n, p->ib_cluster, p->n == 1 ? 1024 : 256, s);
    });
    return k + 1;
  }
  if (p->use_coop && p->grid[K_NODES]) {
    timed(p, 16, s, capture, [&] { p->coop_err = mc::launch_ib_coop(L(p, K_IBCOOP, s), parity); });
    return k + 1;
  }
  // rollouts without nodes have no IB points: nothing to launch when no rollout has any
  if (!p->grid[K_NODES] || !p->grid[K_IB]) return k;
  // when every rollout runs max_iters rounds, the last spread also computes the body force
  const int fuse = p->fuse_finalize ? 1 : 0;
  for (int it = 0; it < p->max_iters; ++it) {
    timed(p, 7, s, capture, [&] { mc::launch_ib_interp(L(p, K_NODES, s), it); });
    timed(p, 8, s, capture, [&] { mc::launch_ib_spread(L(p, K_IB, s), it, fuse); });
    k += 2;
  }
  if (fuse) return k;
  timed(p, 9, s, capture, [&] { mc::launch_ib_finalize(L(p, K_IB, s), parity); });
  return k + 1;
}

int64_t enqueue_lbm(mc_plan* p, int parity, int write_u, cudaStream_t s, bool capture) {
  if (!p->any_fluid) return 0;
  if (p->lbm_stages > 0)
    timed(p, 10, s, capture,
          [&] { mc::launch_lbm_staged(L(p, K_LBM, s), parity, write_u, p->lbm_stages, p->lbm_staged_ctas); });
  else
    timed(p, 10, s, capture, [&] { mc::launch_lbm(L(p, K_LBM, s), parity, write_u, p->lbm_vec, p->lbm_rows); });
  return 1;
}

// The IB-touched cells collided with their body force over the dense pass's result.
int64_t enqueue_heads(mc_plan* p, int parity, int write_u, cudaStream_t s, bool capture) {
  if (!p->any_fluid || !p->grid[K_NODES] || !p->grid[K_IB]) return 0;
  timed(p, 18, s, capture, [&] { mc::launch_collide_heads(L(p, K_IB, s), parity, write_u); });
  return 1;
}

int64_t enqueue_tail(mc_plan* p, int rec_fields, cudaStream_t s, bool capture) {
  int* tdev = at<int>(p->ws, p->r_tdev);
  int64_t k = 0;
  if (p->grid[K_NODES]) {
    timed(p, 11, s, capture, [&] { mc::launch_reaction(L(p, K_NODES, s), tdev); });
    ++k;
  }
  if (rec_fields) {
    timed(p, 12, s, capture, [&] { mc::launch_record_fields(L(p, K_CELLS, s), tdev); });
    ++k;
  }
  timed(p, 13, s, capture, [&] { mc::launch_tick(tdev, s); });
  return k + 1;
}

// Everything of step t after its pipeline, plus pipeline(t+1) when has_next.
//   lbm stream: the dense pass lbm(t) (reads h[parity], writes h[parity^1]) from the start
//               of the body, concurrently with the IB chain, which reads h[parity] only;
//   main:       ib(t) (bins, iterations, body force per touched cell), then, once lbm(t)
//               is done, the touched cells' collision over its result;
//   side:       after ib(t): tail(t) (node reaction) and pipeline(t+1).
// The next body starts when all three have finished.
int64_t enqueue_body(mc_plan* p, int parity, int write_u, int rec_fields, bool has_next, cudaStream_t s,
                     bool capture, mc_status* err) {
  if (rec_fields || p->profiling) {
    // sequential: field recording needs this order; profiling times kernels one at a time
    int64_t k = enqueue_ib(p, parity, s, capture);
    k += enqueue_lbm(p, parity, write_u, s, capture);
    k += enqueue_heads(p, parity, write_u, s, capture);
    k += enqueue_tail(p, rec_fields, s, capture);
    if (has_next) k += enqueue_pipeline(p, s, capture);
    return k;
  }
  auto fork = [&](cudaEvent_t ev, cudaStream_t from, cudaStream_t to, const char* what) {
    cudaError_t e = cudaEventRecord(ev, from);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(to, ev, 0);
    if (e != cudaSuccess && *err == MC_OK) *err = cuda_fail(e, what);
  };
  int64_t k = 0;
  cudaStream_t s2 = p->side_stream, s3 = p->lbm_stream;
  if (p->any_fluid) {
    fork(p->ev_lfork, s, s3, "fork to the dense-pass stream");
    k += enqueue_lbm(p, parity, write_u, s3, capture);
  }
  k += enqueue_ib(p, parity, s, capture);
  fork(p->ev_fork, s, s2, "fork to the side stream");
  k += enqueue_tail(p, 0, s2, capture);
  if (has_next) k += enqueue_pipeline(p, s2, capture);
  if (p->any_fluid) {
    fork(p->ev_ljoin, s3, s, "join from the dense-pass stream");
    k += enqueue_heads(p, parity, write_u, s, capture);
  }
  fork(p->ev_join, s2, s, "join from the side stream");
  return k;
}

// Kernel-node priorities of a captured step graph: the dense pass (off the step's critical
// path: only the touched-cell collision waits for it) gets the device's lowest priority and
// every other kernel (the IB chain, the node pipeline) the highest, so that whenever CTAs of
// both are waiting, the block scheduler starts the critical path's first.  The graph is
// instantiated with cudaGraphInstantiateFlagUseNodePriority; priorities change no result.
cudaError_t prioritise_graph(cudaGraph_t graph) {
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e != cudaSuccess) return e;
  size_t n = 0;
  e = cudaGraphGetNodes(graph, nullptr, &n);
  if (e != cudaSuccess || n == 0) return e;
  std::vector<cudaGraphNode_t> nodes(n);
  e = cudaGraphGetNodes(graph, nodes.data(), &n);
  if (e != cudaSuccess) return e;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    e = cudaGraphNodeGetType(nodes[i], &t);
    if (e != cudaSuccess) return e;
    if (t != cudaGraphNodeTypeKernel) continue;
    cudaKernelNodeParams kp;
    e = cudaGraphKernelNodeGetParams(nodes[i], &kp);
    if (e != cudaSuccess) return e;
    cudaKernelNodeAttrValue v;
    std::memset(&v, 0, sizeof(v));
    v.priority = mc::is_dense_pass_kernel(kp.func) ? least : greatest;
    e = cudaGraphKernelNodeSetAttribute(nodes[i], cudaKernelNodeAttributePriority, &v);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

mc_status run_steps(mc_plan* p, int num, int use_graph, int last, cudaStream_t s, int64_t& launches) {
  const int recv = p->rec_fields ? (p->rec_fluid ? 2 : 1) : 0;
  // the first step of this call needs its node pipeline unless the previous call left it
  // pending (an advance with last != 0 finishes its step without starting the next one)
  if (!p->pending_next && num > 0) launches += enqueue_pipeline(p, s, false);
  int remaining = num;
  while (remaining > 0) {
    const int parity = p->step & 1;
    const bool is_last = last && remaining == 1;
    const int write_u = (is_last || p->rec_fluid) ? 1 : 0;
    const bool has_next = !is_last;
    mc_status err = MC_OK;
    if (use_graph && !p->profiling) {
      // two steps per graph where possible (parity 0 then 1, neither the final step)
      const int ns = (parity == 0 && remaining >= 3) ? 2 : 1;
      const int wu = ns == 2 ? p->rec_fluid : write_u;
      const int nx = has_next ? 1 : 0;
      cudaGraphExec_t& g = p->graph[ns - 1][parity][recv][wu][nx];
      if (!g) {
        cudaGraph_t graph;
        MC_CUDA(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
        int64_t kk = 0;
        for (int j = 0; j < ns && err == MC_OK; ++j)
          kk += enqueue_body(p, (parity + j) & 1, wu, p->rec_fields, j + 1 < ns ? true : has_next, p->cap_stream,
                             true, &err);
        cudaError_t e = cudaStreamEndCapture(p->cap_stream, &graph);
        if (err != MC_OK) return err;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = prioritise_graph(graph);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          g = nullptr;
          return cuda_fail(e, "cudaGraphInstantiate");
        }
        p->graph_kernels[ns - 1][parity][recv][wu][nx] = kk;
      }
      MC_CUDA(cudaGraphLaunch(g, s));
      launches += p->graph_kernels[ns - 1][parity][recv][wu][nx];
      p->step += ns;
      remaining -= ns;
      p->pending_next = has_next;
      continue;
    }
    launches += enqueue_body(p, parity, write_u, p->rec_fields, has_next, s, false, &err);
    if (err != MC_OK) return err;
    p->step += 1;
    remaining -= 1;
    p->pending_next = has_next;
  }
  return MC_OK;
}

void destroy_graphs(mc_plan* p) {
  for (auto& a : p->graph)
    for (auto& b : a)
      for (auto& c : b)
        for (auto& e : c)
          for (auto& g : e)
            if (g) {
              cudaGraphExecDestroy(g);
              g = nullptr;
            }
}

}  // namespace

namespace mc {
void set_last_error(const char* msg) { g_err = msg; }

namespace {
// Rings of pinned host memory, one per host thread that uploads (a thread's ring goes back to
// a free list when the thread exits, for the next new thread; rings are never freed, so that
// no copy can outlive its source).  Each batch of uploads reserves the next span of the
// calling thread's ring, copies its sources there and enqueues the device copies, then
// records an event; a span is reused only after its event has completed (spans are handed
// out in ring order, so the spans in the way are always the oldest live ones).  A thread
// therefore only ever waits for its own earlier uploads: a ring shared by all threads made a
// thread wait for another thread's stream (a serving loop's next epoch behind a gradient
// job's queued reverse steps).  A ring grows (after its live spans complete) when one batch
// does not fit.
struct StageRing {
  char* buf = nullptr;
  size_t cap = 0;
  bool failed = false;
  size_t head = 0;
  struct Span {
    size_t lo, hi;
    cudaEvent_t ev;
  };
  std::deque<Span> live;
  std::vector<cudaEvent_t> pool;
};
constexpr size_t kRingBytes = size_t(16) << 20;  // initial size of a thread's ring
std::mutex g_rings_m;
std::vector<StageRing*> g_free_rings;
struct RingHolder {
  StageRing* r = nullptr;
  ~RingHolder() {
    if (!r) return;
    std::lock_guard<std::mutex> lock(g_rings_m);
    g_free_rings.push_back(r);
  }
};
thread_local RingHolder t_ring;

StageRing& my_ring() {
  if (!t_ring.r) {
    std::lock_guard<std::mutex> lock(g_rings_m);
    if (!g_free_rings.empty()) {
      t_ring.r = g_free_rings.back();
      g_free_rings.pop_back();
    } else {
      t_ring.r = new StageRing;
    }
  }
  return *t_ring.r;
}

// Wait for the ring's oldest live span; false on a CUDA error (returned in *err).
bool retire_oldest(StageRing& g, cudaError_t* err) {
  const cudaError_t e = cudaEventSynchronize(g.live.front().ev);
  if (e != cudaSuccess) {
    *err = e;
    return false;
  }
  g.pool.push_back(g.live.front().ev);
  g.live.pop_front();
  return true;
}
}  // namespace

cudaError_t stage_uploads(const Upload* items, int count, cudaStream_t s) {
  size_t total = 0;
  for (int i = 0; i < count; ++i) total += (items[i].bytes + 15) & ~size_t(15);
  if (total == 0) return cudaSuccess;
  StageRing& g = my_ring();
  cudaError_t err = cudaSuccess;
  if (!g.failed && (!g.buf || total > g.cap)) {
    // first use, or a batch larger than the ring: (re)allocate once nothing is in flight
    while (!g.live.empty())
      if (!retire_oldest(g, &err)) return err;
    size_t want = g.cap ? g.cap : kRingBytes;
    while (want < total) want *= 2;
    if (g.buf) cudaFreeHost(g.buf);
    g.buf = nullptr;
    g.cap = 0;
    g.head = 0;
    void* b = nullptr;
    if (cudaHostAlloc(&b, want, cudaHostAllocDefault) == cudaSuccess) {
      g.buf = static_cast<char*>(b);
      g.cap = want;
    } else {
      cudaGetLastError();
      g.failed = true;
    }
  }
  if (!g.buf) {
    // no staging memory: plain copies (correct, but they wait for the stream)
    for (int i = 0; i < count; ++i) {
      if (!items[i].bytes) continue;
      cudaError_t e = cudaMemcpyAsync(items[i].dst, items[i].src, items[i].bytes, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  size_t lo = g.head;
  if (lo + total > g.cap) lo = 0;
  const size_t hi = lo + total;
  while (!g.live.empty() && g.live.front().lo < hi && lo < g.live.front().hi)
    if (!retire_oldest(g, &err)) return err;
  size_t off = lo;
  for (int i = 0; i < count; ++i) {
    if (!items[i].bytes) continue;
    std::memcpy(g.buf + off, items[i].src, items[i].bytes);
    cudaError_t e = cudaMemcpyAsync(items[i].dst, g.buf + off, items[i].bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    off += (items[i].bytes + 15) & ~size_t(15);
  }
  cudaEvent_t ev = nullptr;
  if (!g.pool.empty()) {
    ev = g.pool.back();
    g.pool.pop_back();
  } else {
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaEventRecord(ev, s);
  if (e != cudaSuccess) return e;
  g.live.push_back({lo, hi, ev});
  g.head = hi;
  return cudaSuccess;
}

// Inside a rollout (between mc_rollout_begin and mc_rollout_end) of a one-rollout plan:
// write the current populations in fields.f_grid layout into dst, leaving the rollout as
// it is (the gradient plan's segment recompute snapshots every step's input this way).
mc_status rollout_snapshot_f(mc_plan* p, float* dst, cudaStream_t s) {
  if (!p || !p->active || p->n != 1 || !dst) return fail(MC_ERR_INVALID, "snapshot outside a one-rollout rollout");
  if (p->pending_next) return fail(MC_ERR_INVALID, "snapshot while the next step's pipeline is in flight");
  if (p->any_fluid) launch_stream_out(L(p, K_CELLS, s), p->step & 1, dst);
  MC_CUDA(cudaGetLastError());
  return MC_OK;
}

size_t filter_desc_bytes() { return align_up(sizeof(RDesc), 256) + 7 * 256; }

cudaError_t filter_prepare(mc_plan* p, void* dev, const float* in, float* tmp, float* out, cudaStream_t s) {
  if (p->desc.empty()) return cudaErrorInvalidValue;
  RDesc d = p->desc[0];
  d.dep = const_cast<float*>(in);
  d.tmp = tmp;
  d.steric = out;
  const StericCtas c = steric_ctas(p->R[0], p->fft_e, p->fft_tv);
  const int cnt[7] = {c.fr16, c.fftr2, c.sconv, c.fc16, c.fftc2, c.fr12, c.fc12};
  std::vector<unsigned char> host(filter_desc_bytes(), 0);
  std::memcpy(host.data(), &d, sizeof(RDesc));
  for (int k = 0; k < 7; ++k) {
    const int off[2] = {0, cnt[k]};
    std::memcpy(host.data() + align_up(sizeof(RDesc), 256) + 256 * k, off, sizeof(off));
  }
  const Upload u{dev, host.data(), host.size()};
  cudaError_t e = stage_uploads(&u, 1, s);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);  // `host` is a temporary
}

void filter_launch(mc_plan* p, const void* dev, cudaStream_t s) {
  const unsigned char* b = static_cast<const unsigned char*>(dev);
  const StericCtas c = steric_ctas(p->R[0], p->fft_e, p->fft_tv);
  const int cnt[7] = {c.fr16, c.fftr2, c.sconv, c.fc16, c.fftc2, c.fr12, c.fc12};
  auto launch = [&](int k) {
    Launch l;
    l.d = reinterpret_cast<const RDesc*>(b);
    l.off = reinterpret_cast<const int*>(b + align_up(sizeof(RDesc), 256) + 256 * k);
    l.n = 1;
    l.grid = cnt[k];
    l.s = s;
    return l;
  };
  if (cnt[0]) launch_fftreg_rows(launch(0), p->fft_e);
  if (cnt[5]) launch_fft12_rows(launch(5));
  if (cnt[1]) launch_fft_rows_p2(launch(1), p->fftr2_smem);
  if (cnt[2]) launch_steric_conv(launch(2), p->sconv_smem);
  if (cnt[3]) launch_fftreg_cols(launch(3), p->fft_e, p->fft_tv);
  if (cnt[6]) launch_fft12_cols(launch(6));
  if (cnt[4]) launch_fft_cols_p2(launch(4), p->fftc2_smem);
}
}  // namespace mc

extern "C" {

const char* mc_last_error(void) { return g_err.c_str(); }
const char* mc_version(void) { return "microcosmos_b200 0.1.0 (sm_100a)"; }

mc_status mc_plan_create(int32_t n, const mc_dims* dims, const mc_config* cfg, const float* dt,
                         const int32_t* const* pairs, const int32_t* const* bending_pairs, mc_plan** out) {
  g_err.clear();
  if (!out || n <= 0 || !dims || !cfg || !dt || !pairs || !bending_pairs) return fail(MC_ERR_INVALID, "null argument");
  *out = nullptr;
  mc_plan* p = new mc_plan();
  p->n = n;
  p->R.resize(n);
  Layout lay;
  p->r_desc = lay.take(sizeof(RDesc) * n);
  p->r_tdev = lay.take(sizeof(int));
  p->r_wl_ctl = lay.take(4 * sizeof(int));
  for (int k = 0; k < K_COUNT; ++k) p->r_off[k] = lay.take(sizeof(int) * (n + 1));
  int vec_all = -1;
  for (int i = 0; i < n; ++i) {
    HostRollout& h = p->R[i];
    h.dims = dims[i];
    h.cfg = cfg[i];
    h.dt = dt[i];
    const mc_dims& D = h.dims;
    const mc_config& c = h.cfg;
    if (D.H < 4 || D.W < 4 || D.N < 0 || D.E < 0 || D.B < 0) {
      delete p;
      return fail(MC_ERR_INVALID, "rollout " + std::to_string(i) + ": grid must be at least 4x4 and counts >= 0");
    }
    h.lH = D.fluid_H > 0 ? D.fluid_H : D.H;
    h.lW = D.fluid_W > 0 ? D.fluid_W : D.W;
    if (D.fluid_H < 0 || D.fluid_W < 0 || h.lH < 4 || h.lW < 4 || h.lH > 7 * D.H || h.lW > 7 * D.W) {
      delete p;
      return fail(MC_ERR_INVALID, "rollout " + std::to_string(i) +
                                      ": the fluid grid must be at least 4x4 and at most 7 times the domain grid");
    }
    if ((D.E > 0 && !pairs[i]) || (D.B > 0 && !bending_pairs[i])) {
      delete p;
      return fail(MC_ERR_INVALID, "null topology array");
    }
    if (!(c.synthetic_node_width >= 0.0f)) {
      delete p;
      return fail(MC_ERR_INVALID, "synthetic_node_width must be >= 0");
    }
    if (c.solver_type != MC_SOLVER_PBD && c.solver_type != MC_SOLVER_COSSERAT) {
      delete p;
      return fail(MC_ERR_INVALID, "solver_type must be MC_SOLVER_PBD or MC_SOLVER_COSSERAT");
    }
    if (c.solver_type == MC_SOLVER_COSSERAT && !(c.solver_dt > 0.0)) {
      delete p;
      return fail(MC_ERR_INVALID, "the Cosserat solver's dt must be > 0");
    }
    if (c.ibm_kernel_size < 1 || c.ibm_kernel_size > 8) {
      delete p;
      return fail(MC_ERR_UNSUPPORTED, "ibm_kernel_size must be in [1, 8]");
    }
    if (!(dt[i] > 0.0f)) {
      delete p;
      return fail(MC_ERR_INVALID, "dt must be > 0");
    }
    // the dense pass indexes the populations (9, h, w) with 32-bit integers
    {
      const long long lh = D.fluid_H > 0 ? D.fluid_H : D.H, lw = D.fluid_W > 0 ? D.fluid_W : D.W;
      if (9LL * lh * lw >= (1LL << 31)) {
        delete p;
        return fail(MC_ERR_UNSUPPORTED, "fluid lattice too large: 9 * h * w must be below 2^31");
      }
    }
    // IB points: the nodes, or a synthetic pair per node (fluid.py:244-263)
    const long long NI = (long long)D.N * (c.synthetic_node_width > 0.0f ? 2 : 1);
    const long long M = c.enable_fluid ? NI * c.ibm_kernel_size * c.ibm_kernel_size : 0;
    if (M >= (1LL << 24) || 4LL * D.N >= (1LL << 24)) {
      delete p;
      return fail(MC_ERR_UNSUPPORTED, "too many IB contributions for 24-bit sort keys (IB points*K*K < 2^24)");
    }
    h.M = (int)M;
    h.pairs.assign(pairs[i] ? pairs[i] : nullptr, pairs[i] ? pairs[i] + 2 * (size_t)D.E : nullptr);
    h.bpairs.assign(bending_pairs[i] ? bending_pairs[i] : nullptr,
                    bending_pairs[i] ? bending_pairs[i] + 2 * (size_t)D.B : nullptr);
    mc_status st = build_topology(h);
    if (st != MC_OK) {
      delete p;
      return st;
    }
    if (c.enable_steric) {
      h.cRW = conv_taps(D.W, c.steric_sigma, h.cgW);
      h.cRH = conv_taps(D.H, c.steric_sigma, h.cgH);
      h.conv_ok = 2 * h.cRW + 1 <= D.W && 2 * h.cRH + 1 <= D.H;
      h.fft_ok = factorize(D.W, h.fW) && factorize(D.H, h.fH) && D.W <= mc::kFftMaxN && D.H <= mc::kFftMaxN;
      h.use_conv = h.conv_ok && !h.fft_ok;
      if (!h.fft_ok) {
        h.fW.clear();
        h.fH.clear();
      }
      if (!h.conv_ok) {
        h.cgW.clear();
        h.cgH.clear();
      }
    }
    if (c.enable_steric && !h.conv_ok && !h.fft_ok) {
      delete p;
      return fail(MC_ERR_UNSUPPORTED,
                  "steric filter: the FFT needs H, W with prime factors <= 13 and at most 4096, the direct "
                  "convolution a kernel radius below min(H, W) / 2 and 24");
    }
    if (c.enable_steric && h.fft_ok) {
      fft_tables(D.W, c.steric_sigma, h.twW, h.gW);
      fft_tables(D.H, c.steric_sigma, h.twH, h.gH);
      auto log2_if_pow2 = [](int v) {
        int l = 0;
        while ((1 << l) < v) ++l;
        return (1 << l) == v && v >= 16 ? l : -1;
      };
      // threads per transform: one radix-4 butterfly each (N / 4), a power of two dividing the
      // CTA size; transforms per CTA fill the CTA (256 threads for rows, 512 for columns)
      auto threads_for = [](int len, int cta) {
        int t = 32;
        while (t * 2 <= len / 4 && t * 2 <= cta) t *= 2;
        return t;
      };
      h.logW = log2_if_pow2(D.W);
      h.logH = log2_if_pow2(D.H);
      h.T_r = threads_for(D.W, 256);
      h.P_r = 256 / h.T_r;
      h.T_c = threads_for(D.H, 512);
      h.P_c = 512 / h.T_c;
    }
    h.vec = (h.lW % 4 == 0) ? 4 : (h.lW % 2 == 0) ? 2 : 1;
    if (vec_all == -1) vec_all = h.vec;
    if (vec_all != h.vec) vec_all = 1;
    h.ntx = div_up(D.W, mc::kBinTile);
    h.nty = div_up(D.H, mc::kBinTile);
    h.lntx = div_up(h.lW, mc::kBinTile);
    h.lnty = div_up(h.lH, mc::kBinTile);
    const size_t HW = (size_t)D.H * D.W, LHW = (size_t)h.lH * h.lW;
    const size_t N = D.N, E = D.E, B = D.B, nt = (size_t)h.ntx * h.nty, lnt = (size_t)h.lntx * h.lnty;
    h.r_h0 = lay.take(9 * LHW * 4);
    h.r_h1 = lay.take(9 * LHW * 4);
    h.r_dep = lay.take(HW * 4);
    h.r_tmp = lay.take(HW * 4);
    h.r_prev = lay.take(2 * N * 4);
    h.r_pred = lay.take(2 * N * 4);
    h.r_predw = lay.take(2 * N * 4);
    const size_t NIz = N * (c.synthetic_node_width > 0.0f ? 2 : 1);
    h.r_nvl = lay.take(2 * NIz * 4);
    h.r_delta = lay.take(2 * NIz * 4);
    const size_t Mz = (size_t)M;
    h.r_ibcell = lay.take(Mz * 4);
    h.r_ibw = lay.take(Mz * 4);
    // bin capacity: at least 3x the mean contributions per tile, a power of two
    auto cap_for = [&](long long contributions, int minimum, size_t tiles) {
      long long want = std::max<long long>(minimum, (3 * contributions + (long long)tiles - 1) / (long long)tiles);
      int c = 1;
      while (c < want && c < mc::kMaxBinCap) c <<= 1;
      return c;
    };
    h.ib_cap = cap_for((long long)Mz, mc::kIbCap, lnt);
    h.c_cap = cap_for(4LL * (long long)N, mc::kCicCap, nt);
    h.r_ibstore = lay.take((lnt * h.ib_cap + 2 * Mz) * 4);
    h.r_ibstorew = lay.take((lnt * h.ib_cap + 2 * Mz) * 4);
    h.r_ibtc = lay.take(lnt * 4);
    h.r_ibovf = lay.take(Mz * 4);
    h.r_ibctl = lay.take(8 * 4);
    h.r_ibslot = lay.take(Mz * 4);
    h.r_hcell = lay.take(Mz * 4);
    h.r_hstart = lay.take(Mz * 4);
    h.r_hlen = lay.take(Mz * 4);
    h.r_srho = lay.take(Mz * 4);
    h.r_svx = lay.take(Mz * 4);
    h.r_svy = lay.take(Mz * 4);
    h.r_sinv = lay.take(Mz * 4);
    h.r_sucx = lay.take(Mz * 4);
    h.r_sucy = lay.take(Mz * 4);
    h.r_sfx = lay.take(Mz * 4);
    h.r_sfy = lay.take(Mz * 4);
    h.r_ccell = lay.take(4 * N * 4);
    h.r_cw = lay.take(4 * N * 4);
    h.r_cstore = lay.take((nt * h.c_cap + 8 * N) * 4);
    h.r_ctc = lay.take(nt * 4);
    h.r_covf = lay.take(4 * N * 4);
    h.r_cctl = lay.take(8 * 4);
    h.r_chain = lay.take(h.chain_comp.size() * 4);
    h.r_generic = lay.take(h.generic_comp.size() * 4);
    h.r_pairs = lay.take(2 * E * 4);
    h.r_bpairs = lay.take(2 * B * 4);
    h.r_compn = lay.take((h.ncomp + 1) * 4);
    h.r_compe = lay.take((h.ncomp + 1) * 4);
    h.r_compb = lay.take((h.ncomp + 1) * 4);
    h.r_epo = lay.take((E + 1) * 4);
    h.r_epi = lay.take(h.ep_idx.size() * 4);
    h.r_neo = lay.take((N + 1) * 4);
    h.r_nei = lay.take(h.ne_idx.size() * 4);
    h.r_edeg = lay.take(E * 4);
    h.r_ndeg = lay.take(N * 4);
    h.r_twW = lay.take(h.twW.size() * 8);
    h.r_twH = lay.take(h.twH.size() * 8);
    h.r_ptW = lay.take(h.twW.size() * 8);
    h.r_ptH = lay.take(h.twH.size() * 8);
    h.r_gW = lay.take(h.gW.size() * 4);
    h.r_gH = lay.take(h.gH.size() * 4);
    h.r_cgW = lay.take(h.cgW.size() * 4);
    h.r_cgH = lay.take(h.cgH.size() * 4);
    h.r_flags = lay.take(4);
    if (c.enable_fluid) p->any_fluid = 1;
    if (c.enable_steric) p->any_steric = 1;
    p->max_iters = std::max(p->max_iters, c.enable_fluid ? c.ibm_iterations : 0);
    p->max_k = std::max(p->max_k, c.ibm_kernel_size);
  }
  // The body force rides on the last multi-direct forcing round when every rollout with a
  // fluid runs the same number of rounds (at least one) and the plan has at most
  // kFuseFinalizeMaxPoints IB points.  Measured (L2 flushed before each step, same bits): one
  // 1024^2 lattice with 16,384 points 0.1674 -> 0.1634 ms per step (one dependent launch
  // less); the 256-rollout batch with 296 k points 1.864 -> 1.892 ms (there the separate
  // pass over the touched cells is faster than the longer last round).
  long long ib_points = 0;
  for (const auto& h : p->R)
    if (h.cfg.enable_fluid) ib_points += (long long)h.dims.N * (h.cfg.synthetic_node_width > 0.0f ? 2 : 1);
  p->fuse_finalize = p->max_iters > 0 && ib_points <= kFuseFinalizeMaxPoints;
  for (const auto& h : p->R)
    if (h.cfg.enable_fluid && h.cfg.ibm_iterations != p->max_iters) p->fuse_finalize = false;
  // default dense-pass tile: 4 cells per lane x 16 rows for plans of >= 4 M lattice cells
  // (measured best at 2048^2 and on the 25 M-cell batch: 0.78 / 0.91 of HBM), 2 x 4 below
  // (best at 1024^2: 20.8 us vs 22.9 us for 4 x 16); narrower when the widths need it
  long long plan_cells = 0;
  for (const auto& h : p->R) plan_cells += (long long)h.lH * h.lW;
  const bool big_plan = plan_cells >= (4LL << 20);
  if (!big_plan && vec_all == 4) vec_all = 2;
  p->lbm_vec = vec_all;
  p->lbm_rows = big_plan ? 16 : 4;
  p->lbm_stages = 0;
  lbm_tiles(p);
  {
    long long tiles = 0, ltiles = 0;
    for (auto& h : p->R) {
      tiles += (long long)h.ntx * h.nty;
      ltiles += (long long)h.lntx * h.lnty;
    }
    p->r_wl_ib = lay.take((size_t)ltiles * sizeof(int2));
    p->r_wl_cic = lay.take((size_t)tiles * sizeof(int2));
    tiles = std::max(tiles, ltiles);
    p->n_tiles = tiles;
    for (auto& h : p->R) {
      p->ib_capS = std::max(p->ib_capS, h.ib_cap);
      p->c_capS = std::max(p->c_capS, h.c_cap);
    }
    // up to 2048 contributions per tile are sorted in shared memory (32 KB per CTA, and only
    // when some rollout's bins are that deep: sparse plans keep their 1024-entry bins): the
    // dense rollouts of a batch then rarely take the global-arena sort, while the residency
    // of the launch's CTAs is not cut further (measured: 2.05 vs 2.10 ms per step of the
    // 256-rollout batch against 1024, 2.23 ms at 4096)
    p->ib_smem = std::min(p->ib_capS, kDefaultSortCap);
    p->c_smem = std::min(p->c_capS, kDefaultSortCap);
  }
  p->ws_bytes = lay.cur;
  // CTA offset tables
  for (int k = 0; k < K_COUNT; ++k) p->off[k].assign(n + 1, 0);
  int mcn = 1, mce = 1, mcb = 1;
  for (int i = 0; i < n; ++i) {
    HostRollout& h = p->R[i];
    const mc_config& c = h.cfg;
    const long long HW = std::max((long long)h.dims.H * h.dims.W, (long long)h.lH * h.lW);
    int cnt[K_COUNT];
    // node kernels cover the IB points too (twice the nodes with synthetic pairs); the
    // node-only kernels return for indices >= N
    const long long npts = (long long)h.dims.N * (c.synthetic_node_width > 0.0f ? 2 : 1);
    cnt[K_NODES] = div_up(npts, mc::kNodeThreads);
    cnt[K_NODES16] = div_up(16LL * npts, 128);
    // fused IB kernel: one thread per touched-cell candidate / 4 (scaled down at bind if
    // the plan's CTAs would not all be resident)
    cnt[K_IBCOOP] = c.enable_fluid ? std::max(1, div_up(h.M, 1024)) : 0;
    cnt[K_COMP] = h.dims.N > 0 ? (int)h.generic_comp.size() : 0;
    cnt[K_CHAIN] = h.dims.N > 0 ? div_up((long long)h.chain_comp.size(), mc::kChainWarps) : 0;
    cnt[K_IB] = div_up(h.M, mc::kHeadThreads);  // touched cells: at most M, one thread each
    cnt[K_TILES] = h.ntx * h.nty;
    cnt[K_LBM] = c.enable_fluid ? h.lbm_tx * h.lbm_ty : 0;
    cnt[K_CELLS] = std::min(div_up(HW, 256), 1024);
    // every length goes through the multi-transform kernels (the one-transform-per-CTA
    // kernels serve the allocation-free entry point)
    cnt[K_FFTR] = 0;
    cnt[K_FFTC] = 0;
    cnt[K_FFTR2] = cnt[K_FFTC2] = cnt[K_SCONV] = cnt[K_FR16] = cnt[K_FC16] = 0;  // recount_steric
    if (h.conv_ok)
      p->sconv_smem = std::max(p->sconv_smem, (size_t)(mc::kConvTile + 2 * h.cRH) *
                                                  (mc::kConvTile + 2 * h.cRW + mc::kConvTile) * sizeof(float));
    if (c.enable_steric && h.fft_ok) {
      p->fftr2_smem = std::max(p->fftr2_smem, (size_t)2 * h.P_r * h.dims.W * sizeof(float2));
      p->fftc2_smem = std::max(p->fftc2_smem, (size_t)2 * h.P_c * (h.dims.H + 1) * sizeof(float2));
    }
    for (int k = 0; k < K_COUNT; ++k) p->off[k][i + 1] = p->off[k][i] + cnt[k];
    if (!h.generic_comp.empty()) {
      mcn = std::max(mcn, h.max_cn);
      mce = std::max(mce, h.max_ce);
      mcb = std::max(mcb, h.max_cb);
    }
    p->max_chain = std::max(p->max_chain, h.max_chain);
    p->fftr_smem = std::max(p->fftr_smem, c.enable_steric && h.fft_ok ? (size_t)3 * h.dims.W * sizeof(float2) + h.dims.W * sizeof(float) : 0);
    p->fftc_smem = std::max(p->fftc_smem,
                            c.enable_steric && h.fft_ok ? (size_t)(2 * mc::kFftColsPerCta + 1) * h.dims.H * sizeof(float2) + h.dims.H * sizeof(float) : 0);
  }
  for (int k = 0; k < K_COUNT; ++k) p->grid[k] = p->off[k][n];
  p->fft_e = default_fft_values(p->R);
  recount_steric(p);
  p->coop_cap_checked = false;
  p->node_smem = (size_t)(2 * mcn + 4 * mce + 3 * mcb) * sizeof(float);
  p->chain_slots = 1;
  while (p->chain_slots * 32 < p->max_chain) p->chain_slots *= 2;
  if (p->node_smem > 200 * 1024) {
    delete p;
    return fail(MC_ERR_UNSUPPORTED, "rod component too large for shared memory (> ~6000 nodes)");
  }
  int work = std::max(mcn, std::max(mce, mcb));
  p->node_bs = std::min(256, std::max(32, (work + 31) / 32 * 32));
  p->desc.resize(n);
  *out = p;
  return MC_OK;
}

mc_status mc_plan_set_bin_threads(mc_plan* p, int32_t threads) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the tile kernel shape is set before mc_plan_bind()");
  if (threads != 0 && threads != 64 && threads != 128 && threads != 256)
    return fail(MC_ERR_INVALID, "threads must be 0 (default), 64, 128 or 256");
  p->bin_threads = threads ? threads : 128;
  return MC_OK;
}

int32_t mc_plan_bin_threads(const mc_plan* p) { return p ? p->bin_threads : 0; }

mc_status mc_plan_set_bin_sort_capacity(mc_plan* p, int32_t entries) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the tile sort capacity is set before mc_plan_bind()");
  if (entries != 0 && (entries < 256 || entries > 8192 || (entries & (entries - 1))))
    return fail(MC_ERR_INVALID, "entries must be 0 (default 2048) or a power of two in 256..8192");
  const int e = entries ? entries : kDefaultSortCap;
  p->ib_smem = std::min(p->ib_capS, e);
  p->c_smem = std::min(p->c_capS, e);
  return MC_OK;
}

int32_t mc_plan_bin_sort_capacity(const mc_plan* p) { return p ? p->ib_smem : 0; }

mc_status mc_plan_set_fft_values_per_thread(mc_plan* p, int32_t values) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the FFT shape is set before mc_plan_bind()");
  if (values != 0 && values != 4 && values != 8 && values != 16)
    return fail(MC_ERR_INVALID, "values per thread must be 0 (default), 4, 8 or 16");
  p->fft_e = values ? values : default_fft_values(p->R);
  recount_steric(p);
  return MC_OK;
}

int32_t mc_plan_fft_values_per_thread(const mc_plan* p) { return p ? p->fft_e : 0; }

mc_status mc_plan_set_steric_method(mc_plan* p, int32_t method) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the steric filter method is set before mc_plan_bind()");
  if (method < 0 || method > 2) return fail(MC_ERR_INVALID, "method must be 0 (auto), 1 (FFT) or 2 (direct)");
  for (auto& h : p->R) {
    if (!h.cfg.enable_steric) continue;
    if (method == 1 && !h.fft_ok) return fail(MC_ERR_UNSUPPORTED, "a rollout's grid has no FFT plan");
    if (method == 2 && !h.conv_ok) return fail(MC_ERR_UNSUPPORTED, "a rollout's grid is too small for the direct filter");
  }
  for (int i = 0; i < p->n; ++i) {
    HostRollout& h = p->R[i];
    h.use_conv = method == 0 ? (h.conv_ok && !h.fft_ok) : method == 2;
  }
  recount_steric(p);
  return MC_OK;
}

int32_t mc_plan_steric_method(const mc_plan* p) {
  if (!p) return -1;
  int conv = 0, fft = 0;
  for (auto& h : p->R)
    if (h.cfg.enable_steric) (h.use_conv ? conv : fft) = 1;
  return conv && fft ? 3 : conv ? 2 : fft ? 1 : 0;
}

mc_status mc_plan_set_lbm_shape(mc_plan* p, int32_t cells_per_lane, int32_t rows_per_cta) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the dense-pass tile shape is set before mc_plan_bind()");
  int vec = cells_per_lane > 0 ? cells_per_lane : p->lbm_vec;
  int rows = rows_per_cta > 0 ? rows_per_cta : p->lbm_rows;
  if (vec != 1 && vec != 2 && vec != 4) return fail(MC_ERR_INVALID, "cells_per_lane must be 1, 2 or 4");
  if (rows != 2 && rows != 4 && rows != 8 && rows != 16 && rows != 32)
    return fail(MC_ERR_INVALID, "rows_per_cta must be 2, 4, 8, 16 or 32");
  for (auto& h : p->R)
    if (h.lW % vec != 0 || h.lW < vec)
      return fail(MC_ERR_UNSUPPORTED, "cells_per_lane must divide every rollout's lattice width");
  p->lbm_vec = vec;
  p->lbm_rows = rows;
  p->lbm_stages = 0;
  lbm_tiles(p);
  return MC_OK;
}

mc_status mc_plan_get_lbm_shape(const mc_plan* p, int32_t* cells_per_lane, int32_t* rows_per_cta) {
  if (!p || !cells_per_lane || !rows_per_cta) return fail(MC_ERR_INVALID, "null argument");
  *cells_per_lane = p->lbm_vec;
  *rows_per_cta = p->lbm_rows;
  return MC_OK;
}

mc_status mc_plan_set_lbm_staging(mc_plan* p, int32_t stages) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->bound) return fail(MC_ERR_INVALID, "the dense-pass staging is set before mc_plan_bind()");
  if (stages != 0 && (stages < 2 || stages > 6)) return fail(MC_ERR_INVALID, "stages must be 0 or 2..6");
  if (stages > 0 && !lbm_staging_fits(p))
    return fail(MC_ERR_UNSUPPORTED, "the staged dense pass needs lattice widths that are multiples of 4 and at most " +
                                        std::to_string(mc::kStageCells));
  p->lbm_stages = stages;
  lbm_tiles(p);
  return MC_OK;
}

int32_t mc_plan_lbm_staging(const mc_plan* p) { return p ? p->lbm_stages : -1; }

void mc_plan_destroy(mc_plan* p) {
  if (!p) return;
  destroy_graphs(p);
  for (auto& e : p->ev_pending) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (auto e : p->ev_pool) cudaEventDestroy(e);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  if (p->side_stream) cudaStreamDestroy(p->side_stream);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  if (p->lbm_stream) cudaStreamDestroy(p->lbm_stream);
  if (p->ev_lfork) cudaEventDestroy(p->ev_lfork);
  if (p->ev_ljoin) cudaEventDestroy(p->ev_ljoin);
  delete p;
}

size_t mc_plan_workspace_bytes(const mc_plan* p) { return p ? p->ws_bytes : 0; }

mc_status mc_plan_bind(mc_plan* p, void* workspace, size_t bytes, void* stream) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (!workspace || bytes < p->ws_bytes) return fail(MC_ERR_WORKSPACE, "workspace missing or smaller than mc_plan_workspace_bytes()");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(MC_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  p->ws = (char*)workspace;
  std::vector<mc::Upload> ups;
  auto up = [&](const Region& r, const void* src, size_t n) -> cudaError_t {
    if (n) ups.push_back({p->ws + r.off, src, n});
    return cudaSuccess;
  };
  for (int i = 0; i < p->n; ++i) {
    HostRollout& h = p->R[i];
    MC_CUDA(up(h.r_pairs, h.pairs.data(), h.pairs.size() * 4));
    MC_CUDA(up(h.r_bpairs, h.bpairs.data(), h.bpairs.size() * 4));
    MC_CUDA(up(h.r_compn, h.comp_n.data(), h.comp_n.size() * 4));
    MC_CUDA(up(h.r_compe, h.comp_e.data(), h.comp_e.size() * 4));
    MC_CUDA(up(h.r_compb, h.comp_b.data(), h.comp_b.size() * 4));
    MC_CUDA(up(h.r_epo, h.ep_off.data(), h.ep_off.size() * 4));
    MC_CUDA(up(h.r_epi, h.ep_idx.data(), h.ep_idx.size() * 4));
    MC_CUDA(up(h.r_neo, h.ne_off.data(), h.ne_off.size() * 4));
    MC_CUDA(up(h.r_nei, h.ne_idx.data(), h.ne_idx.size() * 4));
    MC_CUDA(up(h.r_edeg, h.edeg.data(), h.edeg.size() * 4));
    MC_CUDA(up(h.r_ndeg, h.ndeg.data(), h.ndeg.size() * 4));
    MC_CUDA(up(h.r_chain, h.chain_comp.data(), h.chain_comp.size() * 4));
    MC_CUDA(up(h.r_generic, h.generic_comp.data(), h.generic_comp.size() * 4));
    MC_CUDA(up(h.r_twW, h.twW.data(), h.twW.size() * 8));
    MC_CUDA(up(h.r_twH, h.twH.data(), h.twH.size() * 8));
    pass_twiddles(h.twW, p->fft_e, h.ptW);
    pass_twiddles(h.twH, p->fft_e, h.ptH);
    MC_CUDA(up(h.r_ptW, h.ptW.data(), h.ptW.size() * 8));
    MC_CUDA(up(h.r_ptH, h.ptH.data(), h.ptH.size() * 8));
    MC_CUDA(up(h.r_gW, h.gW.data(), h.gW.size() * 4));
    MC_CUDA(up(h.r_gH, h.gH.data(), h.gH.size() * 4));
    MC_CUDA(up(h.r_cgW, h.cgW.data(), h.cgW.size() * 4));
    MC_CUDA(up(h.r_cgH, h.cgH.data(), h.cgH.size() * 4));
    fill_desc(p, i, nullptr, nullptr, nullptr);
  }
  for (int k = 0; k < K_COUNT; ++k) MC_CUDA(up(p->r_off[k], p->off[k].data(), p->off[k].size() * 4));
  MC_CUDA(up(p->r_desc, p->desc.data(), p->desc.size() * sizeof(RDesc)));
  MC_CUDA(mc::stage_uploads(ups.data(), (int)ups.size(), s));
  // zero the binning counters of every tile before the first clear kernel runs
  {
    // The dynamic shared memory limit is a per-kernel attribute shared by every plan of the
    // process: raise it to the device's opt-in maximum (never lower it to this plan's need,
    // which would break plans with larger grids).
    int dev = 0, optin = 0;
    MC_CUDA(cudaGetDevice(&dev));
    MC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (p->node_smem > (size_t)optin || p->fftr_smem > (size_t)optin || p->fftc_smem > (size_t)optin ||
        p->fftr2_smem > (size_t)optin || p->fftc2_smem + 1024 > (size_t)optin || p->sconv_smem > (size_t)optin)
      return fail(MC_ERR_UNSUPPORTED, "shared memory needed by the plan exceeds the device limit");
    MC_CUDA(mc::node_set_smem((size_t)optin));
    MC_CUDA(mc::tiles_set_smem((size_t)optin));
    if (p->lbm_stages > 0) {
      if (mc::lbm_staged_smem(p->lbm_stages) > (size_t)optin)
        return fail(MC_ERR_UNSUPPORTED, "the staged dense pass's shared memory exceeds the device limit");
      MC_CUDA(mc::lbm_staged_set_smem((size_t)optin));
    }
    if (p->any_steric) {
      MC_CUDA(mc::fft_set_smem((size_t)optin, (size_t)optin));
      MC_CUDA(mc::fft_p2_set_smem((size_t)optin));
    }
  }
  MC_CUDA(cudaMemsetAsync(p->ws + p->r_wl_ctl.off, 0, 4 * sizeof(int), s));
  {
    // the tile kernels take listed tiles from a cursor: launch as many CTAs as fit at once
    int dev = 0, sms = 0, nib = 0, nc = 0;
    MC_CUDA(cudaGetDevice(&dev));
    MC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MC_CUDA(mc::tiles_blocks_per_sm(p->bin_threads, std::max(p->ib_smem, 1), &nib));
    MC_CUDA(mc::tiles_blocks_per_sm(p->bin_threads, std::max(p->c_smem, 1), &nc));
    p->tile_grid = std::max(1, sms * nib);
    p->tile_grid_c = std::max(1, sms * nc);
    if (p->lbm_stages > 0) {
      int nl = 0;
      MC_CUDA(mc::lbm_staged_blocks_per_sm(p->lbm_stages, &nl));
      if (nl < 1) return fail(MC_ERR_UNSUPPORTED, "the staged dense pass does not fit on an SM");
      p->lbm_staged_ctas = sms * nl;
    }
  }
  mc::launch_clear_ws(L(p, K_CELLS, s));
  MC_CUDA(cudaGetLastError());
  destroy_graphs(p);
  if (!p->cap_stream) MC_CUDA(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
  if (!p->side_stream) MC_CUDA(cudaStreamCreateWithFlags(&p->side_stream, cudaStreamNonBlocking));
  if (!p->lbm_stream) MC_CUDA(cudaStreamCreateWithFlags(&p->lbm_stream, cudaStreamNonBlocking));
  {
    // the fused IB kernel needs every CTA resident at once (cooperative launch)
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    MC_CUDA(cudaGetDevice(&dev));
    MC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    MC_CUDA(mc::ib_coop_blocks_per_sm(&per_sm));
    p->coop_possible = coop && p->grid[K_IBCOOP] > 0 && p->grid[K_IBCOOP] <= per_sm * sms;
    p->use_coop = p->fused_ib && p->coop_possible;
  }
  if (!p->ev_fork) MC_CUDA(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  if (!p->ev_join) MC_CUDA(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
  if (!p->ev_lfork) MC_CUDA(cudaEventCreateWithFlags(&p->ev_lfork, cudaEventDisableTiming));
  if (!p->ev_ljoin) MC_CUDA(cudaEventCreateWithFlags(&p->ev_ljoin, cudaEventDisableTiming));
  p->bound = true;
  return MC_OK;
}

mc_status mc_rollout_begin(mc_plan* p, const mc_state* states, const mc_actuation* const* act,
                           const mc_record* const* rec, void* stream) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (!p->bound) return fail(MC_ERR_NOT_BOUND, "mc_plan_bind() was not called");
  if (!states) return fail(MC_ERR_INVALID, "null states");
  cudaStream_t s = (cudaStream_t)stream;
  int rec_fields = 0, rec_fluid = 0;
  for (int i = 0; i < p->n; ++i) {
    const mc_state& st = states[i];
    const HostRollout& h = p->R[i];
    if ((h.dims.N && (!st.position || !st.velocity)) || (h.dims.E && (!st.theta || !st.rest_lengths)) ||
        (h.dims.B && (!st.bending_rest_angles || !st.bending_stiffness)) ||
        (h.cfg.enable_fluid && (!st.f_grid || !st.fluid_velocity)) || (h.cfg.enable_steric && !st.steric))
      return fail(MC_ERR_INVALID, "rollout " + std::to_string(i) + ": null state array");
    if (h.cfg.enable_fluid && (reinterpret_cast<uintptr_t>(st.fluid_velocity) % 16 != 0))
      return fail(MC_ERR_INVALID, "fluid_velocity must be 16-byte aligned");
    const mc_actuation* a = act ? act[i] : nullptr;
    if (a && (!a->c || !a->amp || !a->omega || !a->phase)) return fail(MC_ERR_INVALID, "incomplete actuation");
    const mc_record* r = rec ? rec[i] : nullptr;
    if (r) {
      if (r->every < 1) return fail(MC_ERR_INVALID, "record.every must be >= 1");
      if (r->steric || r->fluid_velocity) rec_fields = 1;
      if (r->fluid_velocity) rec_fluid = 1;
    }
    fill_desc(p, i, &st, a, r);
  }
  {
    const mc::Upload u{p->ws + p->r_desc.off, p->desc.data(), p->desc.size() * sizeof(RDesc)};
    MC_CUDA(mc::stage_uploads(&u, 1, s));
  }
  MC_CUDA(cudaMemsetAsync(at<int>(p->ws, p->r_tdev), 0, sizeof(int), s));
  p->rec_fields = rec_fields;
  p->rec_fluid = rec_fluid;
  p->step = 0;
  p->active = true;
  p->last_launches = 0;
  if (p->any_fluid) {
    mc::launch_unstream(L(p, K_CELLS, s));
    p->last_launches += 1;
  }
  p->pending_next = false;  // the first advance launches step 0's pipeline
  MC_CUDA(cudaGetLastError());
  return MC_OK;
}

mc_status mc_rollout_advance(mc_plan* p, int32_t num_steps, int32_t use_graph, int32_t last, void* stream) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (!p->active) return fail(MC_ERR_INVALID, "mc_rollout_begin() was not called");
  if (num_steps < 0) return fail(MC_ERR_INVALID, "negative num_steps");
  int64_t launches = 0;
  mc_status st = run_steps(p, num_steps, use_graph, last, (cudaStream_t)stream, launches);
  p->last_launches += launches;
  if (p->coop_err != cudaSuccess) {
    cudaError_t e = p->coop_err;
    p->coop_err = cudaSuccess;
    return cuda_fail(e, "cooperative launch of the fused IB kernel");
  }
  if (st != MC_OK) return st;
  MC_CUDA(cudaGetLastError());
  return MC_OK;
}

mc_status mc_rollout_end(mc_plan* p, void* stream) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (!p->active) return fail(MC_ERR_INVALID, "mc_rollout_begin() was not called");
  if (p->pending_next) {
    p->active = false;
    return fail(MC_ERR_INVALID, "the last mc_rollout_advance() before mc_rollout_end() must pass last != 0");
  }
  if (p->any_fluid) {
    mc::launch_stream_out(L(p, K_CELLS, (cudaStream_t)stream), p->step & 1);
    p->last_launches += 1;
  }
  p->active = false;
  MC_CUDA(cudaGetLastError());
  return MC_OK;
}

mc_status mc_rollout(mc_plan* p, const mc_state* states, int32_t num_steps, const mc_actuation* const* act,
                     const mc_record* const* rec, int32_t use_graph, void* stream) {
  if (num_steps < 0) return fail(MC_ERR_INVALID, "negative num_steps");
  mc_status st = mc_rollout_begin(p, states, act, rec, stream);
  if (st != MC_OK) return st;
  st = mc_rollout_advance(p, num_steps, use_graph, 1, stream);
  if (st != MC_OK) {
    p->active = false;
    return st;
  }
  return mc_rollout_end(p, stream);
}

mc_status mc_plan_set_fused_ib(mc_plan* p, int32_t enable) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->active) return fail(MC_ERR_INVALID, "cannot change the IB kernel layout inside a rollout");
  p->fused_ib = enable != 0;
  p->use_coop = p->fused_ib && p->coop_possible;
  destroy_graphs(p);
  return MC_OK;
}

int32_t mc_plan_uses_fused_ib(const mc_plan* p) { return p && p->use_coop ? 1 : 0; }

mc_status mc_plan_set_ib_cluster(mc_plan* p, int32_t ctas) {
  g_err.clear();
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  if (p->active) return fail(MC_ERR_INVALID, "cannot change the IB kernel layout inside a rollout");
  if (ctas < 0 || ctas > 16) return fail(MC_ERR_INVALID, "CTAs per cluster must be in [0, 16]");
  if (ctas > 8) {
    cudaError_t e = mc::ib_cluster_allow_16();
    if (e != cudaSuccess) return cuda_fail(e, "allowing clusters of more than 8 CTAs");
  }
  p->ib_cluster = ctas;
  destroy_graphs(p);
  return MC_OK;
}

int32_t mc_plan_ib_cluster(const mc_plan* p) { return p ? p->ib_cluster : 0; }

mc_status mc_plan_profile(mc_plan* p, int32_t enable) {
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  p->profiling = enable != 0;
  return MC_OK;
}

mc_status mc_plan_profile_read(mc_plan* p, const char* kernel, double* total_ms, int64_t* launches) {
  g_err.clear();
  if (!p || !kernel || !total_ms || !launches) return fail(MC_ERR_INVALID, "null argument");
  for (auto& e : p->ev_pending) {
    float ms = 0.f;
    MC_CUDA(cudaEventSynchronize(e.b));
    MC_CUDA(cudaEventElapsedTime(&ms, e.a, e.b));
    p->prof_ms[e.kind] += ms;
    p->prof_n[e.kind] += 1;
    p->ev_pool.push_back(e.a);
    p->ev_pool.push_back(e.b);
  }
  p->ev_pending.clear();
  for (int k = 0; k < kNumProf; ++k)
    if (std::strcmp(kProfNames[k], kernel) == 0) {
      *total_ms = p->prof_ms[k];
      *launches = p->prof_n[k];
      return MC_OK;
    }
  return fail(MC_ERR_INVALID, std::string("unknown kernel name ") + kernel);
}

mc_status mc_plan_profile_reset(mc_plan* p) {
  if (!p) return fail(MC_ERR_INVALID, "null plan");
  for (int k = 0; k < 32; ++k) {
    p->prof_ms[k] = 0.0;
    p->prof_n[k] = 0;
  }
  return MC_OK;
}

const char* mc_profile_kernel_names(void) {
  static std::string names;
  if (names.empty())
    for (int k = 0; k < kNumProf; ++k) {
      if (k) names += ",";
      names += kProfNames[k];
    }
  return names.c_str();
}

mc_status mc_step(mc_plan* p, const mc_state* states, void* stream) {
  return mc_rollout(p, states, 1, nullptr, nullptr, 0, stream);
}

mc_status mc_plan_read_flags(mc_plan* p, uint32_t* flags, int32_t clear, void* stream) {
  g_err.clear();
  if (!p || !flags) return fail(MC_ERR_INVALID, "null argument");
  if (!p->bound) return fail(MC_ERR_NOT_BOUND, "mc_plan_bind() was not called");
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i < p->n; ++i)
    MC_CUDA(cudaMemcpyAsync(flags + i, p->ws + p->R[i].r_flags.off, 4, cudaMemcpyDeviceToHost, s));
  MC_CUDA(cudaStreamSynchronize(s));
  if (clear)
    for (int i = 0; i < p->n; ++i) MC_CUDA(cudaMemsetAsync(p->ws + p->R[i].r_flags.off, 0, 4, s));
  return MC_OK;
}

int64_t mc_plan_last_launch_count(const mc_plan* p) { return p ? p->last_launches : 0; }

}  // extern "C"
