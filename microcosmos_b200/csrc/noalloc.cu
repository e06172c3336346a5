// mc_steric_potential_noalloc: the steric potential field of a set of node positions
// (cloud-in-cell deposit + spectral Gaussian, the field update_steric_potential computes
// inside every step) for callers that cannot allocate device memory.
//
// All scratch lives in one file-scope __device__ array of fixed size (kNaBytes below): the
// library never calls cudaMalloc/cudaFree here, and the caller passes only the positions
// and the output field.  The kernels are the same ones a rollout step uses.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/microcosmos_b200.h"
#include "mc_internal.cuh"

namespace {

constexpr int kNaMaxGrid = 512;   // H, W <= 512
constexpr int kNaMaxNodes = 16384;
constexpr int kNaMaxTiles = (kNaMaxGrid / mc::kBinTile) * (kNaMaxGrid / mc::kBinTile);

constexpr size_t al(size_t x) { return (x + 255) / 256 * 256; }

// byte offsets of the scratch regions (each 256-byte aligned)
constexpr size_t kOffDesc = 0;
constexpr size_t kOffOff = kOffDesc + al(sizeof(mc::RDesc));                  // 4 kinds x 2 ints
constexpr size_t kOffVel = kOffOff + al(8 * sizeof(int));                      // 2N zeros
constexpr size_t kOffPrev = kOffVel + al(2 * kNaMaxNodes * 4);
constexpr size_t kOffPred = kOffPrev + al(2 * kNaMaxNodes * 4);
constexpr size_t kOffPredw = kOffPred + al(2 * kNaMaxNodes * 4);
constexpr size_t kOffCell = kOffPredw + al(2 * kNaMaxNodes * 4);               // 4N
constexpr size_t kOffW = kOffCell + al(4 * kNaMaxNodes * 4);
constexpr size_t kOffOvf = kOffW + al(4 * kNaMaxNodes * 4);
constexpr size_t kOffStore = kOffOvf + al(4 * kNaMaxNodes * 4);               // tiles*cap + 8N
constexpr size_t kOffTcount = kOffStore + al(((size_t)kNaMaxTiles * mc::kCicCap + 8 * kNaMaxNodes) * 4);
constexpr size_t kOffCtl = kOffTcount + al(kNaMaxTiles * 4);                  // CIC + IB controls
constexpr size_t kOffDep = kOffCtl + al(16 * 4);
constexpr size_t kOffTmp = kOffDep + al((size_t)kNaMaxGrid * kNaMaxGrid * 4);
constexpr size_t kOffTwW = kOffTmp + al((size_t)kNaMaxGrid * kNaMaxGrid * 4);
constexpr size_t kOffTwH = kOffTwW + al(kNaMaxGrid * 8);
constexpr size_t kOffGW = kOffTwH + al(kNaMaxGrid * 8);
constexpr size_t kOffGH = kOffGW + al(kNaMaxGrid * 4);
constexpr size_t kOffFlags = kOffGH + al(kNaMaxGrid * 4);
constexpr size_t kOffWl = kOffFlags + 256;                                    // tile list (int2)
constexpr size_t kOffWlCtl = kOffWl + al(kNaMaxTiles * 8);
constexpr size_t kNaBytes = kOffWlCtl + 256;  // about 6.6 MB

// The scratch.  Every GPU that loads this library holds one copy until the process exits.
// In host code `g_na_scratch` only names the symbol; its device address comes from
// cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_na_scratch[kNaBytes];

mc_status na_fail(mc_status s, const std::string& m) {
  mc::set_last_error(m.c_str());  // reported by mc_last_error()
  return s;
}

// Per-device set-up: the scratch's device address, looked up with cudaGetSymbolAddress on
// the first call made with that device current.  The address belongs to the context that
// loaded the module, so it is cached with that context's unique id: after a context is torn
// down (cudaDeviceReset) and a new one created, the next call looks the address up again.
// (The FFT kernels need at most 23 KB of dynamic shared memory at the 512 x 512 limit,
// under the default 48 KB, so no kernel attribute is changed.)
struct NaDevice {
  unsigned long long ctx_id = 0;
  unsigned char* ptr = nullptr;
};
std::mutex g_na_mutex;
std::vector<NaDevice> g_na_dev;
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;

// id of the calling thread's current context (0 if none is current)
unsigned long long current_ctx_id() {
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

mc_status na_setup(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(MC_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_ctx_current || !g_ctx_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess)
      return na_fail(MC_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId not found");
    g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    g_ctx_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  if ((int)g_na_dev.size() <= dev) g_na_dev.resize(dev + 1);
  NaDevice& nd = g_na_dev[dev];
  const unsigned long long id = current_ctx_id();
  if (!nd.ptr || id == 0 || id != nd.ctx_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess)
      return na_fail(MC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    nd.ptr = static_cast<unsigned char*>(p);
    nd.ctx_id = current_ctx_id();  // the lookup above makes the device's context current
  }
  *out = nd.ptr;
  return MC_OK;
}

// Everything a call writes into the scratch before its kernels run, passed by value as the
// set-up kernel's parameter (about 14 KB, under the 32 KB kernel-parameter limit), so the
// call stages nothing through host memory that outlives it.
struct NaSetup {
  mc::RDesc d;
  int offs[8];
  int N, ntiles;
  size_t HW;
  float2 twW[kNaMaxGrid], twH[kNaMaxGrid];
  float gW[kNaMaxGrid], gH[kNaMaxGrid];
};
static_assert(sizeof(NaSetup) <= 32000, "set-up parameter block must fit the kernel parameter limit");
static_assert(sizeof(mc::RDesc) % 4 == 0, "descriptor is copied as 4-byte words");

// Writes the descriptor, the CTA offset tables and the FFT tables, and clears every
// region the kernels expect at zero (the scratch keeps the previous call's contents).
__global__ void k_na_setup(const __grid_constant__ NaSetup p, unsigned char* __restrict__ base) {
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const int* dw = reinterpret_cast<const int*>(&p.d);
  int* desc = reinterpret_cast<int*>(base + kOffDesc);
  for (size_t i = t0; i < sizeof(mc::RDesc) / 4; i += stride) desc[i] = dw[i];
  if (t0 < 8) reinterpret_cast<int*>(base + kOffOff)[t0] = p.offs[t0];
  for (size_t i = t0; i < (size_t)p.d.W; i += stride) {
    reinterpret_cast<float2*>(base + kOffTwW)[i] = p.twW[i];
    reinterpret_cast<float*>(base + kOffGW)[i] = p.gW[i];
  }
  for (size_t i = t0; i < (size_t)p.d.H; i += stride) {
    reinterpret_cast<float2*>(base + kOffTwH)[i] = p.twH[i];
    reinterpret_cast<float*>(base + kOffGH)[i] = p.gH[i];
  }
  for (size_t i = t0; i < 2 * (size_t)p.N; i += stride) reinterpret_cast<float*>(base + kOffVel)[i] = 0.0f;
  for (size_t i = t0; i < (size_t)p.ntiles; i += stride) reinterpret_cast<int*>(base + kOffTcount)[i] = 0;
  if (t0 < 16) reinterpret_cast<int*>(base + kOffCtl)[t0] = 0;
  if (t0 < 4) reinterpret_cast<int*>(base + kOffWlCtl)[t0] = 0;
  for (size_t i = t0; i < p.HW; i += stride) reinterpret_cast<float*>(base + kOffDep)[i] = 0.0f;
}

bool na_factorize(int N, int* f, int* nf) {
  int n = 0;
  while (N % 4 == 0) { f[n++] = 4; N /= 4; }
  const int ps[] = {2, 3, 5, 7, 11, 13};
  for (int p : ps)
    while (N % p == 0 && n < mc::kFftMaxFactors) { f[n++] = p; N /= p; }
  *nf = n;
  return N == 1;
}

// roots of unity exp(-2 pi i k / N) and the spectral Gaussian exp(-2 pi^2 sigma^2 f_k^2) / N
// at numpy.fft.fftfreq abscissae, in float64 rounded to float32
void na_tables(int N, double sigma, float2* tw, float* g) {
  for (int k = 0; k < N; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)N;
    tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    const double fr = (k < (N + 1) / 2 ? (double)k : (double)(k - N)) / (double)N;
    g[k] = (float)(std::exp(-2.0 * M_PI * M_PI * sigma * sigma * fr * fr) / (double)N);
  }
}

}  // namespace

extern "C" mc_status mc_steric_potential_noalloc(const float* position, int32_t N, int32_t H, int32_t W, float sigma,
                                                 float scatter_value, float* steric_out, void* stream) {
  mc::set_last_error("");
  if (!position || !steric_out) return na_fail(MC_ERR_INVALID, "null position or output pointer");
  if (N < 1 || N > kNaMaxNodes)
    return na_fail(MC_ERR_INVALID, "N must be in [1, " + std::to_string(kNaMaxNodes) + "] for the no-allocation entry point");
  if (H < 4 || W < 4 || H > kNaMaxGrid || W > kNaMaxGrid)
    return na_fail(MC_ERR_INVALID, "H and W must be in [4, " + std::to_string(kNaMaxGrid) +
                                       "] for the no-allocation entry point");
  if (!(sigma > 0.0f)) return na_fail(MC_ERR_INVALID, "sigma must be > 0");
  // the set-up block (about 14 KB) lives on this call's stack: no host heap either
  NaSetup setup;
  std::memset(&setup, 0, sizeof(NaSetup));
  NaSetup* su = &setup;
  mc::RDesc& d = su->d;
  if (!na_factorize(W, d.fftW_f, &d.fftW_nf) || !na_factorize(H, d.fftH_f, &d.fftH_nf))
    return na_fail(MC_ERR_UNSUPPORTED, "H and W need prime factors <= 13");
  unsigned char* base = nullptr;
  mc_status st = na_setup(&base);
  if (st != MC_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  auto P = [&](size_t off) { return base + off; };

  d.H = H;
  d.W = W;
  d.N = N;
  d.K = 1;
  d.ntile_x = (W + mc::kBinTile - 1) / mc::kBinTile;
  d.ntile_y = (H + mc::kBinTile - 1) / mc::kBinTile;
  d.dt = 1.0f;
  d.damping = 1.0f;
  d.st_scatter = scatter_value;
  d.enable_steric = 1;
  d.enable_fluid = 0;
  d.twW = reinterpret_cast<const float2*>(P(kOffTwW));
  d.twH = reinterpret_cast<const float2*>(P(kOffTwH));
  d.gW = reinterpret_cast<const float*>(P(kOffGW));
  d.gH = reinterpret_cast<const float*>(P(kOffGH));
  d.pos = const_cast<float*>(position);  // read only by the deposit kernel
  d.vel = reinterpret_cast<float*>(P(kOffVel));
  d.steric = steric_out;
  d.prev = reinterpret_cast<float*>(P(kOffPrev));
  d.pred = reinterpret_cast<float*>(P(kOffPred));
  d.predw = reinterpret_cast<float*>(P(kOffPredw));
  d.dep = reinterpret_cast<float*>(P(kOffDep));
  d.tmp = reinterpret_cast<float*>(P(kOffTmp));
  d.c_cap = mc::kCicCap;
  d.c_cell = reinterpret_cast<int*>(P(kOffCell));
  d.c_w = reinterpret_cast<float*>(P(kOffW));
  d.c_store = reinterpret_cast<int*>(P(kOffStore));
  d.c_tcount = reinterpret_cast<int*>(P(kOffTcount));
  d.c_ovf = reinterpret_cast<int*>(P(kOffOvf));
  d.c_ctl = reinterpret_cast<int*>(P(kOffCtl));
  d.ib_ctl = reinterpret_cast<int*>(P(kOffCtl)) + 8;
  d.flags = reinterpret_cast<unsigned*>(P(kOffFlags));
  d.ridx = 0;
  d.wl_cic = reinterpret_cast<int2*>(P(kOffWl));
  d.wl_ib = reinterpret_cast<int2*>(P(kOffWl));  // unused (no IB here); k_predict resets its length
  d.wl_ctl = reinterpret_cast<int*>(P(kOffWlCtl));

  // CTA offset tables of the four kernels: deposit (nodes), bin tiles, FFT rows, FFT columns
  const int cnt[4] = {(N + mc::kNodeThreads - 1) / mc::kNodeThreads, d.ntile_x * d.ntile_y, (H + 1) / 2,
                      (W + 2 * mc::kFftColsPerCta - 1) / (2 * mc::kFftColsPerCta)};
  const int offs[8] = {0, cnt[0], 0, cnt[1], 0, cnt[2], 0, cnt[3]};
  std::memcpy(su->offs, offs, sizeof(offs));
  su->N = N;
  su->ntiles = d.ntile_x * d.ntile_y;
  su->HW = (size_t)H * W;
  na_tables(W, sigma, su->twW, su->gW);
  na_tables(H, sigma, su->twH, su->gH);
  k_na_setup<<<128, 256, 0, s>>>(setup, base);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(MC_ERR_CUDA, std::string("scratch set-up kernel: ") + cudaGetErrorString(e));
  const mc::RDesc* dd = reinterpret_cast<const mc::RDesc*>(P(kOffDesc));
  const int* off = reinterpret_cast<const int*>(P(kOffOff));
  mc::Launch l{dd, off, 1, cnt[0], s};
  mc::launch_predict(l);
  l.off = off + 2;
  l.grid = cnt[1] < 1184 ? cnt[1] : 1184;
  mc::launch_bin_tiles(l, reinterpret_cast<const int2*>(P(kOffWl)), reinterpret_cast<int*>(P(kOffWlCtl)) + 1, 1, 0,
                       mc::kCicCap);
  l.off = off + 4;
  l.grid = cnt[2];
  mc::launch_fft_rows(l, (size_t)3 * W * sizeof(float2) + W * sizeof(float));
  l.off = off + 6;
  l.grid = cnt[3];
  mc::launch_fft_cols(l, (size_t)(2 * mc::kFftColsPerCta + 1) * H * sizeof(float2) + H * sizeof(float));
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(MC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MC_OK;
}

static_assert(kNaMaxGrid == MC_NOALLOC_MAX_GRID && kNaMaxNodes == MC_NOALLOC_MAX_NODES,
              "limits must match the header");
static_assert((size_t)3 * kNaMaxGrid * sizeof(float2) + kNaMaxGrid * sizeof(float) <= 48 * 1024 &&
                  (size_t)(2 * mc::kFftColsPerCta + 1) * kNaMaxGrid * sizeof(float2) + kNaMaxGrid * sizeof(float) <=
                      48 * 1024,
              "the FFT kernels must fit the default dynamic shared memory limit");
