// Steric potential filter: V = real(ifft2(fft2(rho) * exp(-2 pi^2 sigma^2 (r^2 + c^2))))
// (src/microcosmos/utils.py:35-49, used by src/microcosmos/forces.py:84-118).
//
// The spectral Gaussian is separable, so the 2-D filter is a row pass then a column
// pass of 1-D circular convolutions, each done as a shared-memory mixed-radix Stockham
// FFT (radices 4, 2, 3, 5, 7, 11, 13) -> multiply by the real even 1-D spectrum ->
// inverse FFT.  Two real rows (columns) ride in one complex transform: with a real even
// spectrum the filtered rows come back as the real and imaginary parts.  Roots of unity
// and spectra are precomputed in float64 on the host and stored as float32.
#include "mc_internal.cuh"

namespace mc {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One Stockham stage of radix R over `nt` transforms of length N laid out [t][N].
// Output index of butterfly j: (j / Ns) * Ns * R + j % Ns + q * Ns.
// Radix 2 and 4 keep their operands in registers; the odd radices (non-power-of-two
// lengths only) use a generic R-point DFT.
template <int R>
__device__ __forceinline__ void stockham_pow2(const float2* __restrict__ in, float2* __restrict__ out, int N,
                                              int Ns, const float2* __restrict__ tw, int nt) {
  const int S = N / R;
  const int twstep = N / (Ns * R);
  for (int idx = threadIdx.x; idx < nt * S; idx += blockDim.x) {
    const int t = idx / S, j = idx - t * S;
    const float2* x = in + t * N;
    float2* y = out + t * N;
    const int k = j & (Ns - 1);
    const int dst = (j - k) * R + k;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 a = x[j + r * S];
      if (r > 0 && k > 0) a = cmul(a, tw[r * k * twstep]);
      v[r] = a;
    }
    if (R == 2) {
      y[dst] = make_float2(v[0].x + v[1].x, v[0].y + v[1].y);
      y[dst + Ns] = make_float2(v[0].x - v[1].x, v[0].y - v[1].y);
    } else {
      float2 a0 = make_float2(v[0].x + v[2 % R].x, v[0].y + v[2 % R].y);
      float2 a1 = make_float2(v[0].x - v[2 % R].x, v[0].y - v[2 % R].y);
      float2 b0 = make_float2(v[1].x + v[3 % R].x, v[1].y + v[3 % R].y);
      float2 b1 = make_float2(v[1].x - v[3 % R].x, v[1].y - v[3 % R].y);
      // b1 * (-i): the forward transform's quarter-turn
      float2 b1m = make_float2(b1.y, -b1.x);
      y[dst] = make_float2(a0.x + b0.x, a0.y + b0.y);
      y[dst + Ns] = make_float2(a1.x + b1m.x, a1.y + b1m.y);
      y[dst + 2 * Ns] = make_float2(a0.x - b0.x, a0.y - b0.y);
      y[dst + 3 * Ns] = make_float2(a1.x - b1m.x, a1.y - b1m.y);
    }
  }
}

__device__ __noinline__ void stockham_generic(const float2* __restrict__ in, float2* __restrict__ out, int N,
                                              int R, int Ns, const float2* __restrict__ tw, int nt) {
  const int S = N / R;
  const int twstep = N / (Ns * R);
  const int rstep = N / R;
  for (int idx = threadIdx.x; idx < nt * S; idx += blockDim.x) {
    const int t = idx / S, j = idx - t * S;
    const float2* x = in + t * N;
    float2* y = out + t * N;
    const int k = j % Ns;
    const int dst = (j / Ns) * Ns * R + k;
    float2 v[13];
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      float2 a = x[j + r * S];
      if (r > 0 && k > 0) a = cmul(a, tw[r * k * twstep]);
      v[r] = a;
    }
#pragma unroll 1
    for (int q = 0; q < R; ++q) {
      float2 acc = v[0];
#pragma unroll 1
      for (int r = 1; r < R; ++r) {
        float2 p = cmul(v[r], tw[((r * q) % R) * rstep]);
        acc.x = acc.x + p.x;
        acc.y = acc.y + p.y;
      }
      y[dst + q * Ns] = acc;
    }
  }
}

__device__ __forceinline__ void stockham_stage(const float2* in, float2* out, int N, int R, int Ns,
                                               const float2* tw, int nt) {
  if (R == 4)
    stockham_pow2<4>(in, out, N, Ns, tw, nt);
  else if (R == 2)
    stockham_pow2<2>(in, out, N, Ns, tw, nt);
  else
    stockham_generic(in, out, N, R, Ns, tw, nt);
}

// Forward FFT of nt transforms in `a` (scratch `b`); returns the buffer holding the result.
__device__ float2* fft_forward(float2* a, float2* b, int N, const int* fac, int nf, const float2* tw, int nt) {
  int Ns = 1;
  for (int s = 0; s < nf; ++s) {
    const int R = fac[s];
    stockham_stage(a, b, N, R, Ns, tw, nt);
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

// filter nt packed transforms: x -> IFFT(G * FFT(x)), G real even, 1/N folded into G.
// IFFT(y) = conj(FFT(conj(y))) / N.
__device__ float2* filter_packed(float2* a, float2* b, int N, const int* fac, int nf, const float2* tw,
                                 const float* g, int nt) {
  float2* r = fft_forward(a, b, N, fac, nf, tw, nt);
  float2* o = (r == a) ? b : a;
  for (int idx = threadIdx.x; idx < nt * N; idx += blockDim.x) {
    const float gk = g[idx % N];
    float2 v = r[idx];
    r[idx] = make_float2(v.x * gk, -(v.y * gk));  // conj(G * X)
  }
  __syncthreads();
  r = fft_forward(r, o, N, fac, nf, tw, nt);
  for (int idx = threadIdx.x; idx < nt * N; idx += blockDim.x) r[idx].y = -r[idx].y;
  __syncthreads();
  return r;
}

// Row pass: CTA q filters rows 2q and 2q+1 of the deposit grid into tmp.
__global__ void __launch_bounds__(256) k_fft_rows(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int q = blockIdx.x - off[r];
  const int W = d.W, H = d.H;
  const int y0 = 2 * q, y1 = 2 * q + 1;
  float2* a = sm;
  float2* b = sm + W;
  float2* tw = sm + 2 * W;
  float* g = reinterpret_cast<float*>(sm + 3 * W);
  const float* r0 = d.dep + (size_t)y0 * W;
  const float* r1 = (y1 < H) ? d.dep + (size_t)y1 * W : nullptr;
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    a[x] = make_float2(r0[x], r1 ? r1[x] : 0.0f);
    tw[x] = d.twW[x];
    g[x] = d.gW[x];
  }
  __syncthreads();
  float2* res = filter_packed(a, b, W, d.fftW_f, d.fftW_nf, tw, g, 1);
  float* o0 = d.tmp + (size_t)y0 * W;
  float* o1 = (y1 < H) ? d.tmp + (size_t)y1 * W : nullptr;
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    o0[x] = res[x].x;
    if (o1) o1[x] = res[x].y;
  }
}

// Column pass: CTA c filters real columns [2*C*c, 2*C*(c+1)) of tmp into the steric field.
__global__ void __launch_bounds__(256) k_fft_cols(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int cblk = blockIdx.x - off[r];
  const int W = d.W, H = d.H;
  const int C = kFftColsPerCta;
  const int xbase = cblk * 2 * C;
  float2* a = sm;
  float2* b = sm + C * H;
  float2* tw = sm + 2 * C * H;
  float* g = reinterpret_cast<float*>(sm + 2 * C * H + H);
  for (int y = threadIdx.x; y < H; y += blockDim.x) {
    tw[y] = d.twH[y];
    g[y] = d.gH[y];
  }
  for (int idx = threadIdx.x; idx < C * H; idx += blockDim.x) {
    const int y = idx / C, t = idx - y * C;  // consecutive threads read consecutive columns
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float* row = d.tmp + (size_t)y * W;
    a[t * H + y] = make_float2(xr < W ? row[xr] : 0.0f, xi < W ? row[xi] : 0.0f);
  }
  __syncthreads();
  float2* res = filter_packed(a, b, H, d.fftH_f, d.fftH_nf, tw, g, C);
  for (int idx = threadIdx.x; idx < C * H; idx += blockDim.x) {
    const int y = idx / C, t = idx - y * C;
    const int xr = xbase + 2 * t, xi = xr + 1;
    float* row = d.steric + (size_t)y * W;
    float2 v = res[t * H + y];
    if (xr < W) row[xr] = v.x;
    if (xi < W) row[xi] = v.y;
  }
}

void launch_fft_rows(const Launch& L, size_t smem) {
  k_fft_rows<<<L.grid, 256, smem, L.s>>>(L.d, L.off, L.n);
}
void launch_fft_cols(const Launch& L, size_t smem) {
  k_fft_cols<<<L.grid, 256, smem, L.s>>>(L.d, L.off, L.n);
}

cudaError_t fft_set_smem(size_t rows, size_t cols) {
  cudaError_t e = cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cols);
}

}  // namespace mc
