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

// ---------------------------------------------------------------- several transforms per CTA
// Radix-4 Stockham stages (and one radix-2 stage for odd log2 N) with shifts instead of
// divisions; several transforms share a CTA, T threads each, all in lockstep.  The roots of
// unity and the spectrum are read through the read-only data cache.
__device__ float2* fft_pow2(float2* x, float2* y, int logN, const float2* __restrict__ tw, int lt, int T) {
  const int N = 1 << logN;
  const int Q = N >> 2;
  int logNs = 0;
  while (logNs + 2 <= logN) {
    const int Ns = 1 << logNs;
    const int sh = logN - logNs - 2;  // twiddle step N / (4 Ns) as a shift
    for (int j = lt; j < Q; j += T) {
      const int k = j & (Ns - 1);
      float2 v0 = x[j], v1 = x[j + Q], v2 = x[j + 2 * Q], v3 = x[j + 3 * Q];
      if (k > 0) {
        v1 = cmul(v1, __ldg(tw + ((1 * k) << sh)));
        v2 = cmul(v2, __ldg(tw + ((2 * k) << sh)));
        v3 = cmul(v3, __ldg(tw + ((3 * k) << sh)));
      }
      const float2 a0 = make_float2(v0.x + v2.x, v0.y + v2.y);
      const float2 a1 = make_float2(v0.x - v2.x, v0.y - v2.y);
      const float2 b0 = make_float2(v1.x + v3.x, v1.y + v3.y);
      const float2 b1 = make_float2(v1.x - v3.x, v1.y - v3.y);
      const float2 b1m = make_float2(b1.y, -b1.x);  // b1 * (-i)
      const int dst = ((j - k) << 2) + k;
      y[dst] = make_float2(a0.x + b0.x, a0.y + b0.y);
      y[dst + Ns] = make_float2(a1.x + b1m.x, a1.y + b1m.y);
      y[dst + 2 * Ns] = make_float2(a0.x - b0.x, a0.y - b0.y);
      y[dst + 3 * Ns] = make_float2(a1.x - b1m.x, a1.y - b1m.y);
    }
    __syncthreads();
    float2* t = x;
    x = y;
    y = t;
    logNs += 2;
  }
  if (logNs < logN) {
    const int Ns = 1 << logNs;
    const int H2 = N >> 1;
    for (int j = lt; j < H2; j += T) {
      const int k = j & (Ns - 1);
      const float2 v0 = x[j];
      float2 v1 = x[j + H2];
      if (k > 0) v1 = cmul(v1, __ldg(tw + k));  // N / (2 Ns) = 1 on the last stage
      const int dst = ((j - k) << 1) + k;
      y[dst] = make_float2(v0.x + v1.x, v0.y + v1.y);
      y[dst + Ns] = make_float2(v0.x - v1.x, v0.y - v1.y);
    }
    __syncthreads();
    float2* t = x;
    x = y;
    y = t;
  }
  return x;
}

// One mixed-radix Stockham stage for one transform, T threads with local index lt.
template <int R>
__device__ __forceinline__ void stage_t(const float2* __restrict__ x, float2* __restrict__ y, int N, int Ns,
                                        const float2* __restrict__ tw, int lt, int T) {
  const int S = N / R;
  const int twstep = N / (Ns * R);
  const int rstep = N / R;
  for (int j = lt; j < S; j += T) {
    const int k = j % Ns;
    const int dst = (j - k) * R + k;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 a = x[j + r * S];
      if (r > 0 && k > 0) a = cmul(a, __ldg(tw + r * k * twstep));
      v[r] = a;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 p = cmul(v[r], __ldg(tw + ((r * q) % R) * rstep));
        acc.x = acc.x + p.x;
        acc.y = acc.y + p.y;
      }
      y[dst + q * Ns] = acc;
    }
  }
}

__device__ __noinline__ void stage_t_generic(const float2* __restrict__ x, float2* __restrict__ y, int N, int R,
                                             int Ns, const float2* __restrict__ tw, int lt, int T) {
  const int S = N / R;
  const int twstep = N / (Ns * R);
  const int rstep = N / R;
  for (int j = lt; j < S; j += T) {
    const int k = j % Ns;
    const int dst = (j - k) * R + k;
    float2 v[13];
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      float2 a = x[j + r * S];
      if (r > 0 && k > 0) a = cmul(a, __ldg(tw + r * k * twstep));
      v[r] = a;
    }
#pragma unroll 1
    for (int q = 0; q < R; ++q) {
      float2 acc = v[0];
#pragma unroll 1
      for (int r = 1; r < R; ++r) {
        const float2 p = cmul(v[r], __ldg(tw + ((r * q) % R) * rstep));
        acc.x = acc.x + p.x;
        acc.y = acc.y + p.y;
      }
      y[dst + q * Ns] = acc;
    }
  }
}

// Forward transform of one length-N sequence (prime factors <= 13): radix-4 stages with
// shifts when N is a power of two, else the factor list (4s, 2, 3, 5, 7, 11, 13), the
// stage sequence of fft_forward.
__device__ float2* fft_any(float2* x, float2* y, int N, int logN, const int* fac, int nf,
                           const float2* __restrict__ tw, int lt, int T) {
  if (logN >= 0) return fft_pow2(x, y, logN, tw, lt, T);
  int Ns = 1;
  for (int s = 0; s < nf; ++s) {
    const int R = fac[s];
    switch (R) {
      case 4: stage_t<4>(x, y, N, Ns, tw, lt, T); break;
      case 2: stage_t<2>(x, y, N, Ns, tw, lt, T); break;
      case 3: stage_t<3>(x, y, N, Ns, tw, lt, T); break;
      case 5: stage_t<5>(x, y, N, Ns, tw, lt, T); break;
      default: stage_t_generic(x, y, N, R, Ns, tw, lt, T); break;
    }
    __syncthreads();
    float2* t = x;
    x = y;
    y = t;
    Ns *= R;
  }
  return x;
}

// x -> IFFT(G * FFT(x)) for one packed transform (1/N folded into G), as filter_packed.
__device__ float2* filter_any(float2* a, float2* b, int N, int logN, const int* fac, int nf,
                              const float2* __restrict__ tw, const float* __restrict__ g, int lt, int T) {
  float2* r = fft_any(a, b, N, logN, fac, nf, tw, lt, T);
  float2* o = (r == a) ? b : a;
  for (int i = lt; i < N; i += T) {
    const float gk = __ldg(g + i);
    const float2 v = r[i];
    r[i] = make_float2(v.x * gk, -(v.y * gk));  // conj(G * X)
  }
  __syncthreads();
  r = fft_any(r, o, N, logN, fac, nf, tw, lt, T);
  for (int i = lt; i < N; i += T) r[i].y = -r[i].y;
  __syncthreads();
  return r;
}

// Row pass: each CTA filters fft_tpc_r row pairs, fft_T_r threads each.
__global__ void __launch_bounds__(256) k_fft_rows_p2(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H, T = d.fft_T_r, P = d.fft_tpc_r, logW = d.fft_logW;
  const int tr = threadIdx.x / T, lt = threadIdx.x - tr * T;  // P * T == blockDim.x
  const int q = (blockIdx.x - off[r]) * P + tr;
  const int y0 = 2 * q, y1 = 2 * q + 1;
  float2* a = sm + (size_t)tr * W;
  float2* b = sm + (size_t)(P + tr) * W;
  const bool act0 = y0 < H, act1 = y1 < H;
  const float* r0 = d.dep + (size_t)(act0 ? y0 : 0) * W;
  const float* r1 = d.dep + (size_t)(act1 ? y1 : 0) * W;
  for (int x = lt; x < W; x += T) a[x] = make_float2(act0 ? r0[x] : 0.0f, act1 ? r1[x] : 0.0f);
  __syncthreads();
  const float2* res = filter_any(a, b, W, logW, d.fftW_f, d.fftW_nf, d.twW, d.gW, lt, T);
  if (act0) {
    float* o0 = d.tmp + (size_t)y0 * W;
    for (int x = lt; x < W; x += T) o0[x] = res[x].x;
  }
  if (act1) {
    float* o1 = d.tmp + (size_t)y1 * W;
    for (int x = lt; x < W; x += T) o1[x] = res[x].y;
  }
}

// Column pass: each CTA filters fft_tpc_c column pairs (2 * fft_tpc_c
// real columns), fft_T_c threads each; columns are stored with stride H + 1 so that the
// transposing loads and stores hit distinct shared-memory banks.
__global__ void __launch_bounds__(512) k_fft_cols_p2(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H, T = d.fft_T_c, P = d.fft_tpc_c, logH = d.fft_logH;
  const int S = H + 1;
  const int xbase = (blockIdx.x - off[r]) * 2 * P;
  float2* a = sm;
  float2* b = sm + (size_t)P * S;
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;  // consecutive threads read consecutive columns of a row
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float* row = d.tmp + (size_t)y * W;
    a[t * S + y] = make_float2(xr < W ? row[xr] : 0.0f, xi < W ? row[xi] : 0.0f);
  }
  __syncthreads();
  const int tr = threadIdx.x / T, lt = threadIdx.x - tr * T;  // P * T == blockDim.x
  const float2* res = filter_any(a + (size_t)tr * S, b + (size_t)tr * S, H, logH, d.fftH_f, d.fftH_nf, d.twH, d.gH,
                                 lt, T);
  // every transform of the CTA ends in the same buffer (same number of stages)
  const float2* base = (res == a + (size_t)tr * S) ? a : b;
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;
    const int xr = xbase + 2 * t, xi = xr + 1;
    float* row = d.steric + (size_t)y * W;
    const float2 v = base[t * S + y];
    if (xr < W) row[xr] = v.x;
    if (xi < W) row[xi] = v.y;
  }
}

void launch_fft_rows_p2(const Launch& L, size_t smem) {
  k_fft_rows_p2<<<L.grid, 256, smem, L.s>>>(L.d, L.off, L.n);
}
void launch_fft_cols_p2(const Launch& L, size_t smem) {
  k_fft_cols_p2<<<L.grid, 512, smem, L.s>>>(L.d, L.off, L.n);
}
cudaError_t fft_p2_set_smem(size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_fft_rows_p2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes a;
  e = cudaFuncGetAttributes(&a, k_fft_cols_p2);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_fft_cols_p2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(bytes - a.sharedSizeBytes));
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


// The spectral Gaussian of update_steric_potential (src/microcosmos/utils.py:35-49) as a
// direct circular convolution: real(ifft2(fft2(dep) * exp(-2 pi^2 sigma^2 (r^2 + c^2))))
// is separable, and along each axis equals the circular convolution of dep with the
// filter's periodic kernel g[k] = (1/N) sum_j exp(-2 pi^2 sigma^2 f_j^2) cos(2 pi j k / N)
// (computed in double on the host).  Taps beyond radius R are below 1e-10 of g[0] and are
// dropped.  One CTA: a 32 x 32 output tile, its input tile with an R halo staged in
// shared memory (wrapped), the x pass into a second shared buffer, then the y pass.
__global__ void __launch_bounds__(256) k_steric_conv(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int lb = blockIdx.x - off[r];
  const int tx = lb % d.conv_ntx, ty = lb / d.conv_ntx;
  const int H = d.H, W = d.W, Rx = d.conv_RW, Ry = d.conv_RH;
  const int iw = kConvTile + 2 * Rx, ih = kConvTile + 2 * Ry;
  extern __shared__ float conv_sm[];
  float* in = conv_sm;             // ih x iw
  float* mid = conv_sm + ih * iw;  // ih x kConvTile
  const int x0 = tx * kConvTile - Rx, y0 = ty * kConvTile - Ry;
  const int nt = blockDim.x;
  for (int i = threadIdx.x; i < ih * iw; i += nt) {
    const int yy = i / iw, xx = i - yy * iw;
    in[i] = d.dep[(size_t)imod_floor(y0 + yy, H) * W + imod_floor(x0 + xx, W)];
  }
  __syncthreads();
  const float* gx = d.conv_gW;
  for (int i = threadIdx.x; i < ih * kConvTile; i += nt) {
    const int yy = i / kConvTile, xx = i - yy * kConvTile;
    const float* row = in + yy * iw + xx;
    float a = 0.0f;
    for (int k = 0; k <= 2 * Rx; ++k) a = a + gx[k] * row[2 * Rx - k];
    mid[i] = a;
  }
  __syncthreads();
  const float* gy = d.conv_gH;
  for (int i = threadIdx.x; i < kConvTile * kConvTile; i += nt) {
    const int yy = i / kConvTile, xx = i - yy * kConvTile;
    const int oy = ty * kConvTile + yy, ox = tx * kConvTile + xx;
    if (oy >= H || ox >= W) continue;
    const float* col = mid + yy * kConvTile + xx;
    float a = 0.0f;
    for (int k = 0; k <= 2 * Ry; ++k) a = a + gy[k] * col[(2 * Ry - k) * kConvTile];
    d.steric[(size_t)oy * W + ox] = a;
  }
}

void launch_steric_conv(const Launch& L, size_t smem) {
  k_steric_conv<<<L.grid, 256, smem, L.s>>>(L.d, L.off, L.n);
}


// ---------------------------------------------------------------- register-radix path
// Power-of-two lengths: G = N / E threads per transform, each holding E = 4, 8 or 16
// complex values in registers.  A Stockham pass of radix R (E, or a smaller power of two
// for the last pass) loads R-strided operands from shared memory, twiddles them, runs an
// R-point DFT in registers and stores the autosorted result back in place: a length-1024
// transform takes three shared-memory passes with E = 16 (16, 16, 4), five with E = 4.
// Fewer values per thread give more threads for small problems; more give fewer
// instructions per value for large batches.  Shared-memory addresses are padded by one
// element every 16 (a -> a + a / 16) so the strided stores of the first pass spread over
// the banks.  Twiddles are the float64-derived roots, read from a table laid out per pass
// (the host's pass_twiddles) so that a butterfly's R - 1 factors sit at one base address.

__device__ __forceinline__ int pad16(int a) { return a + (a >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

// cos(2 pi k / 16), sin(2 pi k / 16) for k = 0..3 (the forward root is cos - i sin)
constexpr float kC16[4] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f};
constexpr float kS16[4] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f};

// a * exp(-2 pi i e / 16) for a compile-time exponent e in 0..15
template <int E>
__device__ __forceinline__ float2 rot16(float2 a) {
  constexpr int e = E & 15;
  if (e == 0) return a;
  if (e == 4) return mul_mi(a);
  if (e == 8) return make_float2(-a.x, -a.y);
  if (e == 12) return make_float2(-a.y, a.x);
  constexpr int q = e & 3, h = e >> 2;  // angle = h * 90 + q * 22.5 degrees
  const float c = kC16[q], sn = kS16[q];
  float2 r = make_float2(a.x * c + a.y * sn, a.y * c - a.x * sn);  // a * (c - i s)
  if (h == 1) return mul_mi(r);
  if (h == 2) return make_float2(-r.x, -r.y);
  if (h == 3) return make_float2(-r.y, r.x);
  return r;
}

__device__ __forceinline__ void dft2(float2& a, float2& b) {
  const float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d) {
  const float2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_mi(csub(b, d));
  a = cadd(t0, t2);
  c = csub(t0, t2);
  b = cadd(t1, t3);
  d = csub(t1, t3);
}

// R-point forward DFT of v[0..R-1] in registers; X[k] ends in v[perm(k)]:
// R = 2, 4: natural order; R = 8: X[k2 + 4 k1] in v[2 k2 + k1]; R = 16: X[k2 + 4 k1] in v[4 k2 + k1].
template <int R>
__device__ __forceinline__ void dft_reg(float2* v) {
  if constexpr (R == 2) {
    dft2(v[0], v[1]);
  } else if constexpr (R == 3) {
    // X1,2 = a - (b + c) / 2 -/+ i (sqrt(3) / 2) (b - c)
    const float2 a = v[0], t1 = cadd(v[1], v[2]), dd = csub(v[1], v[2]);
    const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
    const float s3 = 0.86602540378443865f;
    const float2 t3 = make_float2(s3 * dd.y, -(s3 * dd.x));
    v[0] = cadd(a, t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // n = n1 + 2 n2: length-4 DFTs over n2, twiddle W8^(n1 k2), length-2 DFTs over n1
    dft4(v[0], v[2], v[4], v[6]);
    dft4(v[1], v[3], v[5], v[7]);
    v[3] = rot16<2>(v[3]);
    v[5] = rot16<4>(v[5]);
    v[7] = rot16<6>(v[7]);
    dft2(v[0], v[1]);
    dft2(v[2], v[3]);
    dft2(v[4], v[5]);
    dft2(v[6], v[7]);
  } else {
    // n = n1 + 4 n2: length-4 DFTs over n2, twiddle W16^(n1 k2), length-4 DFTs over n1
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    v[5] = rot16<1>(v[5]);
    v[9] = rot16<2>(v[9]);
    v[13] = rot16<3>(v[13]);
    v[6] = rot16<2>(v[6]);
    v[10] = rot16<4>(v[10]);
    v[14] = rot16<6>(v[14]);
    v[7] = rot16<3>(v[7]);
    v[11] = rot16<6>(v[11]);
    v[15] = rot16<9>(v[15]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
  }
}

template <int R>
__device__ __forceinline__ constexpr int dft_slot(int k) {
  if (R == 8) return 2 * (k & 3) + (k >> 2);
  if (R == 16) return 4 * (k & 3) + (k >> 2);
  return k;
}

// One in-place Stockham pass of radix R over a padded buffer of N = 2^logN values,
// G = N / E threads (local index lt) holding E values each, Ns = 2^logNs.
// `pt`: this length's per-pass twiddle table (pass_twiddles on the host): the R - 1 factors of
// butterfly k of the pass with Ns = 2^logNs start at pt[(Ns - 1) + k (R - 1)].
template <int E, int R>
__device__ __forceinline__ void pass_reg(float2* buf, int logN, int logNs, int lt, const float2* __restrict__ pt) {
  constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
  constexpr int LE = E == 4 ? 2 : E == 8 ? 3 : 4;
  constexpr int C = E / R;  // butterflies per thread
  const int G = 1 << (logN - LE);
  const int S = 1 << (logN - LR);  // butterflies in the pass
  const int Ns = 1 << logNs;
  float2 v[E];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = lt + c * G;
    const int k = j & (Ns - 1);
    const float2* __restrict__ tk = pt + (Ns - 1) + k * (R - 1) - 1;  // tk[m], m = 1..R-1
#pragma unroll
    for (int m = 0; m < R; ++m) {
      float2 a = buf[pad16(j + m * S)];
      if (m > 0 && k > 0) a = cmul(a, __ldg(tk + m));
      v[c * R + m] = a;
    }
    dft_reg<R>(v + c * R);
  }
  (void)S;
  __syncthreads();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = lt + c * G;
    const int k = j & (Ns - 1);
    const int dst = ((j - k) << LR) + k;
#pragma unroll
    for (int m = 0; m < R; ++m) buf[pad16(dst + m * Ns)] = v[c * R + dft_slot<R>(m)];
  }
  __syncthreads();
}

// Forward transform in place (natural order in and out), N = 2^logN >= E.
template <int E>
__device__ __forceinline__ void fft_reg(float2* buf, int logN, int lt, const float2* __restrict__ pt) {
  constexpr int LE = E == 4 ? 2 : E == 8 ? 3 : 4;
  int logNs = 0;
  while (logNs + LE <= logN) {
    pass_reg<E, E>(buf, logN, logNs, lt, pt);
    logNs += LE;
  }
  const int rem = logN - logNs;
  if (rem == 1) pass_reg<E, 2>(buf, logN, logNs, lt, pt);
  if constexpr (E >= 8) {
    if (rem == 2) pass_reg<E, 4>(buf, logN, logNs, lt, pt);
  }
  if constexpr (E >= 16) {
    if (rem == 3) pass_reg<E, 8>(buf, logN, logNs, lt, pt);
  }
}

// x -> IFFT(G * FFT(x)) with 1/N folded into g: conj(FFT(conj(G * FFT(x)))).
template <int E>
__device__ __forceinline__ void filter_reg(float2* buf, int logN, int lt, const float2* __restrict__ pt,
                                           const float* __restrict__ g) {
  const int N = 1 << logN, G = N / E;
  fft_reg<E>(buf, logN, lt, pt);
  for (int i = lt; i < N; i += G) {
    const float gk = __ldg(g + i);
    const float2 v = buf[pad16(i)];
    buf[pad16(i)] = make_float2(v.x * gk, -(v.y * gk));
  }
  __syncthreads();
  fft_reg<E>(buf, logN, lt, pt);
}

// Row pass: 256 / G row pairs per CTA (one packed transform each), G = W / E.
template <int E>
__global__ void __launch_bounds__(256) k_fftreg_rows(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 smr[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H, logN = d.fft_logW;
  const int G = W / E, P = 256 / G;
  const int tr = threadIdx.x / G, lt = threadIdx.x - tr * G;
  const int q = (blockIdx.x - off[r]) * P + tr;
  const int y0 = 2 * q, y1 = 2 * q + 1;
  float2* buf = smr + (size_t)tr * (W + (W >> 4));
  const bool act0 = y0 < H, act1 = y1 < H;
  const float* r0 = d.dep + (size_t)(act0 ? y0 : 0) * W;
  const float* r1 = d.dep + (size_t)(act1 ? y1 : 0) * W;
  for (int x = lt; x < W; x += G) buf[pad16(x)] = make_float2(act0 ? r0[x] : 0.0f, act1 ? r1[x] : 0.0f);
  __syncthreads();
  filter_reg<E>(buf, logN, lt, d.ptW, d.gW);
  if (act0) {
    float* o = d.tmp + (size_t)y0 * W;
    for (int x = lt; x < W; x += G) o[x] = buf[pad16(x)].x;
  }
  if (act1) {
    float* o = d.tmp + (size_t)y1 * W;
    for (int x = lt; x < W; x += G) o[x] = -buf[pad16(x)].y;
  }
}

// Column pass: TV / H column pairs per CTA of TV / E threads (G = H / E per pair), TV = 4096
// values per CTA, or 2048 when a plan has too few columns to give every SM two CTAs (a single
// 1024^2 lattice: 256 CTAs instead of 128); staged from the row-pass output: at H = 1024 a
// CTA reads 32-byte (TV = 4096) or 16-byte row segments.  Every column pair is transformed
// by the same code whatever TV is, so both give the same bits.
template <int E, int TV>
__global__ void __launch_bounds__(TV / E) k_fftreg_cols(const RDesc* __restrict__ D, const int* __restrict__ off,
                                                        int n) {
  extern __shared__ float2 smr[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H, logN = d.fft_logH;
  const int G = H / E, P = blockDim.x / G;
  // one extra slot per column pair staggers the pairs over the shared-memory banks when the
  // tile is staged row by row
  const int S = H + (H >> 4) + 1;
  const int xbase = (blockIdx.x - off[r]) * 2 * P;
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float* row = d.tmp + (size_t)y * W;
    smr[(size_t)t * S + pad16(y)] = make_float2(xr < W ? row[xr] : 0.0f, xi < W ? row[xi] : 0.0f);
  }
  __syncthreads();
  const int tr = threadIdx.x / G, lt = threadIdx.x - tr * G;
  filter_reg<E>(smr + (size_t)tr * S, logN, lt, d.ptH, d.gH);
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float2 v = smr[(size_t)t * S + pad16(y)];
    float* row = d.steric + (size_t)y * W;
    if (xr < W) row[xr] = v.x;
    if (xi < W) row[xi] = -v.y;
  }
}

// ---------------------------------------------------------------- sides N = 3 * 2^a
// Twelve values per thread (G = N / 12 threads per transform): the power-of-two factor
// in radix-4 passes (three butterflies per thread; one radix-2 pass if a is odd), then a
// final radix-3 pass (four butterflies per thread) with Ns = N / 3, so every k = j mod Ns
// is still a mask.  Twiddle index steps N / (Ns R) are integers but not powers of two.
template <int R>
__device__ __forceinline__ void pass12(float2* buf, int N, int Ns, int lt, const float2* __restrict__ tw) {
  constexpr int C = 12 / R;
  const int G = N / 12;
  const int S = N / R;
  const int step = N / (Ns * R);
  float2 v[12];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = lt + c * G;
    const int k = j & (Ns - 1);
#pragma unroll
    for (int m = 0; m < R; ++m) {
      float2 a = buf[pad16(j + m * S)];
      if (m > 0 && k > 0) a = cmul(a, __ldg(tw + m * k * step));
      v[c * R + m] = a;
    }
    dft_reg<R>(v + c * R);
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int j = lt + c * G;
    const int k = j & (Ns - 1);
    const int dst = (j - k) * R + k;
#pragma unroll
    for (int m = 0; m < R; ++m) buf[pad16(dst + m * Ns)] = v[c * R + dft_slot<R>(m)];
  }
  __syncthreads();
}

__device__ __forceinline__ void fft12(float2* buf, int N, int lt, const float2* __restrict__ tw) {
  const int P = N / 3;  // power of two >= 4
  int Ns = 1;
  while (Ns * 4 <= P) {
    pass12<4>(buf, N, Ns, lt, tw);
    Ns *= 4;
  }
  if (Ns < P) {
    pass12<2>(buf, N, Ns, lt, tw);
    Ns *= 2;
  }
  pass12<3>(buf, N, Ns, lt, tw);
}

__device__ __forceinline__ void filter12(float2* buf, int N, int lt, const float2* __restrict__ tw,
                                         const float* __restrict__ g) {
  const int G = N / 12;
  fft12(buf, N, lt, tw);
  for (int i = lt; i < N; i += G) {
    const float gk = __ldg(g + i);
    const float2 v = buf[pad16(i)];
    buf[pad16(i)] = make_float2(v.x * gk, -(v.y * gk));
  }
  __syncthreads();
  fft12(buf, N, lt, tw);
}

// Row pass for W = 3 * 2^a: 256 / G row pairs per CTA, G = W / 12.
__global__ void __launch_bounds__(256) k_fft12_rows(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm12[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H;
  const int G = W / 12, P = 256 / G;
  const int tr = threadIdx.x / G, lt = threadIdx.x - tr * G;
  const int q = (blockIdx.x - off[r]) * P + tr;
  const int y0 = 2 * q, y1 = 2 * q + 1;
  float2* buf = sm12 + (size_t)tr * (W + (W >> 4));
  const bool act0 = y0 < H, act1 = y1 < H;
  const float* r0 = d.dep + (size_t)(act0 ? y0 : 0) * W;
  const float* r1 = d.dep + (size_t)(act1 ? y1 : 0) * W;
  for (int x = lt; x < W; x += G) buf[pad16(x)] = make_float2(act0 ? r0[x] : 0.0f, act1 ? r1[x] : 0.0f);
  __syncthreads();
  filter12(buf, W, lt, d.twW, d.gW);
  if (act0) {
    float* o = d.tmp + (size_t)y0 * W;
    for (int x = lt; x < W; x += G) o[x] = buf[pad16(x)].x;
  }
  if (act1) {
    float* o = d.tmp + (size_t)y1 * W;
    for (int x = lt; x < W; x += G) o[x] = -buf[pad16(x)].y;
  }
}

// Column pass for H = 3 * 2^a: 384 / G column pairs per CTA of 384 threads, G = H / 12.
__global__ void __launch_bounds__(384) k_fft12_cols(const RDesc* __restrict__ D, const int* __restrict__ off, int n) {
  extern __shared__ float2 sm12[];
  const int r = find_rollout(off, n, blockIdx.x);
  const RDesc& d = D[r];
  const int W = d.W, H = d.H;
  const int G = H / 12, P = blockDim.x / G;
  const int S = H + (H >> 4) + 1;  // staggered over the banks, as in k_fftreg_cols
  const int xbase = (blockIdx.x - off[r]) * 2 * P;
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float* row = d.tmp + (size_t)y * W;
    sm12[(size_t)t * S + pad16(y)] = make_float2(xr < W ? row[xr] : 0.0f, xi < W ? row[xi] : 0.0f);
  }
  __syncthreads();
  const int tr = threadIdx.x / G, lt = threadIdx.x - tr * G;
  filter12(sm12 + (size_t)tr * S, H, lt, d.twH, d.gH);
  for (int idx = threadIdx.x; idx < P * H; idx += blockDim.x) {
    const int y = idx / P, t = idx - y * P;
    const int xr = xbase + 2 * t, xi = xr + 1;
    const float2 v = sm12[(size_t)t * S + pad16(y)];
    float* row = d.steric + (size_t)y * W;
    if (xr < W) row[xr] = v.x;
    if (xi < W) row[xi] = -v.y;
  }
}

// 256 * 12 / N (rows) or 384 * 12 / N (columns) transforms of N + N / 16 values
constexpr size_t kFft12RowsSmem = (size_t)256 * 12 * 17 / 16 * sizeof(float2) + 256;
constexpr size_t kFft12ColsSmem = ((size_t)384 * 12 * 17 / 16 + 384) * sizeof(float2) + 256;
void launch_fft12_rows(const Launch& L) { k_fft12_rows<<<L.grid, 256, kFft12RowsSmem, L.s>>>(L.d, L.off, L.n); }
void launch_fft12_cols(const Launch& L) { k_fft12_cols<<<L.grid, 384, kFft12ColsSmem, L.s>>>(L.d, L.off, L.n); }

// shared memory of a CTA: (row pass, 256 threads) 256 E / N transforms or (column pass,
// TV / E threads) TV / N transforms, of N + N / 16 values each (+1 per column pair)
size_t fftreg_smem(int e) { return (size_t)256 * e * 17 / 16 * sizeof(float2); }
size_t fftreg_cols_smem(int tv) { return ((size_t)tv * 17 / 16 + 256) * sizeof(float2); }

void launch_fftreg_rows(const Launch& L, int e) {
  if (e == 16) k_fftreg_rows<16><<<L.grid, 256, fftreg_smem(16), L.s>>>(L.d, L.off, L.n);
  else if (e == 8) k_fftreg_rows<8><<<L.grid, 256, fftreg_smem(8), L.s>>>(L.d, L.off, L.n);
  else k_fftreg_rows<4><<<L.grid, 256, fftreg_smem(4), L.s>>>(L.d, L.off, L.n);
}
void launch_fftreg_cols(const Launch& L, int e, int tv) {
  const size_t sm = fftreg_cols_smem(tv);
  if (tv == 2048) {
    if (e == 16) k_fftreg_cols<16, 2048><<<L.grid, 128, sm, L.s>>>(L.d, L.off, L.n);
    else if (e == 8) k_fftreg_cols<8, 2048><<<L.grid, 256, sm, L.s>>>(L.d, L.off, L.n);
    else k_fftreg_cols<4, 2048><<<L.grid, 512, sm, L.s>>>(L.d, L.off, L.n);
    return;
  }
  if (e == 16) k_fftreg_cols<16, 4096><<<L.grid, 256, sm, L.s>>>(L.d, L.off, L.n);
  else if (e == 8) k_fftreg_cols<8, 4096><<<L.grid, 512, sm, L.s>>>(L.d, L.off, L.n);
  else k_fftreg_cols<4, 4096><<<L.grid, 1024, sm, L.s>>>(L.d, L.off, L.n);
}


}  // namespace mc
