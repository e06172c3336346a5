// Frame rasteriser of a recorded rollout (src/microcosmos/rendering.py:20-80) into a
// headless device buffer: per frame, the steric field as the grey texture
// 1 - clip(V, 0, 1), every node's pixel floor(position) (clipped to the grid) in its
// colour, every node's debug pixel floor(position + debug_vector) in red, then float ->
// uint8 as clip(v * 255, 0, 255) truncated, and a nearest-neighbour resize to
// (size * H / max(H, W), size * W / max(H, W)).
//
// The reference writes the pixels with two scatter-sets, nodes in order then debug
// pixels in order, so at a pixel hit several times the last write is kept.  Here each
// write carries its rank in that order (node i: 1 + i, debug pixel i: 1 + N + i) and
// the largest rank per pixel is kept with an integer atomicMax into a caller-provided
// (T, H, W) int32 buffer; the shading pass then reads one winner per pixel.
#include "mc_internal.cuh"

#include "../../include/microcosmos_b200.h"

namespace mc {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__global__ void __launch_bounds__(256) k_render_scatter(const float* __restrict__ pos, const float* __restrict__ dbg,
                                                        int T, int N, int H, int W, int* __restrict__ winner) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_frame = 2LL * N;
  if (i >= (long long)T * per_frame) return;
  const int t = (int)(i / per_frame);
  const int j = (int)(i - (long long)t * per_frame);
  const bool is_dbg = j >= N;
  const int node = is_dbg ? j - N : j;
  const size_t k = ((size_t)t * N + node) * 2;
  float x = pos[k], y = pos[k + 1];
  if (is_dbg) {
    x = x + (dbg ? dbg[k] : 0.0f);
    y = y + (dbg ? dbg[k + 1] : 0.0f);
  }
  // floor(...).astype(int), then clip to the grid (rendering.py:34-37, 59-62)
  const int px = clampi((int)floorf(x), 0, W - 1);
  const int py = clampi((int)floorf(y), 0, H - 1);
  atomicMax(winner + ((size_t)t * H + py) * W + px, 1 + j);
}

// nearest-neighbour source index of output index o along an axis of m -> n samples:
// floor((o + 0.5) * m / n) in float32, clipped (the identity when m == n)
__device__ __forceinline__ int nearest_src(int o, int m, int n) {
  if (m == n) return o;
  const float f = ((float)o + 0.5f) * (float)m / (float)n;
  return clampi((int)floorf(f), 0, m - 1);
}

__device__ __forceinline__ unsigned char to_u8(float v) {
  v = v * 255.0f;
  v = v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v);
  return (unsigned char)v;  // truncation toward zero, as float -> uint8
}

__global__ void __launch_bounds__(256) k_render_shade(const float* __restrict__ steric, const int* __restrict__ winner,
                                                      const float* __restrict__ color_bend, int T, int N, int H, int W,
                                                      int out_h, int out_w, int uniform_color,
                                                      unsigned char* __restrict__ frames) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_frame = (long long)out_h * out_w;
  if (i >= (long long)T * per_frame) return;
  const int t = (int)(i / per_frame);
  const int r = (int)(i - (long long)t * per_frame);
  const int oy = r / out_w, ox = r - oy * out_w;
  const int sy = nearest_src(oy, H, out_h), sx = nearest_src(ox, W, out_w);
  const size_t src = ((size_t)t * H + sy) * W + sx;
  const int w = winner ? winner[src] : 0;
  float c0, c1, c2;
  if (w == 0) {
    float v = steric[src];
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    c0 = c1 = c2 = 1.0f - v;
  } else if (w <= N) {
    // BASE_COLOR + COLOR_VARIATION * color_bend (rendering.py:16-17, 48-51)
    const float col = (uniform_color || !color_bend) ? 0.0f : color_bend[w - 1];
    if (uniform_color) {
      c0 = 0.3f;
      c1 = 0.6f;
      c2 = 0.9f;
    } else {
      c0 = 0.3f + 0.3f * col;
      c1 = 0.6f + 0.2f * col;
      c2 = 0.9f + 0.0f * col;
    }
  } else {
    c0 = 1.0f;
    c1 = 0.0f;
    c2 = 0.0f;
  }
  unsigned char* o = frames + (size_t)i * 3;
  o[0] = to_u8(c0);
  o[1] = to_u8(c1);
  o[2] = to_u8(c2);
}

}  // namespace mc

extern "C" {

size_t mc_render_scratch_bytes(int32_t T, int32_t H, int32_t W) {
  return (T > 0 && H > 0 && W > 0) ? (size_t)T * H * W * sizeof(int) : 0;
}

mc_status mc_render_frames(const float* position, const float* debug_vector, const float* color_bend,
                           const float* steric, int32_t T, int32_t N, int32_t H, int32_t W, int32_t size,
                           int32_t render_particles, int32_t uniform_color, int32_t* scratch, uint8_t* frames,
                           void* stream) {
  if (T <= 0 || N < 0 || H <= 0 || W <= 0 || size <= 0) {
    mc::set_last_error("mc_render_frames: bad sizes");
    return MC_ERR_INVALID;
  }
  if (!steric || !frames || (render_particles && N > 0 && (!position || !scratch))) {
    mc::set_last_error("mc_render_frames: null pointer");
    return MC_ERR_INVALID;
  }
  const int mx = H > W ? H : W;
  const long long oh = (long long)size * H / mx, ow = (long long)size * W / mx;
  if (oh <= 0 || ow <= 0) {
    mc::set_last_error("mc_render_frames: size gives an empty frame");
    return MC_ERR_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool particles = render_particles && N > 0;
  if (particles) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, (size_t)T * H * W * sizeof(int), s);
    if (e != cudaSuccess) {
      mc::set_last_error(cudaGetErrorString(e));
      return MC_ERR_CUDA;
    }
    const long long n = (long long)T * 2 * N;
    mc::k_render_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(position, debug_vector, T, N, H, W, scratch);
  }
  const long long m = (long long)T * oh * ow;
  mc::k_render_shade<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(steric, particles ? scratch : nullptr, color_bend,
                                                                 T, N, H, W, (int)oh, (int)ow, uniform_color,
                                                                 reinterpret_cast<unsigned char*>(frames));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    mc::set_last_error(cudaGetErrorString(e));
    return MC_ERR_CUDA;
  }
  return MC_OK;
}

}  // extern "C"
