// The gym environment's device work around one rollout step
// (src/microcosmos/gym/base.py:173-196), for a table of environments per launch:
//   k_env_act:     rest lengths / rest angles = base + action (base.py:177-182);
//   k_env_observe: the energy source's periodic walk (base.py:187-190), the observation
//                  [positions - their mean, velocities, energy at the nodes]
//                  (base.py:112-121), the reward = sum of the node energies, per node
//                  range ("creature") when the environment has several
//                  (multi_agent.py:201-212), the step counter and the done flag.
// One CTA per environment; sums are taken in a fixed order (per-thread strided
// sequential sums, then a fixed shuffle/shared-memory tree), so results are
// reproducible from run to run.
#include "mc_internal.cuh"

#include "../../include/microcosmos_b200.h"

namespace mc {

constexpr int kEnvThreads = 256;

__global__ void __launch_bounds__(kEnvThreads) k_env_act(const mc_env* __restrict__ envs) {
  const mc_env& e = envs[blockIdx.x];
  for (int i = threadIdx.x; i < e.E; i += blockDim.x)
    e.rest_lengths[i] = e.d_rest_length ? e.base_rest_lengths[i] + e.d_rest_length[i] : e.base_rest_lengths[i] + 0.0f;
  for (int i = threadIdx.x; i < e.B; i += blockDim.x)
    e.bending_rest_angles[i] =
        e.d_bending_angle ? e.base_bending_rest_angles[i] + e.d_bending_angle[i] : e.base_bending_rest_angles[i] + 0.0f;
}

// Sum of one value per thread over the CTA in a fixed order; every thread gets the result.
__device__ float block_sum(float v, float* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();  // scratch may still be read by a previous call
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  float t = 0.0f;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = t + scratch[w];
  return t;
}

__global__ void __launch_bounds__(kEnvThreads) k_env_observe(const mc_env* __restrict__ envs, int advance) {
  __shared__ float scratch[kEnvThreads / 32];
  __shared__ float s_center[2];
  const mc_env& e = envs[blockIdx.x];
  const float W = (float)e.W, H = (float)e.H;
  if (threadIdx.x == 0 && !advance) {
    s_center[0] = e.energy_center[0];
    s_center[1] = e.energy_center[1];
  }
  if (threadIdx.x == 0 && advance) {
    // (center + normal * std) % (w, h), floored (base.py:187-190)
    float cx = e.energy_center[0], cy = e.energy_center[1];
    const float nx = e.noise ? e.noise[0] * e.energy_walk_std : 0.0f;
    const float ny = e.noise ? e.noise[1] * e.energy_walk_std : 0.0f;
    cx = fmod_floor(cx + nx, W);
    cy = fmod_floor(cy + ny, H);
    e.energy_center[0] = cx;
    e.energy_center[1] = cy;
    s_center[0] = cx;
    s_center[1] = cy;
    const int t = *e.time + 1;
    *e.time = t;
    *e.done = t >= e.max_steps ? 1 : 0;
  }
  // centre of mass (base.py:114-115)
  float sx = 0.0f, sy = 0.0f;
  for (int i = threadIdx.x; i < e.N; i += blockDim.x) {
    sx = sx + e.position[2 * i];
    sy = sy + e.position[2 * i + 1];
  }
  sx = block_sum(sx, scratch);
  sy = block_sum(sy, scratch);
  const float mx = sx / (float)e.N, my = sy / (float)e.N;
  const float cx = s_center[0], cy = s_center[1];
  float* obs = e.observation;
  const int N = e.N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const float x = e.position[2 * i], y = e.position[2 * i + 1];
    obs[2 * i] = x - mx;
    obs[2 * i + 1] = y - my;
    obs[2 * N + 2 * i] = e.velocity[2 * i];
    obs[2 * N + 2 * i + 1] = e.velocity[2 * i + 1];
    // periodic Gaussian at the min-image distance (base.py:89-94)
    const float2 d = min_image(x, y, cx, cy, W, H);
    const float d2 = d.x * d.x + d.y * d.y;
    obs[4 * N + i] = e.energy_amplitude * expf(-d2 / e.energy_two_size_sq);
  }
  __syncthreads();
  // per node range: sum of its energies; reward = sum over the ranges (multi_agent.py:201-212)
  const int nseg = e.num_segments > 0 ? e.num_segments : 1;
  float reward = 0.0f;
  for (int g = 0; g < nseg; ++g) {
    const int a = e.segment_offsets ? e.segment_offsets[g] : 0;
    const int b = e.segment_offsets ? e.segment_offsets[g + 1] : N;
    float s = 0.0f;
    for (int i = a + threadIdx.x; i < b; i += blockDim.x) s = s + obs[4 * N + i];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0 && e.segment_fitness) e.segment_fitness[g] = s;
    reward = reward + s;
  }
  if (threadIdx.x == 0) *e.reward = reward;
}

}  // namespace mc

namespace {
mc_status env_fail(mc_status s, const char* msg) {
  mc::set_last_error(msg);
  return s;
}
}  // namespace

extern "C" {

size_t mc_env_table_bytes(int32_t n) { return n > 0 ? (size_t)n * sizeof(mc_env) : 0; }

mc_status mc_env_table_upload(const mc_env* envs, int32_t n, void* table, void* stream) {
  if (n <= 0 || !envs || !table) return env_fail(MC_ERR_INVALID, "mc_env_table_upload: empty table or null pointer");
  if (reinterpret_cast<uintptr_t>(table) % alignof(mc_env) != 0)
    return env_fail(MC_ERR_INVALID, "mc_env_table_upload: table is not aligned");
  for (int i = 0; i < n; ++i) {
    const mc_env& e = envs[i];
    if (e.N <= 0 || e.E < 0 || e.B < 0 || e.H < 1 || e.W < 1)
      return env_fail(MC_ERR_INVALID, "mc_env_table_upload: bad sizes");
    if ((e.E > 0 && (!e.base_rest_lengths || !e.rest_lengths)) ||
        (e.B > 0 && (!e.base_bending_rest_angles || !e.bending_rest_angles)))
      return env_fail(MC_ERR_INVALID, "mc_env_table_upload: null rest buffer");
    if (!e.position || !e.velocity || !e.energy_center || !e.time || !e.observation || !e.reward || !e.done)
      return env_fail(MC_ERR_INVALID, "mc_env_table_upload: null state or output buffer");
    if (!(e.energy_two_size_sq > 0.0f)) return env_fail(MC_ERR_INVALID, "mc_env_table_upload: energy size must be > 0");
    if (e.num_segments > 1 && !e.segment_offsets)
      return env_fail(MC_ERR_INVALID, "mc_env_table_upload: several segments need segment_offsets");
  }
  const mc::Upload u{table, envs, (size_t)n * sizeof(mc_env)};
  cudaError_t err = mc::stage_uploads(&u, 1, static_cast<cudaStream_t>(stream));
  return err == cudaSuccess ? MC_OK : env_fail(MC_ERR_CUDA, cudaGetErrorString(err));
}

mc_status mc_env_act(const void* table, int32_t n, void* stream) {
  if (n <= 0 || !table) return env_fail(MC_ERR_INVALID, "mc_env_act: empty table");
  mc::k_env_act<<<n, mc::kEnvThreads, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const mc_env*>(table));
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? MC_OK : env_fail(MC_ERR_CUDA, cudaGetErrorString(err));
}

mc_status mc_env_observe(const void* table, int32_t n, int32_t advance, void* stream) {
  if (n <= 0 || !table) return env_fail(MC_ERR_INVALID, "mc_env_observe: empty table");
  mc::k_env_observe<<<n, mc::kEnvThreads, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const mc_env*>(table), advance ? 1 : 0);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? MC_OK : env_fail(MC_ERR_CUDA, cudaGetErrorString(err));
}

}  // extern "C"
