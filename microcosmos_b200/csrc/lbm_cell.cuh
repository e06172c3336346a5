// Per-cell D2Q9 TRT + Guo arithmetic shared by the dense pass and the IB pre-pass.
// Operation order follows src/microcosmos/solver/fluid.py (compiled with -fmad=false so
// every product and sum is rounded as in the reference's float32 elementwise ops).
#pragma once
#include "mc_internal.cuh"

namespace mc {

// D2Q9 velocities and weights (src/microcosmos/solver/fluid.py:15-23)
__device__ __constant__ static const int kEx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
__device__ __constant__ static const int kEy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};

// jnp.maximum / jnp.minimum propagate NaN from the array operand; fmaxf/fminf do not.
__device__ __forceinline__ float max_prop(float v, float c) { return (v < c) ? c : v; }
__device__ __forceinline__ float min_prop(float c, float v) { return (v > c) ? c : v; }

// The same maximum in one instruction: max.NaN returns NaN when an operand is NaN and the
// larger operand otherwise, so for a non-NaN constant c it equals max_prop(v, c).
__device__ __forceinline__ float max_nan(float v, float c) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(v), "f"(c));
  return r;
}

// TRT collision of a cell with no body force whose velocity clamp factor is exactly 1, so
// that u* = u (fluid.py:346 with F = 0) and the Guo source is zero, then the EPSIL floor.
// usq = ux^2 + uy^2 as the reference rounds it.  hwp = wp/2, hwm = wm/2 (exact halvings).
//
// Same bits as collide() with F = 0, with fewer operations, by exact identities:
//  * for opposite directions (i, o), e_o.u = -(e_i.u) exactly, so 3 e_o.u = -(3 e_i.u),
//    1 + 3 e_o.u = 1 - 3 e_i.u and (e_o.u)^2 = (e_i.u)^2: each pair shares those terms;
//  * 0.5 a - 0.5 b = 0.5 (a - b) and wp (0.5 d) = (0.5 wp) d exactly (scaling by a power of
//    two commutes with rounding away from the subnormal range, which populations >= EPSIL
//    and their equilibria never reach), so sym = (f_i + f_o) - (feq_i + feq_o) scaled into
//    hwp, anti likewise into hwm, and the o direction takes the negated antisymmetric term;
//  * the rest direction: 0.5 (f0 + f0) = f0, its antisymmetric part is 0, so
//    out0 = f0 - wp (f0 - feq0).
__device__ __forceinline__ void collide_free(const float f[9], float rho, float ux, float uy, float usq, float wp,
                                             float hwp, float hwm, float out[9]) {
  const float s = 1.5f * usq;
  const float r0 = rho * (4.0f / 9.0f), r1 = rho * (1.0f / 9.0f), r2 = rho * (1.0f / 36.0f);
  out[0] = max_nan(f[0] - wp * (f[0] - r0 * (1.0f - s)), MC_EPSIL);
  // pairs (1,3), (2,4), (5,7), (6,8): e_i.u = ux, uy, ux + uy, uy - ux
  const float e[4] = {ux, uy, ux + uy, uy - ux};
  const int pi[4] = {1, 2, 5, 6};
  const int po[4] = {3, 4, 7, 8};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float rw = q < 2 ? r1 : r2;
    const float t = 3.0f * e[q];
    const float sq = 4.5f * (e[q] * e[q]);
    const float feq_i = rw * (((1.0f + t) + sq) - s);
    const float feq_o = rw * (((1.0f - t) + sq) - s);
    const float fi = f[pi[q]], fo = f[po[q]];
    const float a = hwp * ((fi + fo) - (feq_i + feq_o));
    const float b = hwm * ((fi - fo) - (feq_i - feq_o));
    out[pi[q]] = max_nan((fi - a) - b, MC_EPSIL);
    out[po[q]] = max_nan((fo - a) + b, MC_EPSIL);
  }
}

// min(1, vmax / (sqrt(x^2 + y^2 + EPSIL) + EPSIL))  (fluid.py:272-273, 300-301, 327-328)
__device__ __forceinline__ float clamp_factor(float x, float y, float vmax) {
  float mag = sqrtf((x * x + y * y) + MC_EPSIL);
  return min_prop(1.0f, vmax / (mag + MC_EPSIL));
}

// The same factor with an exact shortcut: when x^2 + y^2 + EPSIL <= vmax^2 / 4 the magnitude
// is at most vmax / 2, so vmax / (mag + EPSIL) > 1 and the factor is exactly 1.
// q4 = vmax^2 / 4 (computed on the host, rounded down).  NaN inputs take the full path.
__device__ __forceinline__ float clamp_factor_fast(float x, float y, float vmax, float q4) {
  const float m2 = (x * x + y * y) + MC_EPSIL;
  if (m2 <= q4) return 1.0f;
  return min_prop(1.0f, vmax / (sqrtf(m2) + MC_EPSIL));
}

// rho = max(sum f, 0.1); u = sum e f / rho; velocity clamp (fluid.py:136-142, 268-274).
// The reference first floors f at EPSIL (fluid.py:268); the pull-scheme state only holds
// values that already passed that floor (the entry conversion applies it, every
// collision output re-applies it), so f is used as is.  Returns rho and the clamped velocity.
__device__ __forceinline__ void macroscopic(const float f[9], float vmax, float q4, float& rho, float& vx, float& vy) {
  float r = f[0];
#pragma unroll
  for (int i = 1; i < 9; ++i) r = r + f[i];
  r = max_prop(r, 0.1f);
  float ux = ((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8];
  float uy = ((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8];
  ux = ux / r;
  uy = uy / r;
  float c1 = clamp_factor_fast(ux, uy, vmax, q4);
  rho = r;
  vx = ux * c1;
  vy = uy * c1;
}

// Force of a cell that no IB point touches: the post-accumulation clamp applied to the
// unchanged velocity (fluid.py:327-339).
__device__ __forceinline__ void free_cell_force(float rho, float vx, float vy, float vmax, float q4, int force_clamp,
                                                float& Fx, float& Fy) {
  float c2 = clamp_factor_fast(vx, vy, vmax, q4);
  if (c2 == 1.0f) {  // (v * 1 - v) * rho == 0 exactly
    Fx = 0.0f;
    Fy = 0.0f;
    return;
  }
  Fx = (vx * c2 - vx) * rho;
  Fy = (vy * c2 - vy) * rho;
  if (force_clamp) {
    float c3 = clamp_factor(Fx, Fy, vmax);
    Fx = Fx * c3;
    Fy = Fy * c3;
  }
}

// TRT collision at u* = u + F/(2 rho) with the TRT-aware Guo source and the EPSIL floor
// (fluid.py:145-199, 342-350).  f holds the clamped populations.  cp = 1 - wp/2 and
// cm = 1 - wm/2 are computed on the host in float32.
__device__ __forceinline__ void collide(const float f[9], float rho, float vx, float vy, float Fx, float Fy,
                                        float wp, float wm, float cp, float cm, float out[9],
                                        float& usx_o, float& usy_o) {
  const float half = 0.5f;
  const bool force = !(Fx == 0.0f && Fy == 0.0f);
  // with F = 0, u* = u + (0.5 * 0) / rho = u exactly
  float usx = force ? vx + (half * Fx) / rho : vx;
  float usy = force ? vy + (half * Fy) / rho : vy;
  float usq = usx * usx + usy * usy;
  float eu[9];
  eu[0] = 0.0f;
  eu[1] = usx;
  eu[2] = usy;
  eu[3] = -usx;
  eu[4] = -usy;
  eu[5] = usx + usy;
  eu[6] = -usx + usy;
  eu[7] = -usx - usy;
  eu[8] = usx - usy;
  const float w[9] = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                      1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
  float feq[9];
#pragma unroll
  for (int i = 0; i < 9; ++i)
    feq[i] = (rho * w[i]) * (((1.0f + 3.0f * eu[i]) + 4.5f * (eu[i] * eu[i])) - 1.5f * usq);
  // Opposite directions (i, o): f_i + f_o and feq_i + feq_o are commutative sums, and
  // 0.5 (f_o - f_i) - 0.5 (feq_o - feq_i) is exactly the negation of the i term, so each
  // pair's symmetric and antisymmetric parts are computed once:
  //   out_i = (f_i - wp*sym) - wm*anti,   out_o = (f_o - wp*sym) - wm*(-anti)
  const int pi[4] = {1, 2, 5, 6};
  const int po[4] = {3, 4, 7, 8};
  {
    // rest direction: f_o = f_i, the antisymmetric part is 0 - 0
    const float sym = half * (f[0] + f[0]) - half * (feq[0] + feq[0]);
    const float anti = half * (f[0] - f[0]) - half * (feq[0] - feq[0]);
    out[0] = (f[0] - wp * sym) - wm * anti;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = pi[q], o = po[q];
    const float sym = half * (f[i] + f[o]) - half * (feq[i] + feq[o]);
    const float anti = half * (f[i] - f[o]) - half * (feq[i] - feq[o]);
    out[i] = (f[i] - wp * sym) - wm * anti;
    out[o] = (f[o] - wp * sym) - wm * (-anti);
  }
  if (!force) {
    // zero force: the Guo source is exactly zero and u* = u
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = max_prop(out[i], MC_EPSIL);
  } else {
    float eF[9];
    eF[0] = 0.0f;
    eF[1] = Fx;
    eF[2] = Fy;
    eF[3] = -Fx;
    eF[4] = -Fy;
    eF[5] = Fx + Fy;
    eF[6] = -Fx + Fy;
    eF[7] = -Fx - Fy;
    eF[8] = Fx - Fy;
    float udF = usx * Fx + usy * Fy;
    float raw[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) raw[i] = w[i] * (3.0f * (eF[i] - udF) + (9.0f * eu[i]) * eF[i]);
    const int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      int o = opp[i];
      float src = cp * (half * (raw[i] + raw[o])) + cm * (half * (raw[i] - raw[o]));
      out[i] = max_prop(out[i] + src, MC_EPSIL);
    }
  }
  usx_o = usx;
  usy_o = usy;
}

}  // namespace mc
