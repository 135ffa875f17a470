// fss_device.cuh -- device building blocks shared by every fast_shepherd_score_b200 kernel.
//
// Math conventions (identical to the reference shepherd_score batched path):
//   * pose = (q, t), q = (w, x, y, z); the fit cloud moves: b' = R(q) b + t
//   * shape overlap  V = K * sum_ij exp(-alpha/2 |a_i - b'_j|^2),  K = pi^1.5 / (2 alpha)^1.5
//     (accel/kernels/shape_triton.py:73-188)
//   * ESP overlap    the same with an extra factor exp(-(c_i - c_j)^2 / lam)
//     (accel/kernels/esp_triton.py:21-172)
//   * typed pharmacophore overlap with directional weights (accel/kernels/pharm_triton.py:296-400)
//   * dV/dt = sum_j f_j,  dV/dq = sum_j f_j . (dR/dq) b_j  with f_j = sum_i alpha g_ij (a_i - b'_j)
//     (the quaternion tail _quat_grad_tail, shape_triton.py:46-65), evaluated here through the
//     3x3 moment G = sum_j f_j b_j^T, which is the same linear form regrouped.
//   * Tanimoto score / Adam tail of accel/kernels/cpu_fused.py:54-167 (no bias correction,
//     eps inside the sqrt, tangent projection of the quaternion gradient, renormalisation).
//
// Arithmetic layout of the pairwise sum (the hot loop): with k = alpha/2 * log2(e) the base-2
// exponent of one term is
//       E_ij = P_i.w + F_j.w + P_i.xyz . b'_j            (+ Qc_i * c_j for ESP)
//   P_i = (2k a_i, -k|a_i|^2 - e c_i^2)   staged once per pair in shared memory
//   F_j.w = -k|b'_j|^2 - e c_j^2          recomputed per pose and step in registers
//   Qc_i = 2 e c_i, e = log2(e) / lam
// so a term costs one ex2 on the MUFU pipe plus 8 FP32 ops (4 for the exponent, 4 for
// the value / gradient accumulation), against 11+ for the direct difference form.  The
// reference cloud is centred on its own centroid before staging, which keeps |a|^2 small
// and the expanded form's cancellation error below 1e-6 relative per term.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fss {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kPi15 = 5.568327996831708f;  // pi ** 1.5
constexpr float kBeta1 = 0.9f;
constexpr float kBeta2 = 0.999f;
constexpr float kAdamEps = 1e-8f;

// 2^x on the MUFU pipe (flush-to-zero; -inf -> +0).
__device__ __forceinline__ float ex2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

struct Rot {
  float r[9];
};

// Rotation matrix from a (w,x,y,z) quaternion, the expression of shape_triton.py:35-43.
__device__ __forceinline__ Rot quat_to_rot(const float q[4]) {
  const float qr = q[0], qi = q[1], qj = q[2], qk = q[3];
  Rot R;
  R.r[0] = 1.f - 2.f * (qj * qj + qk * qk);
  R.r[1] = 2.f * (qi * qj - qk * qr);
  R.r[2] = 2.f * (qi * qk + qj * qr);
  R.r[3] = 2.f * (qi * qj + qk * qr);
  R.r[4] = 1.f - 2.f * (qi * qi + qk * qk);
  R.r[5] = 2.f * (qj * qk - qi * qr);
  R.r[6] = 2.f * (qi * qk - qj * qr);
  R.r[7] = 2.f * (qj * qk + qi * qr);
  R.r[8] = 1.f - 2.f * (qi * qi + qj * qj);
  return R;
}

__device__ __forceinline__ float3 rot_apply(const Rot& R, float x, float y, float z) {
  return make_float3(fmaf(R.r[0], x, fmaf(R.r[1], y, R.r[2] * z)),
                     fmaf(R.r[3], x, fmaf(R.r[4], y, R.r[5] * z)),
                     fmaf(R.r[6], x, fmaf(R.r[7], y, R.r[8] * z)));
}

// Per-lane partial sums of one channel: value, translation force and the 3x3 moment
// G[r][c] = sum_j f_j[r] * b_j[c] (row-major).
struct Moments {
  float v;
  float f[3];
  float g[9];
  __device__ __forceinline__ void zero() {
    v = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] = 0.f;
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] = 0.f;
  }
  __device__ __forceinline__ void add_force(float fx, float fy, float fz, float bx, float by,
                                            float bz) {
    f[0] += fx; f[1] += fy; f[2] += fz;
    g[0] = fmaf(fx, bx, g[0]); g[1] = fmaf(fx, by, g[1]); g[2] = fmaf(fx, bz, g[2]);
    g[3] = fmaf(fy, bx, g[3]); g[4] = fmaf(fy, by, g[4]); g[5] = fmaf(fy, bz, g[5]);
    g[6] = fmaf(fz, bx, g[6]); g[7] = fmaf(fz, by, g[7]); g[8] = fmaf(fz, bz, g[8]);
  }
  // Butterfly sum over an aligned group of `width` lanes; every lane ends with the total.
  template <int WIDTH>
  __device__ __forceinline__ void group_sum() {
#pragma unroll
    for (int o = WIDTH / 2; o > 0; o >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, o);
#pragma unroll
      for (int i = 0; i < 3; ++i) f[i] += __shfl_xor_sync(0xffffffffu, f[i], o);
#pragma unroll
      for (int i = 0; i < 9; ++i) g[i] += __shfl_xor_sync(0xffffffffu, g[i], o);
    }
  }
  __device__ __forceinline__ void scale(float sv, float sf) {
    v *= sv;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] *= sf;
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] *= sf;
  }
};

// dV/dq from the moment G at quaternion q: the reference's per-point tail
// (shape_triton.py:46-65) summed over points and regrouped by G's entries.
__device__ __forceinline__ void quat_grad_from_moment(const float q[4], const float G[9],
                                                      float dq[4]) {
  const float qr = q[0], qi = q[1], qj = q[2], qk = q[3];
  const float xx = G[0], xy = G[1], xz = G[2], yx = G[3], yy = G[4], yz = G[5], zx = G[6],
              zy = G[7], zz = G[8];
  dq[0] = 2.f * (qk * (yx - xy) + qj * (xz - zx) + qi * (zy - yz));
  dq[1] = 2.f * (qj * (xy + yx) + qk * (xz + zx) + qr * (zy - yz) - 2.f * qi * (yy + zz));
  dq[2] = 2.f * (qi * (xy + yx) + qk * (yz + zy) + qr * (xz - zx) - 2.f * qj * (xx + zz));
  dq[3] = 2.f * (qi * (xz + zx) + qj * (yz + zy) + qr * (yx - xy) - 2.f * qk * (xx + yy));
}

// What a pose group reduces per step: value, dV/dt and dV/dq.  dV/dq is linear in the
// moment G, so every lane turns its partial G into a partial dq first and the butterfly
// moves 8 floats instead of 13.
struct Reduced {
  float v, f[3], dq[4];
  __device__ __forceinline__ void from(const Moments& m, const float q[4]) {
    v = m.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] = m.f[i];
    quat_grad_from_moment(q, m.g, dq);
  }
  template <int WIDTH>
  __device__ __forceinline__ void group_sum() {
#pragma unroll
    for (int o = WIDTH / 2; o > 0; o >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, o);
#pragma unroll
      for (int i = 0; i < 3; ++i) f[i] += __shfl_xor_sync(0xffffffffu, f[i], o);
#pragma unroll
      for (int i = 0; i < 4; ++i) dq[i] += __shfl_xor_sync(0xffffffffu, dq[i], o);
    }
  }
  __device__ __forceinline__ void scale(float sv, float sf) {
    v *= sv;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[i] *= sf;
#pragma unroll
    for (int i = 0; i < 4; ++i) dq[i] *= sf;
  }
};

// Loop-carried optimiser state of one pose.
struct PoseState {
  float q[4], t[3];
  float mq[4], vq[4], mt[3], vt[3];
  float best, bq[4], bt[3];
};

// The optimiser state that the hot loop does not read (Adam moments, best score and pose) is
// parked in shared memory between tails, so the registers go to the pairwise loop.  Each
// thread owns one column (field f of thread x at f * nthreads + x), so no synchronisation is
// needed; volatile keeps the compiler from carrying the values in registers across the loop.
constexpr int kColdFields = 22;

__device__ __forceinline__ void cold_store(const PoseState& s, volatile float* c, int stride) {
  int f = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) c[(f++) * stride] = s.mq[i];
#pragma unroll
  for (int i = 0; i < 4; ++i) c[(f++) * stride] = s.vq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) c[(f++) * stride] = s.mt[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) c[(f++) * stride] = s.vt[i];
  c[(f++) * stride] = s.best;
#pragma unroll
  for (int i = 0; i < 4; ++i) c[(f++) * stride] = s.bq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) c[(f++) * stride] = s.bt[i];
}

__device__ __forceinline__ void cold_load(PoseState& s, const volatile float* c, int stride) {
  int f = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) s.mq[i] = c[(f++) * stride];
#pragma unroll
  for (int i = 0; i < 4; ++i) s.vq[i] = c[(f++) * stride];
#pragma unroll
  for (int i = 0; i < 3; ++i) s.mt[i] = c[(f++) * stride];
#pragma unroll
  for (int i = 0; i < 3; ++i) s.vt[i] = c[(f++) * stride];
  s.best = c[(f++) * stride];
#pragma unroll
  for (int i = 0; i < 4; ++i) s.bq[i] = c[(f++) * stride];
#pragma unroll
  for (int i = 0; i < 3; ++i) s.bt[i] = c[(f++) * stride];
}

__device__ __forceinline__ void pose_init(PoseState& s, const float q0[4], const float t0[3]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) { s.q[i] = q0[i]; s.bq[i] = q0[i]; s.mq[i] = 0.f; s.vq[i] = 0.f; }
#pragma unroll
  for (int i = 0; i < 3; ++i) { s.t[i] = t0[i]; s.bt[i] = t0[i]; s.mt[i] = 0.f; s.vt[i] = 0.f; }
  s.best = -INFINITY;
}

#ifndef FSS_TAIL_RCP
#define FSS_TAIL_RCP 1
#endif

// x / sqrt(y) of the Adam update
__device__ __forceinline__ float adam_ratio(float x, float y) {
#if FSS_TAIL_RCP
  return x * __frsqrt_rn(y);
#else
  return x / sqrtf(y);
#endif
}

// Best-pose tracking (pre-update pose) + tangent-projected Adam on q, plain Adam on t,
// quaternion renormalisation: cpu_fused.py:68-108 / shape_triton.py:253-368.
__device__ __forceinline__ void adam_tail(PoseState& s, float score, const float gq[4],
                                          const float gt[3], float lr) {
  if (score > s.best) {  // NaN never replaces the best, as in the reference comparison
    s.best = score;
#pragma unroll
    for (int i = 0; i < 4; ++i) s.bq[i] = s.q[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) s.bt[i] = s.t[i];
  }
  // x / sqrt(y) as x * (correctly rounded 1/sqrt(y)): one rounding more than the quotient of
  // the reference, and a fraction of the instructions of an IEEE square root and division
  // (FSS_TAIL_RCP=0 builds the quotient form)
  const float radial = gq[0] * s.q[0] + gq[1] * s.q[1] + gq[2] * s.q[2] + gq[3] * s.q[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float d = gq[i] - s.q[i] * radial;
    s.mq[i] = kBeta1 * s.mq[i] + (1.f - kBeta1) * d;
    s.vq[i] = kBeta2 * s.vq[i] + (1.f - kBeta2) * d * d;
    s.q[i] = s.q[i] - adam_ratio(lr * s.mq[i], s.vq[i] + kAdamEps);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float d = gt[i];
    s.mt[i] = kBeta1 * s.mt[i] + (1.f - kBeta1) * d;
    s.vt[i] = kBeta2 * s.vt[i] + (1.f - kBeta2) * d * d;
    s.t[i] = s.t[i] - adam_ratio(lr * s.mt[i], s.vt[i] + kAdamEps);
  }
  // renormalise: q / max(|q|, 1e-12)
  const float n2 = s.q[0] * s.q[0] + s.q[1] * s.q[1] + s.q[2] * s.q[2] + s.q[3] * s.q[3];
#if FSS_TAIL_RCP
  const float inv = __frsqrt_rn(fmaxf(n2, 1e-24f));
#pragma unroll
  for (int i = 0; i < 4; ++i) s.q[i] = s.q[i] * inv;
#else
  const float qn = fmaxf(sqrtf(n2), 1e-12f);
#pragma unroll
  for (int i = 0; i < 4; ++i) s.q[i] = s.q[i] / qn;
#endif
}

// Tanimoto score V/(U-V) and its derivative scale U/(U-V)^2 (cpu_fused.py:62-67), from one
// correctly rounded reciprocal of the denominator.
__device__ __forceinline__ void tanimoto(float V, float U, float& score, float& scale) {
  float denom = U - V;
  if (denom == 0.f) denom = 1e-12f;
#if FSS_TAIL_RCP
  const float r = __frcp_rn(denom);
  score = V * r;
  scale = (U * r) * r;
#else
  score = V / denom;
  scale = U / (denom * denom);
#endif
}

// Single-channel step: score, best tracking and Adam from the channel's reduced sums.
__device__ __forceinline__ void step_single(PoseState& s, const Reduced& m, float U, float lr) {
  float score, scale;
  tanimoto(m.v, U, score, scale);
  float gq[4], gt[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) gq[i] = -scale * m.dq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) gt[i] = -scale * m.f[i];
  adam_tail(s, score, gq, gt, lr);
}

// Tversky step (accel/drivers/pharm_overlap.py:36-59, analytical_gradients/_torch.py:416-436):
// score = min(V / D, 1) with D = sigma V_AA + (1 - sigma) V_BB (0 when D <= 1e-8); the
// gradient is V'/D while V < D and 0 once the score is clamped.
__device__ __forceinline__ void step_tversky(PoseState& s, const Reduced& m, float D, float lr) {
  const float score = D > 1e-8f ? fminf(m.v / D, 1.f) : 0.f;
  const float scale = m.v < D ? 1.f / D : 0.f;
  float gq[4], gt[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) gq[i] = -scale * m.dq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) gt[i] = -scale * m.f[i];
  adam_tail(s, score, gq, gt, lr);
}

// vol_and_surf_esp step (accel/drivers/esp_combo.py:497-595): the pose follows the shape
// gradient scaled by (1 - w); on scored steps the tracked score is
// w * (esp1 + esp2) / n_surf + (1 - w) * V / (U - V).  Unscored steps never update the best.
__device__ __forceinline__ void step_esp_combo(PoseState& s, const Reduced& m, float U,
                                               float esp_sum, float n_surf, float w,
                                               bool scored, float lr) {
  float vs, scale;
  tanimoto(m.v, U, vs, scale);
  const float score = scored ? w * (esp_sum / n_surf) + (1.f - w) * vs : -INFINITY;
  const float c = -scale * (1.f - w);
  float gq[4], gt[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) gq[i] = c * m.dq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) gt[i] = c * m.f[i];
  adam_tail(s, score, gq, gt, lr);
}

// One side of the ShaEP ESP comparison for one pose (cpu.py:237-261, esp_triton.py:265-346):
//   sum over field points i of exp(-(pe_i - coulomb * sum_m q_m / max(d_im, 1e-6))^2 / lam')
// skipping points within radius_m + probe of any atom.  Field points (x, y, z, pe) and atoms
// live in different frames: TO_BODY maps a field point of the reference frame into the fit
// body frame (u = R^T (p - t)), otherwise a body-frame field point into the reference frame
// (u = R p + t).  Atoms are staged negated and duplicated for f32x2 arithmetic over two field
// points per lane: atoms[2m] = (-x, -x, -y, -y), atoms[2m+1] = (-z, -z, q, q),
// rp2[m] = (-(r+probe)^2, same).
// The 1e-6 distance floor never matters: an atom that close blocks the point, and blocked
// points contribute nothing, so 1/d is a plain rsqrt.  Lanes split the field points; returns
// this lane's partial sum (nkl = -log2(e) / lam').
template <int LPP, bool TO_BODY>
__device__ __forceinline__ float esp_side(const float4* __restrict__ field, int n,
                                          const float4* __restrict__ atoms,
                                          const float2* __restrict__ rp2, int m, int lane,
                                          const Rot& R, float tx, float ty, float tz,
                                          float coulomb, float nkl) {
  float total = 0.f;
  for (int i0 = lane; i0 < n; i0 += 2 * LPP) {
    const int i1 = i0 + LPP;
    const bool has1 = i1 < n;
    const float4 fa = field[i0];
    const float4 fb = has1 ? field[i1] : fa;
    float u[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float4 f = h ? fb : fa;
      if (TO_BODY) {
        const float px = f.x - tx, py = f.y - ty, pz = f.z - tz;
        u[h][0] = fmaf(R.r[0], px, fmaf(R.r[3], py, R.r[6] * pz));
        u[h][1] = fmaf(R.r[1], px, fmaf(R.r[4], py, R.r[7] * pz));
        u[h][2] = fmaf(R.r[2], px, fmaf(R.r[5], py, R.r[8] * pz));
      } else {
        const float3 p3 = rot_apply(R, f.x, f.y, f.z);
        u[h][0] = p3.x + tx; u[h][1] = p3.y + ty; u[h][2] = p3.z + tz;
      }
    }
    const float2 UX = f2(u[0][0], u[1][0]), UY = f2(u[0][1], u[1][1]), UZ = f2(u[0][2], u[1][2]);
    float2 esp = f2(0.f, 0.f);
    float gap0 = INFINITY, gap1 = INFINITY;  // min over atoms of d^2 - (r + probe)^2
#pragma unroll 2
    for (int j = 0; j < m; ++j) {
      const float4 a = atoms[2 * j], b = atoms[2 * j + 1];
      const float2 dx = __fadd2_rn(UX, f2(a.x, a.y)), dy = __fadd2_rn(UY, f2(a.z, a.w));
      const float2 dz = __fadd2_rn(UZ, f2(b.x, b.y));
      const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
      esp = __ffma2_rn(f2(b.z, b.w), f2(rsqrtf(d2.x), rsqrtf(d2.y)), esp);
      const float2 gap = __fadd2_rn(d2, rp2[j]);
      gap0 = fminf(gap0, gap.x);
      gap1 = fminf(gap1, gap.y);
    }
    if (gap0 >= 0.f) {
      const float diff = fmaf(-coulomb, esp.x, fa.w);
      total += ex2(nkl * diff * diff);
    }
    if (has1 && gap1 >= 0.f) {
      const float diff = fmaf(-coulomb, esp.y, fb.w);
      total += ex2(nkl * diff * diff);
    }
  }
  return total;
}

// Two-channel step (1-w) * shape + w * pharm, the joint gradient of cpu_fused.py:111-167.
__device__ __forceinline__ void step_combo(PoseState& s, const Reduced& ms, float Us,
                                           const Reduced& mc, float Uc, float w, float lr) {
  float ss, scs, sc, scc;
  tanimoto(ms.v, Us, ss, scs);
  tanimoto(mc.v, Uc, sc, scc);
  const float score = (1.f - w) * ss + w * sc;
  const float cs = -(1.f - w) * scs, cc = -w * scc;
  float gq[4], gt[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) gq[i] = cs * ms.dq[i] + cc * mc.dq[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) gt[i] = cs * ms.f[i] + cc * mc.f[i];
  adam_tail(s, score, gq, gt, lr);
}

// ---------------------------------------------------------------------------------------
// Shape / ESP pairwise sum for one pose.
//
// Shared-memory layout of the staged reference cloud (point i):
//   sPd[2i]   = (Px, Px, Py, Py)      sPd[2i+1] = (Pz, Pz, Pw, Pw)      sQd[i] = (Qc, Qc)
// i.e. every component duplicated so that one 16-byte load yields the float2 operands of
// the packed f32x2 instructions (__ffma2_rn / __fadd2_rn), which process two fit points
// per instruction and halve the FP32 issue cost of the hot loop.
//
// The lanes of one pose group (LPP consecutive lanes) split the fit points j = lane + LPP*u;
// every lane loops over all N staged reference points.  Returns the lane's partial moments
// in "raw" units: v = sum g, f_j = sum_i g (a_i - b'_j) (multiply by K and alpha K).
//
// Factored exponent: the per-fit-point part F_j.w of the exponent is constant over i, so
//   sum_i 2^(P_i.w + P_i.b' + F_j.w) = 2^(F_j.w) * sum_i 2^(P_i.w + P_i.b')
// and the hot loop costs 3 FMA (+1 for ESP) for the exponent instead of 4 (+1).  The
// unscaled exponent P_i.w + P_i.b' = -k|a_i-b'|^2 + k|b'|^2 (+ESP terms) is bounded by
// -F_j.w; when that exceeds kFactorMax for any point of the warp the chunk falls back to
// the unfactored form so 2^x can never overflow.
// ---------------------------------------------------------------------------------------
constexpr float kFactorMax = 96.f;

// An odd last fit point per lane goes to a one-point scalar chunk instead of a half-empty
// packed pair (0 keeps the packed pair).
#ifndef FSS_PLAIN_TAIL
#define FSS_PLAIN_TAIL 1
#endif


template <int JB, bool ESP>
__device__ __forceinline__ void shape_chunk_plain(const float4* __restrict__ sPd,
                                                  const float2* __restrict__ sQd,
                                                  const float4* __restrict__ sB, int N, int M,
                                                  int j0, int stride, const Rot& R, float tx,
                                                  float ty, float tz, float k, float e,
                                                  float inv2k, Moments& acc) {
  float bx[JB], by[JB], bz[JB], fw[JB], cj[JB];
  float sg[JB], sx[JB], sy[JB], sz[JB];
#pragma unroll
  for (int u = 0; u < JB; ++u) {
    const int j = j0 + u * stride;
    const bool ok = j < M;
    const float4 b = ok ? sB[j] : make_float4(0.f, 0.f, 0.f, 0.f);
    cj[u] = b.w;
    const float3 p = rot_apply(R, b.x, b.y, b.z);
    bx[u] = p.x + tx; by[u] = p.y + ty; bz[u] = p.z + tz;
    float w = -k * (bx[u] * bx[u] + by[u] * by[u] + bz[u] * bz[u]);
    if (ESP) w = fmaf(-e * b.w, b.w, w);
    fw[u] = ok ? w : -INFINITY;
    sg[u] = 0.f; sx[u] = 0.f; sy[u] = 0.f; sz[u] = 0.f;
  }
  for (int i = 0; i < N; ++i) {
    const float4 a = sPd[2 * i], c = sPd[2 * i + 1];
    const float px = a.x, py = a.z, pz = c.x, pw = c.z;
    float qc = 0.f;
    if (ESP) qc = sQd[i].x;
#pragma unroll
    for (int u = 0; u < JB; ++u) {
      float E = fmaf(px, bx[u], fmaf(py, by[u], fmaf(pz, bz[u], pw + fw[u])));
      if (ESP) E = fmaf(qc, cj[u], E);
      const float g = ex2(E);
      sg[u] += g;
      sx[u] = fmaf(g, px, sx[u]);
      sy[u] = fmaf(g, py, sy[u]);
      sz[u] = fmaf(g, pz, sz[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < JB; ++u) {
    const int j = j0 + u * stride;
    if (j < M) {
      const float4 b = sB[j];
      acc.v += sg[u];
      acc.add_force(fmaf(sx[u], inv2k, -bx[u] * sg[u]), fmaf(sy[u], inv2k, -by[u] * sg[u]),
                    fmaf(sz[u], inv2k, -bz[u] * sg[u]), b.x, b.y, b.z);
    }
  }
}

// Packed chunk: JB2 float2 pairs = 2*JB2 fit points per lane, f32x2 arithmetic, factored
// exponent.  Returns false (and does nothing) when the factored form could overflow.
template <int JB2, bool ESP, int UNR>
__device__ __forceinline__ bool shape_chunk_packed(const float4* __restrict__ sPd,
                                                   const float2* __restrict__ sQd,
                                                   const float4* __restrict__ sB, int N, int M,
                                                   int j0, int stride, const Rot& R, float tx,
                                                   float ty, float tz, float k, float e,
                                                   float inv2k, Moments& acc) {
  float2 bx[JB2], by[JB2], bz[JB2], cj[JB2];
  float2 sg[JB2], sx[JB2], sy[JB2], sz[JB2];
  bool big = false;
#pragma unroll
  for (int v = 0; v < JB2; ++v) {
    float xs[2], ys[2], zs[2], cs[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = j0 + (2 * v + h) * stride;
      const float4 b = j < M ? sB[j] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float3 p = rot_apply(R, b.x, b.y, b.z);
      xs[h] = p.x + tx; ys[h] = p.y + ty; zs[h] = p.z + tz; cs[h] = b.w;
      float w = k * (xs[h] * xs[h] + ys[h] * ys[h] + zs[h] * zs[h]);
      if (ESP) w = fmaf(e * b.w, b.w, w);
      big = big || (j < M && w > kFactorMax);
    }
    bx[v] = f2(xs[0], xs[1]); by[v] = f2(ys[0], ys[1]); bz[v] = f2(zs[0], zs[1]);
    cj[v] = f2(cs[0], cs[1]);
    sg[v] = f2(0.f, 0.f); sx[v] = f2(0.f, 0.f); sy[v] = f2(0.f, 0.f); sz[v] = f2(0.f, 0.f);
  }
  // vote of this pose's lanes only (stride = lanes per pose, a power of two <= 32): a pose's
  // arithmetic path must not depend on the other poses that share its warp
  const unsigned vote = __ballot_sync(0xffffffffu, big);
  const unsigned own = stride >= 32 ? 0xffffffffu
                                    : ((1u << stride) - 1u) << ((threadIdx.x & 31) & ~(stride - 1));
  if (vote & own) return false;
#pragma unroll UNR
  for (int i = 0; i < N; ++i) {
    const float4 a = sPd[2 * i], c = sPd[2 * i + 1];
    const float2 PX = f2(a.x, a.y), PY = f2(a.z, a.w), PZ = f2(c.x, c.y), PW = f2(c.z, c.w);
    float2 QC;
    if (ESP) QC = sQd[i];
#pragma unroll
    for (int v = 0; v < JB2; ++v) {
      float2 E = __ffma2_rn(PX, bx[v], __ffma2_rn(PY, by[v], __ffma2_rn(PZ, bz[v], PW)));
      if (ESP) E = __ffma2_rn(QC, cj[v], E);
      const float2 g = f2(ex2(E.x), ex2(E.y));
      sg[v] = __fadd2_rn(sg[v], g);
      sx[v] = __ffma2_rn(g, PX, sx[v]);
      sy[v] = __ffma2_rn(g, PY, sy[v]);
      sz[v] = __ffma2_rn(g, PZ, sz[v]);
    }
  }
#pragma unroll
  for (int v = 0; v < JB2; ++v) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = j0 + (2 * v + h) * stride;
      if (j < M) {
        const float4 b = sB[j];
        const float x = h ? bx[v].y : bx[v].x, y = h ? by[v].y : by[v].x,
                    z = h ? bz[v].y : bz[v].x;
        float w = -k * (x * x + y * y + z * z);
        if (ESP) w = fmaf(-e * b.w, b.w, w);
        const float scale = ex2(w);
        const float g = (h ? sg[v].y : sg[v].x) * scale;
        const float gx = (h ? sx[v].y : sx[v].x) * scale;
        const float gy = (h ? sy[v].y : sy[v].x) * scale;
        const float gz = (h ? sz[v].y : sz[v].x) * scale;
        acc.v += g;
        acc.add_force(fmaf(gx, inv2k, -x * g), fmaf(gy, inv2k, -y * g),
                      fmaf(gz, inv2k, -z * g), b.x, b.y, b.z);
      }
    }
  }
  return true;
}

template <int JB2, bool ESP, int UNR>
__device__ __forceinline__ void shape_chunk(const float4* __restrict__ sPd,
                                            const float2* __restrict__ sQd,
                                            const float4* __restrict__ sB, int N, int M, int j0,
                                            int stride, const Rot& R, float tx, float ty,
                                            float tz, float k, float e, float inv2k,
                                            Moments& acc) {
  if (!shape_chunk_packed<JB2, ESP, UNR>(sPd, sQd, sB, N, M, j0, stride, R, tx, ty, tz, k, e, inv2k,
                                    acc))
    shape_chunk_plain<2 * JB2, ESP>(sPd, sQd, sB, N, M, j0, stride, R, tx, ty, tz, k, e, inv2k,
                                    acc);
}

// JB2: float2 pairs of fit points per lane per pass (register tile, 2*JB2 points);
// UNR: unroll depth of the loop over reference points.
template <int LPP, bool ESP, int JB2 = 2, int UNR = 2>
__device__ __forceinline__ void shape_pose(const float4* __restrict__ sPd,
                                           const float2* __restrict__ sQd,
                                           const float4* __restrict__ sB, int N, int M, int lane,
                                           const Rot& R, float tx, float ty, float tz, float k,
                                           float e, float inv2k, Moments& acc) {
  static_assert(JB2 >= 1 && JB2 <= 4, "register tile of 2..8 fit points");
  // Trip counts depend only on M and LPP, so every lane of the group (and every group of
  // the warp, which share one pair) runs the same loop; points past M are masked.
  int base = 0;
  for (; base + 2 * JB2 * LPP <= M; base += 2 * JB2 * LPP)
    shape_chunk<JB2, ESP, UNR>(sPd, sQd, sB, N, M, base + lane, LPP, R, tx, ty, tz, k, e, inv2k,
                               acc);
  // 0..2*JB2 points per lane are left: whole f32x2 pairs in the smallest packed tile that
  // holds them, and an odd last point per lane in a scalar chunk (FSS_PLAIN_TAIL), which
  // costs half the FP32/MUFU pipe time of a packed pair whose second slot would be empty
  const int ppl = (M - base + LPP - 1) / LPP;
  const int pairs = FSS_PLAIN_TAIL ? ppl / 2 : (ppl + 1) / 2;
  if (JB2 >= 4 && pairs == 4) {
    shape_chunk<(JB2 >= 4 ? 4 : 1), ESP, UNR>(sPd, sQd, sB, N, M, base + lane, LPP, R, tx, ty,
                                              tz, k, e, inv2k, acc);
  } else if (JB2 >= 3 && pairs == 3) {
    shape_chunk<(JB2 >= 3 ? 3 : 1), ESP, UNR>(sPd, sQd, sB, N, M, base + lane, LPP, R, tx, ty,
                                              tz, k, e, inv2k, acc);
  } else if (pairs == 2) {
    shape_chunk<2, ESP, UNR>(sPd, sQd, sB, N, M, base + lane, LPP, R, tx, ty, tz, k, e, inv2k,
                             acc);
  } else if (pairs == 1) {
    shape_chunk<1, ESP, UNR>(sPd, sQd, sB, N, M, base + lane, LPP, R, tx, ty, tz, k, e, inv2k,
                             acc);
  }
  if (FSS_PLAIN_TAIL && (ppl & 1))
    shape_chunk_plain<1, ESP>(sPd, sQd, sB, N, M, base + lane + 2 * pairs * LPP, LPP, R, tx, ty,
                              tz, k, e, inv2k, acc);
}

// ---------------------------------------------------------------------------------------
// Typed pharmacophore sum for one pose (pharm_triton.py:296-400, cpu.py:500-582).
// Anchors are staged as float4 (x, y, z, type bits); vectors are unit (x, y, z, 0).
// Lanes split the fit features; the same-type test is an exact integer compare.
// Partial moments in final units (K and alpha folded in per type).
// ---------------------------------------------------------------------------------------
struct PharmTables {
  float alpha[9];
  float K[9];
  int cat[9];
};

// EXT: 0 cosine-weighted directional types (the default); 1 extended points -- for acceptors
// and donors the anchor term gets weight 1 and an extra Gaussian between the extended points
// anchor + unit vector is added; 2 only the extended-point term (anchor weight 0).  The
// extended types are the typed overlap's EXTENDED_POINT_TYPES = {acceptor, donor}
// (accel/drivers/pharm_overlap.py:33, :185-200), which the batched fine loop differentiates;
// halogens keep their cosine weight.
template <int LPP, int EXT = 0>
__device__ __forceinline__ void pharm_pose(const float4* __restrict__ sRA,
                                           const float4* __restrict__ sRV,
                                           const float4* __restrict__ sFA,
                                           const float4* __restrict__ sFV, int N, int M,
                                           int lane, const Rot& R, float tx, float ty, float tz,
                                           const PharmTables& tab, Moments& acc,
                                           const int* __restrict__ toff = nullptr) {
  for (int j = lane; j < M; j += LPP) {
    const float4 fa = sFA[j];
    const int ityp = __float_as_int(fa.w);
    const int icat = tab.cat[ityp];
    if (icat == 3) continue;
    const float ialpha = tab.alpha[ityp], iK = tab.K[ityp];
    const float nk = -0.5f * ialpha * kLog2e;
    const float4 fv = sFV[j];
    const float3 pa = rot_apply(R, fa.x, fa.y, fa.z);
    const float ax = pa.x + tx, ay = pa.y + ty, az = pa.z + tz;
    const float3 pv = rot_apply(R, fv.x, fv.y, fv.z);
    const bool ext = EXT != 0 && (ityp == 0 || ityp == 1);  // acceptor, donor
    float fx = 0.f, fy = 0.f, fz = 0.f, wx = 0.f, wy = 0.f, wz = 0.f, o = 0.f;
    float ex = 0.f, ey = 0.f, ez = 0.f;  // force at the extended point (EXT)
    // reference features grouped by type (stage_ref_pharm with toff): only this type's range
    const int i0 = toff ? toff[ityp] : 0, i1 = toff ? toff[ityp + 1] : N;
    for (int i = i0; i < i1; ++i) {
      const float4 ra = sRA[i];
      if (__float_as_int(ra.w) != ityp) continue;
      const float dx = ra.x - ax, dy = ra.y - ay, dz = ra.z - az;  // ref - rotfit
      const float r2 = dx * dx + dy * dy + dz * dz;
      const float E = ex2(nk * r2);
      float w = 1.f, c = 0.f;
      float4 rv = make_float4(0.f, 0.f, 0.f, 0.f);
      if (icat == 1 || icat == 2) {
        rv = sRV[i];
        if (ext) {
          w = EXT == 1 ? 1.f : 0.f;
          // extended points: (a_ref + v_ref) - (R (a_fit + v_fit) + t)
          const float gx = dx + rv.x - pv.x, gy = dy + rv.y - pv.y, gz = dz + rv.z - pv.z;
          const float KEe = iK * ex2(nk * (gx * gx + gy * gy + gz * gz));
          o += KEe;
          const float ae = ialpha * KEe;
          ex = fmaf(ae, gx, ex); ey = fmaf(ae, gy, ey); ez = fmaf(ae, gz, ez);
        } else {
          const float D = pv.x * rv.x + pv.y * rv.y + pv.z * rv.z;
          if (icat == 1) {
            const float Dc = fminf(fmaxf(D, 0.f), 1.f);
            w = (Dc + 2.f) * (1.f / 3.f);
            c = (D > 0.f && D < 1.f) ? 1.f : 0.f;
          } else {
            w = (fabsf(D) + 2.f) * (1.f / 3.f);
            c = D > 0.f ? 1.f : (D < 0.f ? -1.f : 0.f);
          }
        }
      }
      const float KE = iK * E;
      const float KwE = KE * w;
      o += KwE;
      const float a = ialpha * KwE;
      fx = fmaf(a, dx, fx); fy = fmaf(a, dy, fy); fz = fmaf(a, dz, fz);
      const float cf = (1.f / 3.f) * KE * c;
      wx = fmaf(cf, rv.x, wx); wy = fmaf(cf, rv.y, wy); wz = fmaf(cf, rv.z, wz);
    }
    acc.v += o;
    acc.add_force(fx, fy, fz, fa.x, fa.y, fa.z);
    if (ext) acc.add_force(ex, ey, ez, fa.x + fv.x, fa.y + fv.y, fa.z + fv.z);
    // weight force acts through the body-frame vector; it does not move t
    acc.g[0] = fmaf(wx, fv.x, acc.g[0]); acc.g[1] = fmaf(wx, fv.y, acc.g[1]);
    acc.g[2] = fmaf(wx, fv.z, acc.g[2]); acc.g[3] = fmaf(wy, fv.x, acc.g[3]);
    acc.g[4] = fmaf(wy, fv.y, acc.g[4]); acc.g[5] = fmaf(wy, fv.z, acc.g[5]);
    acc.g[6] = fmaf(wz, fv.x, acc.g[6]); acc.g[7] = fmaf(wz, fv.y, acc.g[7]);
    acc.g[8] = fmaf(wz, fv.z, acc.g[8]);
  }
}

// Unit vector with the reference's 1e-12 norm floor (cpu.py:524-526).
__device__ __forceinline__ float4 unit4(float x, float y, float z) {
  float n = sqrtf(x * x + y * y + z * z);
  const float inv = 1.f / (n > 1e-12f ? n : 1e-12f);
  return make_float4(x * inv, y * inv, z * inv, 0.f);
}

}  // namespace fss
