// fss_eval.cu -- single-evaluation kernels on the reference's padded (K, N_pad, 3) layout,
// and the per-step Tanimoto/Adam kernel.  These back the reference-compatible kernel API
// (overlap value + SE(3) gradient per pose) used by parity tests, the step-by-step
// (graph-capturable) driver and the one-launch-per-pair comparator.  The arithmetic is the
// same device code the fused kernel runs (fss_device.cuh).
#include <algorithm>
#include <cmath>

#include "fss_internal.cuh"

namespace fss {

template <bool ESP>
__global__ void __launch_bounds__(32) overlap_eval_kernel(
    const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ CA,
    const float* __restrict__ CB, const float* __restrict__ q, const float* __restrict__ t,
    const int* __restrict__ Nr, const int* __restrict__ Mr, int Npad, int Mpad, float k, float e,
    float inv2k, float Kc, float aKc, int need_grad, float* V, float* dQ, float* dT) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float red[96];
  const int row = blockIdx.x;
  const int N = Nr ? min(max(Nr[row], 0), Npad) : Npad;
  const int M = Mr ? min(max(Mr[row], 0), Mpad) : Mpad;
  float4* sP = smem;  // 2 * Npad (duplicated expanded reference)
  float4* sB = sP + 2 * Npad;
  float2* sQc = reinterpret_cast<float2*>(sB + Mpad);
  const float* a = A + (size_t)row * Npad * 3;
  const float* b = B + (size_t)row * Mpad * 3;
  // centroid of the real reference points
  float3 s = make_float3(0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    s.x += a[3 * i]; s.y += a[3 * i + 1]; s.z += a[3 * i + 2];
  }
  s = block_sum3(s, red);
  const float inv = 1.f / (float)(N > 0 ? N : 1);
  const float3 c = make_float3(s.x * inv, s.y * inv, s.z * inv);
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const float ax = a[3 * i] - c.x, ay = a[3 * i + 1] - c.y, az = a[3 * i + 2] - c.z;
    float w = -k * (ax * ax + ay * ay + az * az);
    if (ESP) {
      const float ci = CA[(size_t)row * Npad + i];
      w = fmaf(-e * ci, ci, w);
      sQc[i] = make_float2(2.f * e * ci, 2.f * e * ci);
    }
    const float px = 2.f * k * ax, py = 2.f * k * ay, pz = 2.f * k * az;
    sP[2 * i] = make_float4(px, px, py, py);
    sP[2 * i + 1] = make_float4(pz, pz, w, w);
  }
  for (int j = threadIdx.x; j < M; j += blockDim.x)
    sB[j] = make_float4(b[3 * j], b[3 * j + 1], b[3 * j + 2],
                        ESP ? CB[(size_t)row * Mpad + j] : 0.f);
  __syncthreads();
  float qq[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) qq[i] = q[(size_t)row * 4 + i];
  const Rot R = quat_to_rot(qq);
  Moments acc;
  acc.zero();
  shape_pose<32, ESP>(sP, sQc, sB, N, M, threadIdx.x, R, t[(size_t)row * 3] - c.x,
                      t[(size_t)row * 3 + 1] - c.y, t[(size_t)row * 3 + 2] - c.z, k, e, inv2k,
                      acc);
  acc.group_sum<32>();
  acc.scale(Kc, aKc);
  if (threadIdx.x == 0) {
    V[row] = acc.v;
    if (need_grad) {
      float d[4];
      quat_grad_from_moment(qq, acc.g, d);
#pragma unroll
      for (int i = 0; i < 4; ++i) dQ[(size_t)row * 4 + i] = d[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) dT[(size_t)row * 3 + i] = acc.f[i];
    }
  }
}

__global__ void __launch_bounds__(32) pharm_eval_kernel(
    const float* __restrict__ A, const float* __restrict__ B, const float* __restrict__ RV,
    const float* __restrict__ FV, const int* __restrict__ At, const int* __restrict__ Bt,
    const float* __restrict__ q, const float* __restrict__ t, const int* __restrict__ Nr,
    const int* __restrict__ Mr, int Npad, int Mpad, PharmTables tab, int need_grad, float* O,
    float* dQ, float* dT) {
  extern __shared__ __align__(16) float4 smem[];
  const int row = blockIdx.x;
  const int N = Nr ? min(max(Nr[row], 0), Npad) : Npad;
  const int M = Mr ? min(max(Mr[row], 0), Mpad) : Mpad;
  float4* sRA = smem;
  float4* sRV = sRA + Npad;
  float4* sFA = sRV + Npad;
  float4* sFV = sFA + Mpad;
  const float* a = A + (size_t)row * Npad * 3;
  const float* b = B + (size_t)row * Mpad * 3;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    int ty = At[(size_t)row * Npad + i];
    ty = (ty < 0 || ty > 8) ? 8 : ty;  // out-of-table types are treated as Dummy
    sRA[i] = make_float4(a[3 * i], a[3 * i + 1], a[3 * i + 2], __int_as_float(ty));
    sRV[i] = RV ? unit4(RV[((size_t)row * Npad + i) * 3], RV[((size_t)row * Npad + i) * 3 + 1],
                        RV[((size_t)row * Npad + i) * 3 + 2])
                : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    int ty = Bt[(size_t)row * Mpad + j];
    ty = (ty < 0 || ty > 8) ? 8 : ty;
    sFA[j] = make_float4(b[3 * j], b[3 * j + 1], b[3 * j + 2], __int_as_float(ty));
    sFV[j] = FV ? unit4(FV[((size_t)row * Mpad + j) * 3], FV[((size_t)row * Mpad + j) * 3 + 1],
                        FV[((size_t)row * Mpad + j) * 3 + 2])
                : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  float qq[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) qq[i] = q[(size_t)row * 4 + i];
  const Rot R = quat_to_rot(qq);
  Moments acc;
  acc.zero();
  pharm_pose<32>(sRA, sRV, sFA, sFV, N, M, threadIdx.x, R, t[(size_t)row * 3],
                 t[(size_t)row * 3 + 1], t[(size_t)row * 3 + 2], tab, acc);
  acc.group_sum<32>();
  if (threadIdx.x == 0) {
    O[row] = acc.v;
    if (need_grad) {
      float d[4];
      quat_grad_from_moment(qq, acc.g, d);
#pragma unroll
      for (int i = 0; i < 4; ++i) dQ[(size_t)row * 4 + i] = d[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) dT[(size_t)row * 3 + i] = acc.f[i];
    }
  }
}

__global__ void tanimoto_adam_kernel(const float* __restrict__ V, const float* __restrict__ dQ,
                                     const float* __restrict__ dT, const float* __restrict__ U,
                                     float* q, float* t, float* mq, float* vq, float* mt,
                                     float* vt, float* best, float* bq, float* bt, int K,
                                     float lr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= K) return;
  PoseState s;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    s.q[i] = q[(size_t)r * 4 + i]; s.mq[i] = mq[(size_t)r * 4 + i];
    s.vq[i] = vq[(size_t)r * 4 + i]; s.bq[i] = bq[(size_t)r * 4 + i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    s.t[i] = t[(size_t)r * 3 + i]; s.mt[i] = mt[(size_t)r * 3 + i];
    s.vt[i] = vt[(size_t)r * 3 + i]; s.bt[i] = bt[(size_t)r * 3 + i];
  }
  s.best = best[r];
  float score, scale;
  tanimoto(V[r], U[r], score, scale);
  float gq[4], gt[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) gq[i] = -scale * dQ[(size_t)r * 4 + i];
#pragma unroll
  for (int i = 0; i < 3; ++i) gt[i] = -scale * dT[(size_t)r * 3 + i];
  adam_tail(s, score, gq, gt, lr);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    q[(size_t)r * 4 + i] = s.q[i]; mq[(size_t)r * 4 + i] = s.mq[i];
    vq[(size_t)r * 4 + i] = s.vq[i]; bq[(size_t)r * 4 + i] = s.bq[i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    t[(size_t)r * 3 + i] = s.t[i]; mt[(size_t)r * 3 + i] = s.mt[i];
    vt[(size_t)r * 3 + i] = s.vt[i]; bt[(size_t)r * 3 + i] = s.bt[i];
  }
  best[r] = s.best;
}

int overlap_eval_launch(const float* A, const float* B, const float* CA, const float* CB,
                        const float* q, const float* t, const int32_t* Nr, const int32_t* Mr,
                        int K, int Npad, int Mpad, float alpha, float inv_lam, int need_grad,
                        float* V, float* dQ, float* dT, cudaStream_t st) {
  if (K < 0 || Npad < 0 || Mpad < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_overlap_grad: bad sizes or alpha");
  if (K == 0) return FSS_OK;
  if (!A || !B || !q || !t || !V || (need_grad && (!dQ || !dT)))
    return set_error(FSS_ERR_INVALID, "fss_overlap_grad: null pointer");
  if ((CA == nullptr) != (CB == nullptr))
    return set_error(FSS_ERR_INVALID, "fss_overlap_grad: give both charge arrays or neither");
  if (Npad > kMaxPoints || Mpad > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_overlap_grad: more than fss_max_points() points");
  const bool esp = CA != nullptr;
  const double a = alpha;
  const float k = (float)(0.5 * a * 1.4426950408889634);
  const float e = esp ? (float)((double)inv_lam * 1.4426950408889634) : 0.f;
  const float inv2k = (float)(1.0 / (a * 1.4426950408889634));
  const double Kd = std::pow(M_PI, 1.5) / std::pow(2.0 * a, 1.5);
  const size_t smem = sizeof(float4) * (2 * (size_t)Npad + Mpad) + sizeof(float2) * (size_t)Npad + 16;
  cudaError_t ce;
  if (esp) {
    ce = cudaFuncSetAttribute(overlap_eval_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      overlap_eval_kernel<true><<<K, 32, smem, st>>>(A, B, CA, CB, q, t, Nr, Mr, Npad, Mpad, k, e,
                                                     inv2k, (float)Kd, (float)(a * Kd), need_grad, V, dQ, dT);
  } else {
    ce = cudaFuncSetAttribute(overlap_eval_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      overlap_eval_kernel<false><<<K, 32, smem, st>>>(A, B, nullptr, nullptr, q, t, Nr, Mr, Npad,
                                                      Mpad, k, 0.f, inv2k, (float)Kd, (float)(a * Kd),
                                                      need_grad, V, dQ, dT);
  }
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_overlap_grad: ") + cudaGetErrorString(ce));
  return check_launch("fss_overlap_grad");
}

int pharm_eval_launch(const float* A, const float* B, const float* RV, const float* FV,
                      const int32_t* At, const int32_t* Bt, const float* q, const float* t,
                      const int32_t* Nr, const int32_t* Mr, int K, int Npad, int Mpad,
                      int directional, int need_grad, float* O, float* dQ, float* dT,
                      cudaStream_t st) {
  if (K < 0 || Npad < 0 || Mpad < 0) return set_error(FSS_ERR_INVALID, "fss_pharm_grad: bad sizes");
  if (K == 0) return FSS_OK;
  if (!A || !B || !At || !Bt || !q || !t || !O || (need_grad && (!dQ || !dT)))
    return set_error(FSS_ERR_INVALID, "fss_pharm_grad: null pointer");
  if (directional && (!RV || !FV))
    return set_error(FSS_ERR_INVALID, "fss_pharm_grad: directional scoring needs vectors");
  if (Npad > kMaxPoints || Mpad > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_pharm_grad: more than fss_max_points() features");
  const size_t smem = sizeof(float4) * 2 * ((size_t)Npad + Mpad) + 16;
  cudaError_t ce = cudaFuncSetAttribute(pharm_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_pharm_grad: ") + cudaGetErrorString(ce));
  pharm_eval_kernel<<<K, 32, smem, st>>>(A, B, directional ? RV : nullptr,
                                         directional ? FV : nullptr, At, Bt, q, t, Nr, Mr, Npad,
                                         Mpad, make_pharm_tables(directional != 0), need_grad, O,
                                         dQ, dT);
  return check_launch("fss_pharm_grad");
}

int tanimoto_adam_launch(const float* V, const float* dQ, const float* dT, const float* U,
                         float* q, float* t, float* mq, float* vq, float* mt, float* vt,
                         float* best, float* bq, float* bt, int K, float lr, cudaStream_t st) {
  if (K < 0) return set_error(FSS_ERR_INVALID, "fss_tanimoto_adam_step: K < 0");
  if (K == 0) return FSS_OK;
  if (!V || !dQ || !dT || !U || !q || !t || !mq || !vq || !mt || !vt || !best || !bq || !bt)
    return set_error(FSS_ERR_INVALID, "fss_tanimoto_adam_step: null pointer");
  tanimoto_adam_kernel<<<(K + 127) / 128, 128, 0, st>>>(V, dQ, dT, U, q, t, mq, vq, mt, vt,
                                                        best, bq, bt, K, lr);
  return check_launch("fss_tanimoto_adam_step");
}

}  // namespace fss
