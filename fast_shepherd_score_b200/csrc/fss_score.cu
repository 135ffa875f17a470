// fss_score.cu -- differentiable Tanimoto scoring of packed cloud pairs: forward value and
// the hand-written adjoint with respect to every point coordinate and charge.
//
// score = V_AB / (V_AA + V_BB - V_AB) with V_XY = K sum_ij exp(-alpha/2 |x_i - y_j|^2)
// [* exp(-(c_i - c_j)^2 / lam) for ESP]: the functions get_overlap / get_overlap_esp
// (score/gaussian_overlap.py:62-117, score/electrostatic_scoring.py:17-120) whose gradients
// the reference obtains by torch autograd.  Here they are explicit:
//   d score/d V_AB = U / D^2,  d score/d V_AA = d score/d V_BB = -V_AB / D^2  (U = V_AA + V_BB,
//   D = U - V_AB);  d V_XY / d x_i = -alpha sum_j g_ij (x_i - y_j) (twice that for V_XX),
//   d V_XY / d c_i = -(2/lam) sum_j g_ij (c_i - c_j).
// The direct difference form is used (not the expanded exponent of the alignment kernels)
// so coordinate gradients keep full fp32 accuracy.  One CTA per pair, both clouds staged in
// shared memory; gradients are accumulated with atomics because a molecule may appear in
// several pairs (a fixed target scored against many queries).
#include <cmath>

#include "fss_internal.cuh"

namespace fss {
namespace {

constexpr int kScoreThreads = 128;

__device__ __forceinline__ float block_sum(float v, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  return s;
}

// sum_j g(x, y_j) for one point x against a staged cloud (value only)
template <bool ESP>
__device__ __forceinline__ float point_sum(float4 x, const float4* __restrict__ Y, int m,
                                           float nk, float ne) {
  float s = 0.f;
  for (int j = 0; j < m; ++j) {
    const float4 y = Y[j];
    const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
    float E = nk * (dx * dx + dy * dy + dz * dz);
    if (ESP) { const float dc = x.w - y.w; E = fmaf(ne * dc, dc, E); }
    s += ex2(E);
  }
  return s;
}

// gradient pieces for one point x: sum_j g (x - y_j) and sum_j g (c_x - c_j)
template <bool ESP>
__device__ __forceinline__ void point_grad(float4 x, const float4* __restrict__ Y, int m, float nk,
                                           float ne, float& gx, float& gy, float& gz, float& gc) {
  gx = gy = gz = gc = 0.f;
  for (int j = 0; j < m; ++j) {
    const float4 y = Y[j];
    const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
    float E = nk * (dx * dx + dy * dy + dz * dz);
    float dc = 0.f;
    if (ESP) { dc = x.w - y.w; E = fmaf(ne * dc, dc, E); }
    const float g = ex2(E);
    gx = fmaf(g, dx, gx); gy = fmaf(g, dy, gy); gz = fmaf(g, dz, gz);
    if (ESP) gc = fmaf(g, dc, gc);
  }
}

template <bool ESP>
__global__ void __launch_bounds__(kScoreThreads) score_fwd_kernel(
    const float4* __restrict__ rp, const int* __restrict__ roff, const float4* __restrict__ fp,
    const int* __restrict__ foff, const int* __restrict__ pr, const int* __restrict__ pf,
    int maxN, int maxM, float nk, float ne, float Kc, float* score, float* ov) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float red[32];
  const int p = blockIdx.x;
  const int ri = pr[p], fi = pf[p];
  const int n = roff[ri + 1] - roff[ri], m = foff[fi + 1] - foff[fi];
  if (n < 0 || m < 0 || n > maxN || m > maxM) {  // outside the staged tile: NaN, no access
    if (threadIdx.x == 0) {
      const float nan = __int_as_float(0x7fc00000);
      score[p] = nan; ov[3 * p] = nan; ov[3 * p + 1] = nan; ov[3 * p + 2] = nan;
    }
    return;
  }
  const float4* A = rp + roff[ri];
  const float4* B = fp + foff[fi];
  float4* sA = smem;
  float4* sB = smem + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sA[i] = A[i];
  for (int j = threadIdx.x; j < m; j += blockDim.x) sB[j] = B[j];
  __syncthreads();
  float ab = 0.f, aa = 0.f, bb = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    ab += point_sum<ESP>(sA[i], sB, m, nk, ne);
    aa += point_sum<ESP>(sA[i], sA, n, nk, ne);
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) bb += point_sum<ESP>(sB[j], sB, m, nk, ne);
  ab = block_sum(ab, red) * Kc;
  aa = block_sum(aa, red) * Kc;
  bb = block_sum(bb, red) * Kc;
  if (threadIdx.x == 0) {
    ov[3 * p] = ab; ov[3 * p + 1] = aa; ov[3 * p + 2] = bb;
    score[p] = ab / (aa + bb - ab);
  }
}

template <bool ESP>
__global__ void __launch_bounds__(kScoreThreads) score_bwd_kernel(
    const float4* __restrict__ rp, const int* __restrict__ roff, const float4* __restrict__ fp,
    const int* __restrict__ foff, const int* __restrict__ pr, const int* __restrict__ pf,
    int maxN, int maxM, float nk, float ne, float aKc, float cKc, const float* __restrict__ ov,
    const float* __restrict__ gs, float* gref, float* gfit) {
  extern __shared__ __align__(16) float4 smem[];
  const int p = blockIdx.x;
  const int ri = pr[p], fi = pf[p];
  const int r0 = roff[ri], f0 = foff[fi];
  const int n = roff[ri + 1] - r0, m = foff[fi + 1] - f0;
  if (n < 0 || m < 0 || n > maxN || m > maxM) return;
  float4* sA = smem;
  float4* sB = smem + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sA[i] = rp[r0 + i];
  for (int j = threadIdx.x; j < m; j += blockDim.x) sB[j] = fp[f0 + j];
  __syncthreads();
  const float vab = ov[3 * p], U = ov[3 * p + 1] + ov[3 * p + 2];
  const float D = U - vab;
  const float g = gs[p];
  const float dAB = g * U / (D * D);        // d loss / d V_AB
  const float dSelf = -g * vab / (D * D);   // d loss / d V_AA (= d / d V_BB)
  // d V_XY / d x = -alpha K sum g (x - y); self terms count twice
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float ax, ay, az, ac, sx, sy, sz, sc;
    point_grad<ESP>(sA[i], sB, m, nk, ne, ax, ay, az, ac);
    point_grad<ESP>(sA[i], sA, n, nk, ne, sx, sy, sz, sc);
    float* o = gref + 4 * (size_t)(r0 + i);
    atomicAdd(o + 0, -aKc * (dAB * ax + 2.f * dSelf * sx));
    atomicAdd(o + 1, -aKc * (dAB * ay + 2.f * dSelf * sy));
    atomicAdd(o + 2, -aKc * (dAB * az + 2.f * dSelf * sz));
    if (ESP) atomicAdd(o + 3, -cKc * (dAB * ac + 2.f * dSelf * sc));
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    float ax, ay, az, ac, sx, sy, sz, sc;
    point_grad<ESP>(sB[j], sA, n, nk, ne, ax, ay, az, ac);
    point_grad<ESP>(sB[j], sB, m, nk, ne, sx, sy, sz, sc);
    float* o = gfit + 4 * (size_t)(f0 + j);
    atomicAdd(o + 0, -aKc * (dAB * ax + 2.f * dSelf * sx));
    atomicAdd(o + 1, -aKc * (dAB * ay + 2.f * dSelf * sy));
    atomicAdd(o + 2, -aKc * (dAB * az + 2.f * dSelf * sz));
    if (ESP) atomicAdd(o + 3, -cKc * (dAB * ac + 2.f * dSelf * sc));
  }
}

}  // namespace

int score_fwd_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                     const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                     int P, int maxN, int maxM, float alpha, int esp, float inv_lam, float* score,
                     float* overlaps, cudaStream_t st) {
  if (P < 0 || maxN < 0 || maxM < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_fwd: bad sizes or alpha");
  if (maxN > kMaxPoints || maxM > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_score_fwd: more than fss_max_points() points");
  if (P == 0) return FSS_OK;
  if (!ref_pts || !ref_off || !fit_pts || !fit_off || !pair_ref || !pair_fit || !score || !overlaps)
    return set_error(FSS_ERR_INVALID, "fss_score_fwd: null pointer");
  const double a = alpha;
  const float nk = (float)(-0.5 * a * 1.4426950408889634);
  const float ne = esp ? (float)(-(double)inv_lam * 1.4426950408889634) : 0.f;
  const float Kc = (float)(std::pow(M_PI, 1.5) / std::pow(2.0 * a, 1.5));
  const size_t smem = sizeof(float4) * ((size_t)maxN + maxM) + 16;
  const float4* R = reinterpret_cast<const float4*>(ref_pts);
  const float4* F = reinterpret_cast<const float4*>(fit_pts);
  cudaError_t ce;
  if (esp) {
    ce = cudaFuncSetAttribute(score_fwd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      score_fwd_kernel<true><<<P, kScoreThreads, smem, st>>>(R, ref_off, F, fit_off, pair_ref, pair_fit,
                                                             maxN, maxM, nk, ne, Kc, score, overlaps);
  } else {
    ce = cudaFuncSetAttribute(score_fwd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      score_fwd_kernel<false><<<P, kScoreThreads, smem, st>>>(R, ref_off, F, fit_off, pair_ref, pair_fit,
                                                              maxN, maxM, nk, 0.f, Kc, score, overlaps);
  }
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_score_fwd: ") + cudaGetErrorString(ce));
  return check_launch("fss_score_fwd");
}

int score_bwd_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                     const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                     int P, int maxN, int maxM, float alpha, int esp, float inv_lam,
                     const float* overlaps, const float* grad_score, float* grad_ref,
                     float* grad_fit, cudaStream_t st) {
  if (P < 0 || maxN < 0 || maxM < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd: bad sizes or alpha");
  if (maxN > kMaxPoints || maxM > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_score_bwd: more than fss_max_points() points");
  if (P == 0) return FSS_OK;
  if (!ref_pts || !ref_off || !fit_pts || !fit_off || !pair_ref || !pair_fit || !overlaps ||
      !grad_score || !grad_ref || !grad_fit)
    return set_error(FSS_ERR_INVALID, "fss_score_bwd: null pointer");
  const double a = alpha;
  const float nk = (float)(-0.5 * a * 1.4426950408889634);
  const float ne = esp ? (float)(-(double)inv_lam * 1.4426950408889634) : 0.f;
  const double Kd = std::pow(M_PI, 1.5) / std::pow(2.0 * a, 1.5);
  const float aKc = (float)(a * Kd);
  const float cKc = (float)(2.0 * (double)inv_lam * Kd);
  const size_t smem = sizeof(float4) * ((size_t)maxN + maxM) + 16;
  const float4* R = reinterpret_cast<const float4*>(ref_pts);
  const float4* F = reinterpret_cast<const float4*>(fit_pts);
  cudaError_t ce;
  if (esp) {
    ce = cudaFuncSetAttribute(score_bwd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      score_bwd_kernel<true><<<P, kScoreThreads, smem, st>>>(R, ref_off, F, fit_off, pair_ref, pair_fit,
                                                             maxN, maxM, nk, ne, aKc, cKc, overlaps,
                                                             grad_score, grad_ref, grad_fit);
  } else {
    ce = cudaFuncSetAttribute(score_bwd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      score_bwd_kernel<false><<<P, kScoreThreads, smem, st>>>(R, ref_off, F, fit_off, pair_ref, pair_fit,
                                                              maxN, maxM, nk, 0.f, aKc, 0.f, overlaps,
                                                              grad_score, grad_ref, grad_fit);
  }
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_score_bwd: ") + cudaGetErrorString(ce));
  return check_launch("fss_score_bwd");
}

}  // namespace fss
