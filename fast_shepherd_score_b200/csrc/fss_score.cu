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
// The two-pass kernels (score_fwd_kernel / score_bwd_kernel) use the direct difference form.
// The forward-with-moments kernel for batches with grad uses the factored exponent of the
// alignment kernels over clouds centred on the ref centroid (within 1e-5 of the fp64 oracle on
// scores and 1e-4 on gradients, like the direct form), falling back to the direct form for
// rows whose factor could overflow.  One CTA per pair, both clouds staged in shared memory;
// gradients are accumulated with atomics because a molecule may appear in several pairs (a
// fixed target scored against many queries).
#include <algorithm>
#include <cmath>

#include "fss_internal.cuh"

namespace fss {
namespace {

constexpr int kScoreMaxThreads = 256;
// The moments kernel: at most 5 warps per CTA and <= 56 registers, so 7 CTAs (one pair
// each) stay resident per SM -- 1036 pairs per wave on 148 SMs.
constexpr int kMomMaxThreads = 160;
constexpr int kMomMinBlocks = 7;

// Threads per pair: about two points of the larger cloud per thread (load balance of the
// thread-strided point loops), whole warps, 64..256.
int score_threads(int maxN, int maxM) {
  const int half = (std::max(maxN, maxM) + 1) / 2;
  const int t = ((half + 31) / 32) * 32;
  return std::min(kScoreMaxThreads, std::max(64, t));
}

// Block-wide sums of three values (fixed order: warp butterfly, then warps in index order).
// Threads per pair of the moments kernel: about two rows (points of the larger cloud) per
// thread, whole warps, 64..kMomMaxThreads.
int mom_threads(int maxN, int maxM) {
  const int half = (std::max(maxN, maxM) + 1) / 2;
  const int t = ((half + 31) / 32) * 32;
  return std::min(kMomMaxThreads, std::max(64, t));
}

__device__ __forceinline__ float3 block_sum3(float a, float b, float c, float3* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = make_float3(a, b, c);
  __syncthreads();
  float3 s = make_float3(0.f, 0.f, 0.f);
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
    s.x += red[i].x; s.y += red[i].y; s.z += red[i].z;
  }
  return s;
}

// sum_j g(x, y_j) for one point x against a staged cloud (value only).  Four independent
// partial sums (j mod 4) keep four ex2 in flight per thread instead of one serial chain;
// they are combined in a fixed order, so the result does not depend on the launch shape.
template <bool ESP>
__device__ __forceinline__ float point_sum(float4 x, const float4* __restrict__ Y, int m,
                                           float nk, float ne) {
  auto g = [&](int k) {
    const float4 y = Y[k];
    const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
    float E = nk * (dx * dx + dy * dy + dz * dz);
    if (ESP) { const float dc = x.w - y.w; E = fmaf(ne * dc, dc, E); }
    return ex2(E);
  };
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  int j = 0;
  for (; j + 4 <= m; j += 4) {
    s0 += g(j); s1 += g(j + 1); s2 += g(j + 2); s3 += g(j + 3);
  }
  // remainder with static accumulator indices (a runtime index would put them in local memory)
  if (j < m) s0 += g(j);
  if (j + 1 < m) s1 += g(j + 1);
  if (j + 2 < m) s2 += g(j + 2);
  return (s0 + s1) + (s2 + s3);
}

// Strict upper triangle of a self overlap, sum_{i<j} g(x_i, x_j), for the rows owned by
// thread slot `t` (0..blockDim-1).  Rows are taken in balanced pairs (r, n-1-r), n-1 terms
// per pair; the middle row of an odd cloud goes to slot n/2, which owns no pair.  The full
// self overlap is n (the diagonal, exactly ex2(0) = 1 per point) plus twice the block total
// of these sums.  The two clouds of a pair use slots counted from opposite ends of the block,
// so when their n/2 row pairs fill less than the block they land on different warps.
template <bool ESP>
__device__ __forceinline__ float self_upper(const float4* __restrict__ X, int n, int t, float nk,
                                            float ne) {
  float s = 0.f;
  for (int r = t; r < n / 2; r += blockDim.x)
    s += point_sum<ESP>(X[r], X + r + 1, n - 1 - r, nk, ne) +
         point_sum<ESP>(X[n - 1 - r], X + n - r, r, nk, ne);
  if ((n & 1) && t == (n / 2) % blockDim.x)
    s += point_sum<ESP>(X[n / 2], X + n / 2 + 1, n / 2, nk, ne);
  return s;
}

// gradient pieces for one point x: sum_j g (x - y_j) and sum_j g (c_x - c_j), with two
// independent partial sums (j mod 2) per component; returns sum_j g (callers that only need
// the moments let the compiler drop that accumulator)
template <bool ESP>
__device__ __forceinline__ float point_grad(float4 x, const float4* __restrict__ Y, int m,
                                            float nk, float ne, float& gx, float& gy, float& gz,
                                            float& gc) {
  float ax[2] = {0.f, 0.f}, ay[2] = {0.f, 0.f}, az[2] = {0.f, 0.f}, ac[2] = {0.f, 0.f};
  float as[2] = {0.f, 0.f};
  int j = 0;
  for (; j + 2 <= m; j += 2) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const float4 y = Y[j + u];
      const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
      float E = nk * (dx * dx + dy * dy + dz * dz);
      float dc = 0.f;
      if (ESP) { dc = x.w - y.w; E = fmaf(ne * dc, dc, E); }
      const float g = ex2(E);
      as[u] += g;
      ax[u] = fmaf(g, dx, ax[u]); ay[u] = fmaf(g, dy, ay[u]); az[u] = fmaf(g, dz, az[u]);
      if (ESP) ac[u] = fmaf(g, dc, ac[u]);
    }
  }
  if (j < m) {
    const float4 y = Y[j];
    const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
    float E = nk * (dx * dx + dy * dy + dz * dz);
    float dc = 0.f;
    if (ESP) { dc = x.w - y.w; E = fmaf(ne * dc, dc, E); }
    const float g = ex2(E);
    as[0] += g;
    ax[0] = fmaf(g, dx, ax[0]); ay[0] = fmaf(g, dy, ay[0]); az[0] = fmaf(g, dz, az[0]);
    if (ESP) ac[0] = fmaf(g, dc, ac[0]);
  }
  gx = ax[0] + ax[1]; gy = ay[0] + ay[1]; gz = az[0] + az[1]; gc = ac[0] + ac[1];
  return as[0] + as[1];
}

// Cloud sources: packed float4 clouds with prefix offsets, or the reference's dense padded
// batches (molecule b = points [b*n, (b+1)*n) of an (B, n, 3) array plus optional (B, n)
// charges, every point real).
struct PackedSrc {
  const float4* p;
  const int* off;
  __device__ __forceinline__ int begin(int mol) const { return off[mol]; }
  __device__ __forceinline__ int size(int mol) const { return off[mol + 1] - off[mol]; }
  __device__ __forceinline__ float4 load(int k) const { return p[k]; }
};

struct DenseSrc {
  const float* xyz;
  const float* q;
  int n;
  __device__ __forceinline__ int begin(int mol) const { return mol * n; }
  __device__ __forceinline__ int size(int) const { return n; }
  __device__ __forceinline__ float4 load(int k) const {
    return make_float4(xyz[3 * (size_t)k], xyz[3 * (size_t)k + 1], xyz[3 * (size_t)k + 2],
                       q ? q[k] : 0.f);
  }
};

// Gradient sinks matching the sources: float4 rows (w = d/d charge), or separate (., 3)
// coordinate and (.) charge arrays.  Atomic: a molecule may appear in several pairs.  A null
// sink (on() false) marks a side whose gradient is not wanted: its adjoint loop is skipped.
struct PackedSink {
  float* g;
  __device__ __forceinline__ bool on() const { return g != nullptr; }
  __device__ __forceinline__ void add(int k, float x, float y, float z, float c, bool esp) const {
    float* o = g + 4 * (size_t)k;
    atomicAdd(o + 0, x); atomicAdd(o + 1, y); atomicAdd(o + 2, z);
    if (esp) atomicAdd(o + 3, c);
  }
};

struct DenseSink {
  float* gxyz;
  float* gq;
  __device__ __forceinline__ bool on() const { return gxyz != nullptr; }
  __device__ __forceinline__ void add(int k, float x, float y, float z, float c, bool esp) const {
    float* o = gxyz + 3 * (size_t)k;
    atomicAdd(o + 0, x); atomicAdd(o + 1, y); atomicAdd(o + 2, z);
    if (esp && gq) atomicAdd(gq + k, c);
  }
  // plain stores, for a side whose every molecule row belongs to exactly one pair
  __device__ __forceinline__ void put(int k, float x, float y, float z, float c, bool esp) const {
    float* o = gxyz + 3 * (size_t)k;
    o[0] = x; o[1] = y; o[2] = z;
    if (esp && gq) gq[k] = c;
  }
};

template <bool ESP, class Src>
__global__ void __launch_bounds__(kScoreMaxThreads) score_fwd_kernel(
    const Src ref, const Src fit, const int* __restrict__ pr, const int* __restrict__ pf,
    int maxN, int maxM, float nk, float ne, float Kc, float* score, float* ov) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float3 red[kScoreMaxThreads / 32];
  const int p = blockIdx.x;
  const int ri = pr[p], fi = pf[p];
  const int n = ref.size(ri), m = fit.size(fi);
  if (n < 0 || m < 0 || n > maxN || m > maxM) {  // outside the staged tile: NaN, no access
    if (threadIdx.x == 0) {
      const float nan = __int_as_float(0x7fc00000);
      score[p] = nan; ov[3 * p] = nan; ov[3 * p + 1] = nan; ov[3 * p + 2] = nan;
    }
    return;
  }
  const int r0 = ref.begin(ri), f0 = fit.begin(fi);
  float4* sA = smem;
  float4* sB = smem + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sA[i] = ref.load(r0 + i);
  for (int j = threadIdx.x; j < m; j += blockDim.x) sB[j] = fit.load(f0 + j);
  __syncthreads();
  float ab = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) ab += point_sum<ESP>(sA[i], sB, m, nk, ne);
  const float3 t = block_sum3(ab, self_upper<ESP>(sA, n, threadIdx.x, nk, ne),
                              self_upper<ESP>(sB, m, blockDim.x - 1 - threadIdx.x, nk, ne), red);
  ab = t.x * Kc;
  const float aa = fmaf(2.f, t.y, (float)n) * Kc;
  const float bb = fmaf(2.f, t.z, (float)m) * Kc;
  if (threadIdx.x == 0) {
    ov[3 * p] = ab; ov[3 * p + 1] = aa; ov[3 * p + 2] = bb;
    score[p] = ab / (aa + bb - ab);
  }
}

template <bool ESP, class Src, class Sink>
__global__ void __launch_bounds__(kScoreMaxThreads) score_bwd_kernel(
    const Src ref, const Src fit, const int* __restrict__ pr, const int* __restrict__ pf,
    int maxN, int maxM, float nk, float ne, float aKc, float cKc, const float* __restrict__ ov,
    const float* __restrict__ gs, const Sink gref, const Sink gfit) {
  extern __shared__ __align__(16) float4 smem[];
  const int p = blockIdx.x;
  const int ri = pr[p], fi = pf[p];
  const int n = ref.size(ri), m = fit.size(fi);
  if (n < 0 || m < 0 || n > maxN || m > maxM) return;
  const int r0 = ref.begin(ri), f0 = fit.begin(fi);
  float4* sA = smem;
  float4* sB = smem + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sA[i] = ref.load(r0 + i);
  for (int j = threadIdx.x; j < m; j += blockDim.x) sB[j] = fit.load(f0 + j);
  __syncthreads();
  const float vab = ov[3 * p], U = ov[3 * p + 1] + ov[3 * p + 2];
  const float D = U - vab;
  const float g = gs[p];
  const float dAB = g * U / (D * D);        // d loss / d V_AB
  const float dSelf = -g * vab / (D * D);   // d loss / d V_AA (= d / d V_BB)
  // d V_XY / d x = -alpha K sum g (x - y); self terms count twice
  for (int i = gref.on() ? threadIdx.x : n; i < n; i += blockDim.x) {
    float ax, ay, az, ac, sx, sy, sz, sc;
    point_grad<ESP>(sA[i], sB, m, nk, ne, ax, ay, az, ac);
    point_grad<ESP>(sA[i], sA, n, nk, ne, sx, sy, sz, sc);
    gref.add(r0 + i, -aKc * (dAB * ax + 2.f * dSelf * sx), -aKc * (dAB * ay + 2.f * dSelf * sy),
             -aKc * (dAB * az + 2.f * dSelf * sz), -cKc * (dAB * ac + 2.f * dSelf * sc), ESP);
  }
  for (int j = gfit.on() ? threadIdx.x : m; j < m; j += blockDim.x) {
    float ax, ay, az, ac, sx, sy, sz, sc;
    point_grad<ESP>(sB[j], sA, n, nk, ne, ax, ay, az, ac);
    point_grad<ESP>(sB[j], sB, m, nk, ne, sx, sy, sz, sc);
    gfit.add(f0 + j, -aKc * (dAB * ax + 2.f * dSelf * sx), -aKc * (dAB * ay + 2.f * dSelf * sy),
             -aKc * (dAB * az + 2.f * dSelf * sz), -cKc * (dAB * ac + 2.f * dSelf * sc), ESP);
  }
}

// Factored staging of a (centred) cloud for the moment rows: with
//   E_jk = nk |b_j - y_k|^2 + ne (c_j - c_k)^2 = w_j + P_k . b_j + P_k.w + Q_k c_j,
//   w_j = nk |b_j|^2 + ne c_j^2,  P_k = -2 nk y_k,  P_k.w = nk |y_k|^2 + ne c_k^2,
//   Q_k = -2 ne c_k,
// a term costs 3 FFMA (+1 for the charge) instead of the direct form's 4 differences, 3 for
// the square and 2 more for the charge.  Points go in pairs (k, k+1) along the f32x2 lanes:
// F[2r] = (Px_k, Px_k+1, Py_k, Py_k+1), F[2r+1] = (Pz_k, Pz_k+1, Pw_k, Pw_k+1),
// Qp[r] = (Q_k, Q_k+1); an odd cloud's last pair has a dummy second point with Pw = -inf
// (its Gaussian is exactly 0).
__device__ __forceinline__ void stage_factored(const float4* __restrict__ X, int cnt, float nk,
                                               float ne, float4* __restrict__ F,
                                               float2* __restrict__ Qp) {
  for (int r = threadIdx.x; r < (cnt + 1) / 2; r += blockDim.x) {
    float px[2], py[2], pz[2], pw[2], q[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 2 * r + h;
      if (k < cnt) {
        const float4 y = X[k];
        px[h] = -2.f * nk * y.x; py[h] = -2.f * nk * y.y; pz[h] = -2.f * nk * y.z;
        pw[h] = fmaf(ne * y.w, y.w, nk * (y.x * y.x + y.y * y.y + y.z * y.z));
        q[h] = -2.f * ne * y.w;
      } else {
        px[h] = py[h] = pz[h] = q[h] = 0.f;
        pw[h] = -INFINITY;
      }
    }
    F[2 * r] = make_float4(px[0], px[1], py[0], py[1]);
    F[2 * r + 1] = make_float4(pz[0], pz[1], pw[0], pw[1]);
    Qp[r] = make_float2(q[0], q[1]);
  }
}

// One row b (centred, w = charge) against a factored cloud: S' = sum_k 2^(E_jk - w_j) and the
// raw sums sum_k 2^(E_jk - w_j) (P_k, Q_k), two points per f32x2 instruction.
template <bool ESP>
__device__ __forceinline__ void row_factored(float4 b, const float4* __restrict__ F,
                                             const float2* __restrict__ Qp, int npair, float& S,
                                             float& sx, float& sy, float& sz, float& sq) {
  const float2 z2 = make_float2(0.f, 0.f);
  const float2 bx = make_float2(b.x, b.x), by = make_float2(b.y, b.y),
               bz = make_float2(b.z, b.z), bc = make_float2(b.w, b.w);
  float2 s = z2, ax = z2, ay = z2, az = z2, aq = z2;
#pragma unroll 4
  for (int r = 0; r < npair; ++r) {
    const float4 f0 = F[2 * r], f1 = F[2 * r + 1];
    const float2 PX = make_float2(f0.x, f0.y), PY = make_float2(f0.z, f0.w),
                 PZ = make_float2(f1.x, f1.y), PW = make_float2(f1.z, f1.w);
    float2 E = __ffma2_rn(PX, bx, __ffma2_rn(PY, by, __ffma2_rn(PZ, bz, PW)));
    float2 Q = z2;
    if (ESP) {
      Q = Qp[r];
      E = __ffma2_rn(Q, bc, E);
    }
    const float2 g = make_float2(ex2(E.x), ex2(E.y));
    s = __fadd2_rn(s, g);
    ax = __ffma2_rn(g, PX, ax);
    ay = __ffma2_rn(g, PY, ay);
    az = __ffma2_rn(g, PZ, az);
    if (ESP) aq = __ffma2_rn(g, Q, aq);
  }
  S = s.x + s.y; sx = ax.x + ax.y; sy = ay.x + ay.y; sz = az.x + az.y; sq = aq.x + aq.y;
}

// Upper-triangle row of a self overlap, sum_{k > r} g(x_r, x_k), against the cloud's own
// factored pairs: value only, 5 FP32 lane-ops a term (3 + 1 FFMA and the running sum) instead
// of the direct form's 11.  An odd first index takes one direct term so the packed loop starts
// on a pair boundary; a row beyond the factor bound takes the direct form throughout.
template <bool ESP>
__device__ __forceinline__ float upper_row(const float4* __restrict__ X, int n, int r,
                                           const float4* __restrict__ F,
                                           const float2* __restrict__ Qp, float nk, float ne) {
  const float4 b = X[r];
  float w = nk * (b.x * b.x + b.y * b.y + b.z * b.z);
  if (ESP) w = fmaf(ne * b.w, b.w, w);
  int k = r + 1;
  if (k >= n) return 0.f;   // the last row has no later points (and pair k/2 would hold r)
  if (-w > kFactorMax) return point_sum<ESP>(b, X + k, n - k, nk, ne);
  float S = 0.f;
  if (k & 1) {   // scaled like the packed terms: 2^(E - w)
    const float4 y = X[k];
    const float dx = b.x - y.x, dy = b.y - y.y, dz = b.z - y.z;
    float E = nk * (dx * dx + dy * dy + dz * dz);
    if (ESP) { const float dc = b.w - y.w; E = fmaf(ne * dc, dc, E); }
    S = ex2(E - w);
    ++k;
  }
  const float2 z2 = make_float2(0.f, 0.f);
  const float2 bx = make_float2(b.x, b.x), by = make_float2(b.y, b.y),
               bz = make_float2(b.z, b.z), bc = make_float2(b.w, b.w);
  float2 s = z2;
#pragma unroll 4
  for (int q = k / 2; q < (n + 1) / 2; ++q) {
    const float4 f0 = F[2 * q], f1 = F[2 * q + 1];
    float2 E = __ffma2_rn(make_float2(f0.x, f0.y), bx,
                          __ffma2_rn(make_float2(f0.z, f0.w), by,
                                     __ffma2_rn(make_float2(f1.x, f1.y), bz,
                                                make_float2(f1.z, f1.w))));
    if (ESP) E = __ffma2_rn(Qp[q], bc, E);
    s = __fadd2_rn(s, make_float2(ex2(E.x), ex2(E.y)));
  }
  return ex2(w) * (S + (s.x + s.y));
}

// Full row against another cloud's factored pairs, value only: sum_k g(b, y_k) (direct form
// beyond the factor bound).
template <bool ESP>
__device__ __forceinline__ float cross_row(float4 b, const float4* __restrict__ Y, int cnt,
                                           const float4* __restrict__ F,
                                           const float2* __restrict__ Qp, float nk, float ne) {
  float w = nk * (b.x * b.x + b.y * b.y + b.z * b.z);
  if (ESP) w = fmaf(ne * b.w, b.w, w);
  if (-w > kFactorMax) return point_sum<ESP>(b, Y, cnt, nk, ne);
  const float2 bx = make_float2(b.x, b.x), by = make_float2(b.y, b.y),
               bz = make_float2(b.z, b.z), bc = make_float2(b.w, b.w);
  float2 s = make_float2(0.f, 0.f);
#pragma unroll 4
  for (int q = 0; q < (cnt + 1) / 2; ++q) {
    const float4 f0 = F[2 * q], f1 = F[2 * q + 1];
    float2 E = __ffma2_rn(make_float2(f0.x, f0.y), bx,
                          __ffma2_rn(make_float2(f0.z, f0.w), by,
                                     __ffma2_rn(make_float2(f1.x, f1.y), bz,
                                                make_float2(f1.z, f1.w))));
    if (ESP) E = __ffma2_rn(Qp[q], bc, E);
    s = __fadd2_rn(s, make_float2(ex2(E.x), ex2(E.y)));
  }
  return ex2(w) * (s.x + s.y);
}

// Strict upper triangle of a self overlap from the factored pairs, rows in balanced pairs
// (r, n-1-r) owned by thread slot t, as self_upper.
template <bool ESP>
__device__ __forceinline__ float self_upper_factored(const float4* __restrict__ X, int n, int t,
                                                     const float4* __restrict__ F,
                                                     const float2* __restrict__ Qp, float nk,
                                                     float ne) {
  float s = 0.f;
  for (int r = t; r < n / 2; r += blockDim.x)
    s += upper_row<ESP>(X, n, r, F, Qp, nk, ne) + upper_row<ESP>(X, n, n - 1 - r, F, Qp, nk, ne);
  if ((n & 1) && t == (n / 2) % blockDim.x) s += upper_row<ESP>(X, n, n / 2, F, Qp, nk, ne);
  return s;
}

// Moments of one row against one cloud: returns sum_k g and writes the float4
// sum_k g (b - y_k, c_b - c_k).  Factored (two points per packed instruction) unless the
// row's factor 2^(-w_j) could overflow, then the direct form (point_grad on the plain cloud).
template <bool ESP>
__device__ __forceinline__ float row_moments(float4 b, float w, bool direct,
                                             const float4* __restrict__ Xp, int cnt,
                                             const float4* __restrict__ F,
                                             const float2* __restrict__ Qp, float nk, float ne,
                                             float inv2nk, float inv2ne, float& mx,
                                             float& my, float& mz, float& mq) {
  if (direct) return point_grad<ESP>(b, Xp, cnt, nk, ne, mx, my, mz, mq);
  float S, sx, sy, sz, sq;
  row_factored<ESP>(b, F, Qp, (cnt + 1) / 2, S, sx, sy, sz, sq);
  // sum g (b - y) = 2^w (b S' - sum g' y), y = P / (-2 nk); likewise the charges
  const float scale = ex2(w);
  mx = scale * fmaf(sx, inv2nk, b.x * S);
  my = scale * fmaf(sy, inv2nk, b.y * S);
  mz = scale * fmaf(sz, inv2nk, b.z * S);
  mq = ESP ? scale * fmaf(sq, inv2ne, b.w * S) : 0.f;
  return scale * S;
}

// Rows of cloud X with moments against the other cloud and itself; adds the rows' Gaussian
// sums to cross / self and writes the two moment rows of each point of pair p.
template <bool ESP>
__device__ __forceinline__ void moment_rows(const float4* __restrict__ X, int cnt,
                                            const float4* __restrict__ Fx,
                                            const float2* __restrict__ Qx,
                                            const float4* __restrict__ O, int n_other,
                                            const float4* __restrict__ Fo,
                                            const float2* __restrict__ Qo, float nk, float ne,
                                            float inv2nk, float inv2ne, float4* __restrict__ mom,
                                            float& cross, float& self) {
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    const float4 b = X[j];
    float w = nk * (b.x * b.x + b.y * b.y + b.z * b.z);
    if (ESP) w = fmaf(ne * b.w, b.w, w);
    const bool direct = -w > kFactorMax;
    float mx, my, mz, mq;
    cross += row_moments<ESP>(b, w, direct, O, n_other, Fo, Qo, nk, ne, inv2nk, inv2ne, mx, my,
                              mz, mq);
    mom[2 * j] = make_float4(mx, my, mz, mq);
    self += row_moments<ESP>(b, w, direct, X, cnt, Fx, Qx, nk, ne, inv2nk, inv2ne, mx, my, mz,
                             mq);
    mom[2 * j + 1] = make_float4(mx, my, mz, mq);
  }
}

// Forward with adjoint moments.  For a side whose moments are wanted (MR: ref, MF: fit) every
// point k of pair p gets two float4 rows, mom[2(p*size + k)] = sum over the other cloud of
// g (x_k - y) and mom[2(p*size + k) + 1] = the same over its own cloud (w = the charge
// differences).  The pair's overlaps come out of the same passes (V_AB from the fit rows when
// MF, V_XX from the full rows of a side with moments, the upper triangle otherwise), so the
// backward is one elementwise step and the Gaussians are evaluated once per step instead of
// twice.  Both clouds are moved to the ref centroid (the score and every difference are
// translation invariant) so the factored rows stay inside their overflow bound.  Shared
// memory per point: plain float4 (16 B) + factored half-pairs (20 B).
template <bool ESP, bool MR, bool MF>
__global__ void __launch_bounds__(kMomMaxThreads, kMomMinBlocks) score_fwd_mom_kernel(
    const DenseSrc ref, const DenseSrc fit, const int* __restrict__ pr,
    const int* __restrict__ pf, float nk, float ne, float Kc, float inv2nk, float inv2ne,
    float* score, float* ov, float4* __restrict__ momR, float4* __restrict__ momF) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float3 red[kScoreMaxThreads / 32];
  const int p = blockIdx.x;
  const int n = ref.n, m = fit.n;
  const int hn = (n + 1) / 2, hm = (m + 1) / 2;
  const int r0 = ref.begin(pr[p]), f0 = fit.begin(pf[p]);
  float4* sA = smem;
  float4* sB = sA + n;
  float4* fA = sB + m;
  float4* fB = fA + 2 * hn;
  float2* qA = reinterpret_cast<float2*>(fB + 2 * hm);
  float2* qB = qA + hn;
  float cx = 0.f, cy = 0.f, cz = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 v = ref.load(r0 + i);
    sA[i] = v;
    cx += v.x; cy += v.y; cz += v.z;
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) sB[j] = fit.load(f0 + j);
  const float3 c = block_sum3(cx, cy, cz, red);   // includes the barrier after the loads
  const float inv_n = n > 0 ? 1.f / (float)n : 0.f;
  const float ox = c.x * inv_n, oy = c.y * inv_n, oz = c.z * inv_n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 v = sA[i];
    sA[i] = make_float4(v.x - ox, v.y - oy, v.z - oz, v.w);
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const float4 v = sB[j];
    sB[j] = make_float4(v.x - ox, v.y - oy, v.z - oz, v.w);
  }
  __syncthreads();
  stage_factored(sA, n, nk, ESP ? ne : 0.f, fA, qA);
  stage_factored(sB, m, nk, ESP ? ne : 0.f, fB, qB);
  __syncthreads();
  float ab = 0.f, aa = 0.f, bb = 0.f;
  if (MF) {
    moment_rows<ESP>(sB, m, fB, qB, sA, n, fA, qA, nk, ne, inv2nk, inv2ne,
                     momF + 2 * (size_t)p * m, ab, bb);
  } else {
    bb = self_upper_factored<ESP>(sB, m, blockDim.x - 1 - threadIdx.x, fB, qB, nk, ne);
  }
  if (MR) {
    float abr = 0.f;
    moment_rows<ESP>(sA, n, fA, qA, sB, m, fB, qB, nk, ne, inv2nk, inv2ne,
                     momR + 2 * (size_t)p * n, abr, aa);
    if (!MF) ab = abr;
  } else {
    // counted from the far end of the block: the fit rows fill it from thread 0
    aa = self_upper_factored<ESP>(sA, n, blockDim.x - 1 - threadIdx.x, fA, qA, nk, ne);
  }
  if (!MR && !MF) {   // value only: the cross term from the fit rows
    for (int j = threadIdx.x; j < m; j += blockDim.x)
      ab += cross_row<ESP>(sB[j], sA, n, fA, qA, nk, ne);
  }
  __syncthreads();   // red is reused
  const float3 t = block_sum3(ab, aa, bb, red);
  const float vab = t.x * Kc;
  const float vaa = (MR ? t.y : fmaf(2.f, t.y, (float)n)) * Kc;
  const float vbb = (MF ? t.z : fmaf(2.f, t.z, (float)m)) * Kc;
  if (threadIdx.x == 0) {
    ov[3 * p] = vab; ov[3 * p + 1] = vaa; ov[3 * p + 2] = vbb;
    score[p] = vab / (vaa + vbb - vab);
  }
}

// Backward from the moments: one thread per (pair, point) of each side with moments; the
// same chain rule and the same expressions as score_bwd_kernel, added atomically into the
// molecule's row (a broadcast molecule is shared by every pair), or stored for a side whose
// bit is set in `overwrite` (bit 0 ref, bit 1 fit: each row belongs to one pair).
__global__ void score_bwd_mom_kernel(const int* __restrict__ pr, const int* __restrict__ pf,
                                     int P, int n, int m, float aKc, float cKc, int esp,
                                     int overwrite,
                                     const float* __restrict__ ov, const float* __restrict__ gs,
                                     const float4* __restrict__ momR,
                                     const float4* __restrict__ momF, const DenseSink gR,
                                     const DenseSink gF) {
  const long long nR = momR ? (long long)P * n : 0;
  const long long nT = nR + (momF ? (long long)P * m : 0);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nT;
       t += (long long)gridDim.x * blockDim.x) {
    const bool isR = t < nR;
    const long long u = isR ? t : t - nR;
    const int cnt = isR ? n : m;
    const int p = (int)(u / cnt), k = (int)(u - (long long)p * cnt);
    const float vab = ov[3 * p], U = ov[3 * p + 1] + ov[3 * p + 2];
    const float D = U - vab;
    const float g = gs[p];
    const float dAB = g * U / (D * D);
    const float dSelf = -g * vab / (D * D);
    const float4* mom = (isR ? momR : momF) + 2 * u;
    const float4 c = mom[0], o = mom[1];
    const int row = (isR ? pr[p] : pf[p]) * cnt + k;
    const DenseSink sink{isR ? gR.gxyz : gF.gxyz, isR ? gR.gq : gF.gq};
    const float gx = -aKc * (dAB * c.x + 2.f * dSelf * o.x);
    const float gy = -aKc * (dAB * c.y + 2.f * dSelf * o.y);
    const float gz = -aKc * (dAB * c.z + 2.f * dSelf * o.z);
    const float gc = -cKc * (dAB * c.w + 2.f * dSelf * o.w);
    if ((overwrite >> (isR ? 0 : 1)) & 1) sink.put(row, gx, gy, gz, gc, esp != 0);
    else sink.add(row, gx, gy, gz, gc, esp != 0);
  }
}

struct ScoreConsts {
  float nk, ne, Kc, aKc, cKc;
};

ScoreConsts score_consts(float alpha, int esp, float inv_lam) {
  const double a = alpha;
  const double Kd = std::pow(M_PI, 1.5) / std::pow(2.0 * a, 1.5);
  ScoreConsts c;
  c.nk = (float)(-0.5 * a * 1.4426950408889634);
  c.ne = esp ? (float)(-(double)inv_lam * 1.4426950408889634) : 0.f;
  c.Kc = (float)Kd;
  c.aKc = (float)(a * Kd);
  c.cKc = esp ? (float)(2.0 * (double)inv_lam * Kd) : 0.f;
  return c;
}

template <class Src>
int fwd_dispatch(const Src& R, const Src& F, const int32_t* pr, const int32_t* pf, int P,
                 int maxN, int maxM, float alpha, int esp, float inv_lam, float* score,
                 float* overlaps, cudaStream_t st) {
  const ScoreConsts c = score_consts(alpha, esp, inv_lam);
  const size_t smem = sizeof(float4) * ((size_t)maxN + maxM) + 16;
  auto kern = esp ? score_fwd_kernel<true, Src> : score_fwd_kernel<false, Src>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_score_fwd: ") + cudaGetErrorString(ce));
  kern<<<P, score_threads(maxN, maxM), smem, st>>>(R, F, pr, pf, maxN, maxM, c.nk, c.ne, c.Kc,
                                                   score, overlaps);
  return check_launch("fss_score_fwd");
}

template <class Src, class Sink>
int bwd_dispatch(const Src& R, const Src& F, const int32_t* pr, const int32_t* pf, int P,
                 int maxN, int maxM, float alpha, int esp, float inv_lam, const float* overlaps,
                 const float* grad_score, const Sink& gR, const Sink& gF, cudaStream_t st) {
  const ScoreConsts c = score_consts(alpha, esp, inv_lam);
  const size_t smem = sizeof(float4) * ((size_t)maxN + maxM) + 16;
  auto kern = esp ? score_bwd_kernel<true, Src, Sink> : score_bwd_kernel<false, Src, Sink>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_score_bwd: ") + cudaGetErrorString(ce));
  kern<<<P, score_threads(maxN, maxM), smem, st>>>(R, F, pr, pf, maxN, maxM, c.nk, c.ne, c.aKc,
                                                   c.cKc, overlaps, grad_score, gR, gF);
  return check_launch("fss_score_bwd");
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
  const PackedSrc R{reinterpret_cast<const float4*>(ref_pts), ref_off};
  const PackedSrc F{reinterpret_cast<const float4*>(fit_pts), fit_off};
  return fwd_dispatch(R, F, pair_ref, pair_fit, P, maxN, maxM, alpha, esp, inv_lam, score,
                      overlaps, st);
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
      !grad_score || (!grad_ref && !grad_fit))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd: null pointer");
  const PackedSrc R{reinterpret_cast<const float4*>(ref_pts), ref_off};
  const PackedSrc F{reinterpret_cast<const float4*>(fit_pts), fit_off};
  return bwd_dispatch(R, F, pair_ref, pair_fit, P, maxN, maxM, alpha, esp, inv_lam, overlaps,
                      grad_score, PackedSink{grad_ref}, PackedSink{grad_fit}, st);
}

int score_fwd_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                           const float* fit_xyz, const float* fit_q, int fit_n,
                           const int32_t* pair_ref, const int32_t* pair_fit, int P, float alpha,
                           int esp, float inv_lam, float* score, float* overlaps,
                           cudaStream_t st) {
  if (P < 0 || ref_n < 0 || fit_n < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_fwd_dense: bad sizes or alpha");
  if (ref_n > kMaxPoints || fit_n > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_score_fwd_dense: more than fss_max_points() points");
  if (P == 0) return FSS_OK;
  if (!ref_xyz || !fit_xyz || !pair_ref || !pair_fit || !score || !overlaps ||
      (esp && (!ref_q || !fit_q)))
    return set_error(FSS_ERR_INVALID, "fss_score_fwd_dense: null pointer");
  return fwd_dispatch(DenseSrc{ref_xyz, esp ? ref_q : nullptr, ref_n},
                      DenseSrc{fit_xyz, esp ? fit_q : nullptr, fit_n}, pair_ref, pair_fit, P,
                      ref_n, fit_n, alpha, esp, inv_lam, score, overlaps, st);
}

int score_bwd_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                           const float* fit_xyz, const float* fit_q, int fit_n,
                           const int32_t* pair_ref, const int32_t* pair_fit, int P, float alpha,
                           int esp, float inv_lam, const float* overlaps, const float* grad_score,
                           float* grad_ref_xyz, float* grad_ref_q, float* grad_fit_xyz,
                           float* grad_fit_q, cudaStream_t st) {
  if (P < 0 || ref_n < 0 || fit_n < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd_dense: bad sizes or alpha");
  if (ref_n > kMaxPoints || fit_n > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_score_bwd_dense: more than fss_max_points() points");
  if (P == 0) return FSS_OK;
  if (!ref_xyz || !fit_xyz || !pair_ref || !pair_fit || !overlaps || !grad_score ||
      (!grad_ref_xyz && !grad_fit_xyz) || (esp && (!ref_q || !fit_q)))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd_dense: null pointer");
  return bwd_dispatch(DenseSrc{ref_xyz, esp ? ref_q : nullptr, ref_n},
                      DenseSrc{fit_xyz, esp ? fit_q : nullptr, fit_n}, pair_ref, pair_fit, P,
                      ref_n, fit_n, alpha, esp, inv_lam, overlaps, grad_score,
                      DenseSink{grad_ref_xyz, grad_ref_q}, DenseSink{grad_fit_xyz, grad_fit_q},
                      st);
}


int score_fwd_mom_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                               const float* fit_xyz, const float* fit_q, int fit_n,
                               const int32_t* pair_ref, const int32_t* pair_fit, int P,
                               float alpha, int esp, float inv_lam, float* score, float* overlaps,
                               float* ref_mom, float* fit_mom, cudaStream_t st) {
  if (P < 0 || ref_n < 0 || fit_n < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_fwd_moments_dense: bad sizes or alpha");
  if (ref_n > kMaxPoints || fit_n > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED,
                     "fss_score_fwd_moments_dense: more than fss_max_points() points");
  if (P == 0) return FSS_OK;
  if (!ref_xyz || !fit_xyz || !pair_ref || !pair_fit || !score || !overlaps ||
      (esp && (!ref_q || !fit_q)))
    return set_error(FSS_ERR_INVALID, "fss_score_fwd_moments_dense: null pointer");
  const ScoreConsts c = score_consts(alpha, esp, inv_lam);
  // plain (16 bytes a point) + factored half-pairs (2 float4 + 1 float2 per two points) of
  // both clouds: clouds whose sum exceeds the per-CTA shared memory (about 6000 points) take
  // the two-pass form instead
  const size_t hn = ((size_t)ref_n + 1) / 2, hm = ((size_t)fit_n + 1) / 2;
  const size_t smem = sizeof(float4) * ((size_t)ref_n + fit_n + 2 * (hn + hm)) +
                      sizeof(float2) * (hn + hm) + 16;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return set_error(FSS_ERR_CUDA, "fss_score_fwd_moments_dense: device query failed");
  if (smem > (size_t)optin)
    return set_error(FSS_ERR_UNSUPPORTED,
                     "fss_score_fwd_moments_dense: clouds too large for the staged moments "
                     "kernel; use fss_score_fwd_dense + fss_score_bwd_dense");
  // 1/(2 nk), 1/(2 ne): the factored rows' sums of g P and g Q back to sums of g y and g c
  const float inv2nk = (float)(0.5 / (double)c.nk);
  const float inv2ne = (esp && c.ne < 0.f) ? (float)(0.5 / (double)c.ne) : 0.f;
  using K = void (*)(const DenseSrc, const DenseSrc, const int*, const int*, float, float, float,
                     float, float, float*, float*, float4*, float4*);
  const K table[2][4] = {
      {score_fwd_mom_kernel<false, true, false>, score_fwd_mom_kernel<false, false, true>,
       score_fwd_mom_kernel<false, true, true>, score_fwd_mom_kernel<false, false, false>},
      {score_fwd_mom_kernel<true, true, false>, score_fwd_mom_kernel<true, false, true>,
       score_fwd_mom_kernel<true, true, true>, score_fwd_mom_kernel<true, false, false>}};
  const K kern = table[esp ? 1 : 0][ref_mom ? (fit_mom ? 2 : 0) : (fit_mom ? 1 : 3)];
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  // all of the unified L1 as shared memory: 7 CTAs of ~30 KB (300 + 300 points) per SM
  if (ce == cudaSuccess)
    ce = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                              (int)cudaSharedmemCarveoutMaxShared);
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_score_fwd_moments_dense: ") + cudaGetErrorString(ce));
  kern<<<P, mom_threads(ref_n, fit_n), smem, st>>>(
      DenseSrc{ref_xyz, esp ? ref_q : nullptr, ref_n}, DenseSrc{fit_xyz, esp ? fit_q : nullptr, fit_n},
      pair_ref, pair_fit, c.nk, c.ne, c.Kc, inv2nk, inv2ne, score, overlaps,
      reinterpret_cast<float4*>(ref_mom),
      reinterpret_cast<float4*>(fit_mom));
  return check_launch("fss_score_fwd_moments_dense");
}

int score_bwd_mom_dense_launch(const int32_t* pair_ref, const int32_t* pair_fit, int P,
                               int ref_n, int fit_n, float alpha, int esp, float inv_lam,
                               const float* overlaps, const float* grad_score,
                               const float* ref_mom, const float* fit_mom, float* grad_ref_xyz,
                               float* grad_ref_q, float* grad_fit_xyz, float* grad_fit_q,
                               int overwrite, cudaStream_t st) {
  if (P < 0 || ref_n < 0 || fit_n < 0 || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd_moments_dense: bad sizes or alpha");
  if (P == 0) return FSS_OK;
  // a side takes part when both its moments and its gradient are given
  if (!grad_ref_xyz) ref_mom = nullptr;
  if (!grad_fit_xyz) fit_mom = nullptr;
  if (!pair_ref || !pair_fit || !overlaps || !grad_score || (!ref_mom && !fit_mom))
    return set_error(FSS_ERR_INVALID, "fss_score_bwd_moments_dense: null pointer");
  const ScoreConsts c = score_consts(alpha, esp, inv_lam);
  const long long total = (ref_mom ? (long long)P * ref_n : 0) + (fit_mom ? (long long)P * fit_n : 0);
  if (total == 0) return FSS_OK;
  const long long want = (total + 255) / 256;
  const int grid = (int)std::min<long long>(want, (long long)num_sms() * 8);
  score_bwd_mom_kernel<<<grid, 256, 0, st>>>(
      pair_ref, pair_fit, P, ref_n, fit_n, c.aKc, c.cKc, esp, overwrite & 3, overlaps, grad_score,
      reinterpret_cast<const float4*>(ref_mom), reinterpret_cast<const float4*>(fit_mom),
      DenseSink{grad_ref_xyz, grad_ref_q}, DenseSink{grad_fit_xyz, grad_fit_q});
  return check_launch("fss_score_bwd_moments_dense");
}

}  // namespace fss
