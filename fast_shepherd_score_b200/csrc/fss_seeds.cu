// fss_seeds.cu -- multi-start seed poses for a batch of pairs, one thread per pair.
//
// Restates batched_seeds_torch (shepherd_score/accel/drivers/_common.py:281-441):
//   identity, 4 principal-axis alignments (ref axes with the sign flips of :358-362; the
//   fit axis-0 then axis-1 alignment of :369-390), up to 6 structured +-90 degree rotations
//   about the ref axes composed onto the first PCA seed (:401-413), then a Fibonacci fill
//   (given by the caller), every seed with the COM-aligning translation of :425-428, and the
//   fixed fallback rotations for pairs with < 3 points or non-finite coordinates (:430-439).
// The PCA runs in fp64 with the closed-form symmetric 3x3 eigensolver of :207-255.  The
// second fit-axis PCA of the reference is taken on the rotated fit cloud; its inertia tensor
// is R0 I R0^T exactly, so it is formed that way instead of re-reading the points.
#include <cmath>

#include "fss_internal.cuh"

namespace fss {
namespace {

struct M3 {
  double m[3][3];
};

__device__ void sym3x3_axes(const M3& A, M3& out) {
  const double eps = 1e-12;
  const double a00 = A.m[0][0], a11 = A.m[1][1], a22 = A.m[2][2];
  const double a01 = A.m[0][1], a02 = A.m[0][2], a12 = A.m[1][2];
  const double q = (a00 + a11 + a22) / 3.0;
  const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
  const double p2 = (a00 - q) * (a00 - q) + (a11 - q) * (a11 - q) + (a22 - q) * (a22 - q) + 2.0 * p1;
  const double p = sqrt(fmax(p2 / 6.0, eps));
  const double ip = 1.0 / p;
  const double b00 = (a00 - q) * ip, b11 = (a11 - q) * ip, b22 = (a22 - q) * ip;
  const double b01 = a01 * ip, b02 = a02 * ip, b12 = a12 * ip;
  const double detB = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                      b02 * (b01 * b12 - b11 * b02);
  const double r = fmin(fmax(detB * 0.5, -1.0), 1.0);
  const double phi = acos(r) / 3.0;
  const double e1 = q + 2.0 * p * cos(phi);
  const double e3 = q + 2.0 * p * cos(phi + 2.0 * M_PI / 3.0);
  const double e2 = 3.0 * q - e1 - e3;
  auto evec = [&](double lj, double lk, double v[3]) -> double {
    double X[3][3], Y[3][3], P[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        X[i][j] = A.m[i][j] - (i == j ? lj : 0.0);
        Y[i][j] = A.m[i][j] - (i == j ? lk : 0.0);
      }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        P[i][j] = X[i][0] * Y[0][j] + X[i][1] * Y[1][j] + X[i][2] * Y[2][j];
    int idx = 0;
    double best = -1.0;
    for (int j = 0; j < 3; ++j) {  // max-norm column, first index on ties
      const double n = sqrt(P[0][j] * P[0][j] + P[1][j] * P[1][j] + P[2][j] * P[2][j]);
      if (n > best) { best = n; idx = j; }
    }
    const double nrm = best;
    const double inv = 1.0 / fmax(nrm, eps);
    for (int i = 0; i < 3; ++i) v[i] = P[i][idx] * inv;
    return nrm;
  };
  double v1[3], v2[3], v3[3];
  const double n1 = evec(e2, e3, v1);
  const double n3 = evec(e1, e2, v3);
  auto cross = [](const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  };
  auto normalize = [&](double v[3]) {
    const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double inv = 1.0 / fmax(n, eps);
    v[0] *= inv; v[1] *= inv; v[2] *= inv;
  };
  cross(v3, v1, v2);
  normalize(v2);
  cross(v2, v3, v1);
  normalize(v1);
  bool bad = n1 < 1e-9 || n3 < 1e-9;
  for (int i = 0; i < 3; ++i)
    bad = bad || !isfinite(v1[i]) || !isfinite(v2[i]) || !isfinite(v3[i]);
  for (int i = 0; i < 3; ++i) {
    out.m[0][i] = bad ? (i == 0 ? 1.0 : 0.0) : v1[i];
    out.m[1][i] = bad ? (i == 1 ? 1.0 : 0.0) : v2[i];
    out.m[2][i] = bad ? (i == 2 ? 1.0 : 0.0) : v3[i];
  }
}

// Inertia tensor about the fp64 centroid of n points (_masked_principal_axes, :258-278).
__device__ void inertia(const Pts pts, int n, double shift_x, double shift_y,
                        double shift_z, M3& I) {
  double cx = 0, cy = 0, cz = 0;
  for (int i = 0; i < n; ++i) {
    const float4 p = pts[i];
    cx += (double)p.x - shift_x; cy += (double)p.y - shift_y; cz += (double)p.z - shift_z;
  }
  const double inv = 1.0 / (double)(n > 0 ? n : 1);
  cx *= inv; cy *= inv; cz *= inv;
  double s = 0, xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
  for (int i = 0; i < n; ++i) {
    const float4 p = pts[i];
    const double x = (double)p.x - shift_x - cx, y = (double)p.y - shift_y - cy,
                 z = (double)p.z - shift_z - cz;
    s += x * x + y * y + z * z;
    xx += x * x; xy += x * y; xz += x * z; yy += y * y; yz += y * z; zz += z * z;
  }
  I.m[0][0] = s - xx; I.m[0][1] = -xy; I.m[0][2] = -xz;
  I.m[1][0] = -xy; I.m[1][1] = s - yy; I.m[1][2] = -yz;
  I.m[2][0] = -xz; I.m[2][1] = -yz; I.m[2][2] = s - zz;
}

template <typename T>
__device__ void quat_mul(const T a[4], const T b[4], T o[4]) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

// rotation matrix of a quaternion after normalising it (quaternion_to_rotation_matrix, :59-97)
template <typename T>
__device__ void quat_rot(const T q_in[4], T R[3][3]) {
  const T n = sqrt(q_in[0] * q_in[0] + q_in[1] * q_in[1] + q_in[2] * q_in[2] + q_in[3] * q_in[3]);
  const T inv = T(1) / (n > T(1e-12) ? n : T(1e-12));
  const T w = q_in[0] * inv, x = q_in[1] * inv, y = q_in[2] * inv, z = q_in[3] * inv;
  R[0][0] = 1 - 2 * (y * y + z * z); R[0][1] = 2 * (x * y - z * w); R[0][2] = 2 * (x * z + y * w);
  R[1][0] = 2 * (x * y + z * w); R[1][1] = 1 - 2 * (x * x + z * z); R[1][2] = 2 * (y * z - x * w);
  R[2][0] = 2 * (x * z - y * w); R[2][1] = 2 * (y * z + x * w); R[2][2] = 1 - 2 * (x * x + y * y);
}

__global__ void seeds_kernel(const float4* __restrict__ rp, const int* __restrict__ roff,
                             const Pts fp, const int* __restrict__ foff,
                             const int* __restrict__ pair_ref, const int* __restrict__ pair_fit,
                             int P, int S, const float* __restrict__ fibo, int n_fibo,
                             float* __restrict__ sq, float* __restrict__ st) {
  const int pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= P) return;
  float* oq = sq + (size_t)pi * S * 4;
  float* ot = st + (size_t)pi * S * 3;
  if (S == 1) {
    oq[0] = 1.f; oq[1] = 0.f; oq[2] = 0.f; oq[3] = 0.f;
    ot[0] = 0.f; ot[1] = 0.f; ot[2] = 0.f;
    return;
  }
  const int ri = pair_ref[pi], fi = pair_fit[pi];
  const float4* A = rp + roff[ri];
  const Pts B = fp + foff[fi];
  const int N = roff[ri + 1] - roff[ri], M = foff[fi + 1] - foff[fi];
  // float32 centroids (the COM used by the translations)
  float rc[3] = {0.f, 0.f, 0.f}, fc[3] = {0.f, 0.f, 0.f};
  bool finite = true;
  for (int i = 0; i < N; ++i) {
    const float4 p = A[i];
    rc[0] += p.x; rc[1] += p.y; rc[2] += p.z;
    finite = finite && isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
  }
  for (int i = 0; i < M; ++i) {
    const float4 p = B[i];
    fc[0] += p.x; fc[1] += p.y; fc[2] += p.z;
    finite = finite && isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
  }
  const float nr = (float)(N > 0 ? N : 1), nf = (float)(M > 0 ? M : 1);
  for (int i = 0; i < 3; ++i) { rc[i] /= nr; fc[i] /= nf; }
  const bool valid = N >= 3 && M >= 3 && finite;

  float quats[64][4];  // S <= 64 is enforced by the launcher
  if (valid) {
    M3 Ir, ref_axes, If, fax;
    inertia(A, N, 0.0, 0.0, 0.0, Ir);
    sym3x3_axes(Ir, ref_axes);
    inertia(B, M, (double)fc[0], (double)fc[1], (double)fc[2], If);
    sym3x3_axes(If, fax);  // fit axes before any rotation (axis-0 alignment)
    float pca[4][4];
    for (int v = 0; v < 4; ++v) {
      double rax[2][3];
      for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 3; ++c) {
          double s = ref_axes.m[a][c];
          if ((v == 1 && a == 0) || (v == 2 && a == 1) || (v == 3)) s = -s;
          rax[a][c] = s;
        }
      double qo[2][4];
      M3 cur = fax;   // fit axes of the (rotated) fit cloud
      M3 Irot = If;
      for (int ax = 0; ax < 2; ++ax) {
        if (ax == 1) sym3x3_axes(Irot, cur);
        const double* v1 = cur.m[ax];
        const double* v2 = rax[ax];
        double cs = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
        cs = fmin(fmax(cs, -1.0), 1.0);
        const double ang = acos(cs);
        double axis[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                          v1[0] * v2[1] - v1[1] * v2[0]};
        const double an = sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
        if (an < 1e-8) {
          axis[0] = 1.0; axis[1] = 0.0; axis[2] = 0.0;
        } else {
          const double inv = 1.0 / fmax(an, 1e-12);
          axis[0] *= inv; axis[1] *= inv; axis[2] *= inv;
        }
        const double h = ang * 0.5, sh = sin(h);
        qo[ax][0] = cos(h); qo[ax][1] = axis[0] * sh; qo[ax][2] = axis[1] * sh; qo[ax][3] = axis[2] * sh;
        if (ax == 0) {  // inertia of the rotated cloud: R I R^T
          double R[3][3];
          quat_rot<double>(qo[0], R);
          double T[3][3];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
              T[i][j] = R[i][0] * If.m[0][j] + R[i][1] * If.m[1][j] + R[i][2] * If.m[2][j];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
              Irot.m[i][j] = T[i][0] * R[j][0] + T[i][1] * R[j][1] + T[i][2] * R[j][2];
        }
      }
      double qq[4];
      quat_mul<double>(qo[1], qo[0], qq);
      for (int c = 0; c < 4; ++c) pca[v][c] = (float)qq[c];
    }
    int n = 0;
    quats[n][0] = 1.f; quats[n][1] = 0.f; quats[n][2] = 0.f; quats[n][3] = 0.f; ++n;
    for (int v = 0; v < 4 && n < S; ++v, ++n)
      for (int c = 0; c < 4; ++c) quats[n][c] = pca[v][c];
    const int n_struct = min(max(S - 5, 0), 6);
    const float ch = 0.70710678118654757f, sh = 0.70710678118654757f;
    for (int s = 0; s < n_struct; ++s) {
      const int a = s / 2;
      const float sg = (s % 2 == 0) ? sh : -sh;
      const float qa[4] = {ch, sg * (float)ref_axes.m[a][0], sg * (float)ref_axes.m[a][1],
                           sg * (float)ref_axes.m[a][2]};
      quat_mul<float>(qa, pca[0], quats[n]);
      ++n;
    }
    for (int f = 0; n < S && f < n_fibo; ++f, ++n)
      for (int c = 0; c < 4; ++c) quats[n][c] = fibo[f * 4 + c];
    for (; n < S; ++n) { quats[n][0] = 1.f; quats[n][1] = quats[n][2] = quats[n][3] = 0.f; }
  } else {
    // fixed fallback rotations (_common.py:189-204), cycled
    const float s2 = 0.70710678118654757f;
    const float base[10][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}, {s2, s2, 0, 0},
                               {s2, 0, s2, 0}, {s2, 0, 0, s2}, {0, s2, s2, 0}, {0, s2, 0, s2}, {0, 0, s2, s2}};
    for (int n = 0; n < S; ++n)
      for (int c = 0; c < 4; ++c) quats[n][c] = base[n % 10][c];
  }
  for (int n = 0; n < S; ++n) {
    float* q = quats[n];
    const float nn = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float inv = 1.f / fmaxf(nn, 1e-12f);
    for (int c = 0; c < 4; ++c) { q[c] *= inv; oq[n * 4 + c] = q[c]; }
    if (valid) {
      float R[3][3];
      quat_rot<float>(q, R);
      for (int r = 0; r < 3; ++r)
        ot[n * 3 + r] = rc[r] - (R[r][0] * fc[0] + R[r][1] * fc[1] + R[r][2] * fc[2]);
    } else {
      for (int r = 0; r < 3; ++r) ot[n * 3 + r] = rc[r] - fc[r];
    }
  }
}

}  // namespace

int seeds_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                 const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                 int P, int S, const float* fibo, int n_fibo, int fit_f16, float* sq, float* st,
                 cudaStream_t stream) {
  if (P < 0 || S < 1 || S > 64 || (S > 1 && S < 5))
    return set_error(FSS_ERR_INVALID, "fss_seeds: n_seeds must be 1 or in [5, 64]");
  if (n_fibo < 0 || (n_fibo > 0 && !fibo))
    return set_error(FSS_ERR_INVALID, "fss_seeds: bad Fibonacci table");
  if (P == 0) return FSS_OK;
  if (!ref_pts || !ref_off || !fit_pts || !fit_off || !pair_ref || !pair_fit || !sq || !st)
    return set_error(FSS_ERR_INVALID, "fss_seeds: null pointer");
  seeds_kernel<<<(P + 63) / 64, 64, 0, stream>>>(
      reinterpret_cast<const float4*>(ref_pts), ref_off, Pts(fit_pts, fit_f16 ? 1 : 0), fit_off,
      pair_ref, pair_fit, P, S, fibo, n_fibo, sq, st);
  return check_launch("fss_seeds");
}

}  // namespace fss
