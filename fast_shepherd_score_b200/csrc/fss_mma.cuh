// fss_mma.cuh -- tensor-core accumulation of the shape / ESP pairwise sums.
//
// The hot loop of the FP32 path spends 8 FP32 lane-ops per pair term (4 for the exponent,
// 4 to accumulate value and gradient) next to one MUFU ex2, which loads the FP32 pipe
// exactly as hard as the MUFU pipe (128 vs 16 lanes per clock per SM).  The accumulation
//     (G_j, S_j) = sum_i g_ij (1, a_i)
// is a product of the [fit rows x N] term matrix with an [N x 8] column table, so here it
// runs on the tensor cores as mma.m16n8k8 with tf32 operands: the term values come out of
// the MUFU in registers, already in the A-fragment layout, and the column table is a static
// per-pair fragment array in shared memory.  mma.sync (register operands) rather than
// tcgen05.mma is used because the A operand is produced per instruction in registers; the
// tensor work is ~1/8 of the tensor-core rate, so its issue path is not the bound.
//
// Precision: tf32 keeps 11 significant bits, so both sides are split into hi + lo parts:
//   g = g_hi + g_lo   (g_hi = g with the low 13 mantissa bits cleared, g_lo = g - g_hi)
//   a = a_hi + a_lo   (staged once per pair; a_lo rounded to tf32)
// and the columns of the table are (1, a_hi, a_lo, 0).  Two MMAs (A = g_hi, A = g_lo)
// against the same table accumulate g_hi a_hi + g_hi a_lo + g_lo a_hi + g_lo a_lo into
// FP32, leaving a relative error of about 2^-21 per product -- the same order as the FP32
// path's own accumulation error.
//
// Work split: one warp owns one pose and walks the fit cloud in passes of 32 rows (two
// 16-row MMA tiles).  Lane (g = lane/4, t = lane%4) evaluates rows {g, g+8, g+16, g+24} of
// the pass against reference points {8kb+t, 8kb+t+4} of block kb -- exactly the A-fragment
// positions (a0..a3) of the two tiles -- with f32x2 arithmetic over the two reference
// points.  FP32 work per term drops to 3 (shape) / 4 (ESP) exponent ops plus one split op.
#pragma once
#include "fss_device.cuh"

namespace fss {

__device__ __forceinline__ float tf32_hi(float x) {
  return __int_as_float(__float_as_int(x) & 0xffffe000);
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t y;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(x));
  return __uint_as_float(y);
}

// D (16x8, FP32) += A (16x8, tf32) * B (8x8, tf32).  Fragment layout (g = lane/4, t = lane%4):
//   a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4]
//   b.x = B[t][g], b.y = B[t+4][g]
//   d0 = D[g][2t], d1 = D[g][2t+1], d2 = D[g+8][2t], d3 = D[g+8][2t+1]
__device__ __forceinline__ void mma_tf32(float d[4], float a0, float a1, float a2, float a3,
                                         float2 b) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(__float_as_uint(a0)), "r"(__float_as_uint(a1)), "r"(__float_as_uint(a2)),
        "r"(__float_as_uint(a3)), "r"(__float_as_uint(b.x)), "r"(__float_as_uint(b.y)));
}

// Shared-memory words per reference block of 8 points (float4 / float2 units).
constexpr int kMmaP4PerBlock = 8;    // sPm: 4 quads x 2 float4
constexpr int kMmaQ2PerBlock = 4;    // sQm: 4 float2
constexpr int kMmaC2PerBlock = 32;   // sCm: one float2 B fragment per lane

// Stage a reference cloud (centred on c) for the tensor-core path.  Reference slot
// i = 8kb + t + 4h (h = 0, 1) of block kb goes to
//   sPm[(4kb+t)*2]     = (2k ax_i, 2k ax_i', 2k ay_i, 2k ay_i')       (i' = i + 4)
//   sPm[(4kb+t)*2 + 1] = (2k az_i, 2k az_i', P.w_i, P.w_i')
//   sQm[4kb+t]         = (2e c_i, 2e c_i')                            (ESP only)
//   sCm[32kb + 4n + t] = (C[i][n], C[i'][n]),  C[i] = (1, ax_hi, ay_hi, az_hi, ax_lo, ay_lo, az_lo, 0)
// with P.w = -k|a|^2 - e c^2.  Slots past n get P.w = -inf (a zero term) and a zero row of C.
template <bool ESP>
__device__ __forceinline__ void stage_ref_mma(const float4* __restrict__ g, int n, float3 c,
                                              float k, float e, float4* sPm, float2* sQm,
                                              float2* sCm) {
  const int slots = ((n + 7) >> 3) << 3;
  for (int i = threadIdx.x; i < slots; i += blockDim.x) {
    const int kb = i >> 3, t = i & 3, h = (i >> 2) & 1;
    float ax = 0.f, ay = 0.f, az = 0.f, w = -INFINITY, q = 0.f, one = 0.f;
    if (i < n) {
      const float4 p = g[i];
      ax = p.x - c.x; ay = p.y - c.y; az = p.z - c.z;
      w = -k * (ax * ax + ay * ay + az * az);
      if (ESP) {
        w = fmaf(-e * p.w, p.w, w);
        q = 2.f * e * p.w;
      }
      one = 1.f;
    }
    float* P = reinterpret_cast<float*>(sPm + (4 * kb + t) * 2);
    P[0 + h] = 2.f * k * ax;
    P[2 + h] = 2.f * k * ay;
    P[4 + h] = 2.f * k * az;
    P[6 + h] = w;
    if (ESP) reinterpret_cast<float*>(sQm + 4 * kb + t)[h] = q;
    const float hx = tf32_hi(ax), hy = tf32_hi(ay), hz = tf32_hi(az);
    const float col[8] = {one, hx, hy, hz, tf32_round(ax - hx), tf32_round(ay - hy),
                          tf32_round(az - hz), 0.f};
#pragma unroll
    for (int nn = 0; nn < 8; ++nn)
      reinterpret_cast<float*>(sCm + 32 * kb + 4 * nn + t)[h] = col[nn];
  }
}

// One pass of 32 fit rows against every reference block: D[m] accumulates tile m (rows
// 16m .. 16m+15 of the pass).  FACT: the per-row factor 2^-W_r is applied after the sum
// (see shape_chunk_packed); otherwise NW_r = -W_r is added to every exponent.
template <bool ESP, bool FACT>
__device__ __forceinline__ void mma_pass(const float4* __restrict__ sPm,
                                         const float2* __restrict__ sQm,
                                         const float2* __restrict__ sCm, int nb, int lane,
                                         const float2 BX[4], const float2 BY[4],
                                         const float2 BZ[4], const float2 CJ[4],
                                         const float2 NW[4], float D[2][4]) {
  const int t = lane & 3;
  const float4* pp = sPm + 2 * t;
  const float2* qp = sQm + t;
  const float2* cp = sCm + lane;
#pragma unroll 2
  for (int kb = 0; kb < nb; ++kb) {
    const float4 pa = pp[kMmaP4PerBlock * kb], pb = pp[kMmaP4PerBlock * kb + 1];
    const float2 PX = f2(pa.x, pa.y), PY = f2(pa.z, pa.w), PZ = f2(pb.x, pb.y),
                 PW = f2(pb.z, pb.w);
    float2 QC;
    if (ESP) QC = qp[kMmaQ2PerBlock * kb];
    const float2 cb = cp[kMmaC2PerBlock * kb];
    float2 G[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      float2 E = __ffma2_rn(PX, BX[r], __ffma2_rn(PY, BY[r], __ffma2_rn(PZ, BZ[r], PW)));
      if (ESP) E = __ffma2_rn(QC, CJ[r], E);
      if (!FACT) E = __fadd2_rn(E, NW[r]);
      G[r] = f2(ex2(E.x), ex2(E.y));
    }
    const float2 neg1 = f2(-1.f, -1.f);
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const float2 u = G[2 * m], v = G[2 * m + 1];  // rows g / g+8 of tile m; k = t, t+4
      const float2 uh = f2(tf32_hi(u.x), tf32_hi(u.y)), vh = f2(tf32_hi(v.x), tf32_hi(v.y));
      // lo = g - hi, exact (hi is a truncation of g)
      const float2 ul = __ffma2_rn(uh, neg1, u), vl = __ffma2_rn(vh, neg1, v);
      mma_tf32(D[m], uh.x, vh.x, uh.y, vh.y, cb);
      mma_tf32(D[m], ul.x, vl.x, ul.y, vl.y, cb);
    }
  }
}

// Shape / ESP sums of one pose with the whole warp (lane 0..31).  Adds this lane's share of
// the value, force and moment to acc in the units of shape_pose (raw v, f_j = S_j - b'_j G_j).
template <bool ESP>
__device__ __forceinline__ void shape_pose_mma(const float4* __restrict__ sPm,
                                               const float2* __restrict__ sQm,
                                               const float2* __restrict__ sCm,
                                               const float4* __restrict__ sB, int N, int M,
                                               int lane, const Rot& R, float tx, float ty,
                                               float tz, float k, float e, Moments& acc) {
  const int nb = (N + 7) >> 3;
  const int g = lane >> 2, t = lane & 3;
  for (int j0 = 0; j0 < M; j0 += 32) {
    float2 BX[4], BY[4], BZ[4], CJ[4], NW[4];
    float W[4];
    bool big = false;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int j = j0 + g + 8 * r;
      const bool ok = j < M;
      // rows past M evaluate the origin (finite terms) and are dropped below
      float x = 0.f, y = 0.f, z = 0.f, cj = 0.f;
      if (ok) {
        const float4 b = sB[j];
        const float3 p = rot_apply(R, b.x, b.y, b.z);
        x = p.x + tx; y = p.y + ty; z = p.z + tz; cj = b.w;
      }
      float w = k * (x * x + y * y + z * z);
      if (ESP) w = fmaf(e * cj, cj, w);
      big = big || (ok && w > kFactorMax);
      W[r] = w;
      BX[r] = f2(x, x); BY[r] = f2(y, y); BZ[r] = f2(z, z); CJ[r] = f2(cj, cj);
      NW[r] = f2(-w, -w);
    }
    float D[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int i = 0; i < 4; ++i) D[m][i] = 0.f;
    const bool fact = !__any_sync(0xffffffffu, big);
    if (fact)
      mma_pass<ESP, true>(sPm, sQm, sCm, nb, lane, BX, BY, BZ, CJ, NW, D);
    else
      mma_pass<ESP, false>(sPm, sQm, sCm, nb, lane, BX, BY, BZ, CJ, NW, D);
    // Lane t holds columns 2t, 2t+1 of its rows: (G, Sx) (Sy, Sz) (Sx', Sy') (Sz', 0) with
    // S = S_hi-part + S_lo-part summed below; every term is linear, so each lane adds its
    // own columns and the pose-wide butterfly completes the sums.
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int j = j0 + g + 8 * r;
      if (j < M) {
        const float u0 = D[r >> 1][2 * (r & 1)], u1 = D[r >> 1][2 * (r & 1) + 1];
        const float s = fact ? ex2(-W[r]) : 1.f;
        const float gs = (t == 0 ? u0 : 0.f) * s;
        const float sx = (t == 0 ? u1 : (t == 2 ? u0 : 0.f)) * s;
        const float sy = (t == 1 ? u0 : (t == 2 ? u1 : 0.f)) * s;
        const float sz = (t == 1 ? u1 : (t == 3 ? u0 : 0.f)) * s;
        const float4 b = sB[j];
        acc.v += gs;
        acc.add_force(sx - BX[r].x * gs, sy - BY[r].x * gs, sz - BZ[r].x * gs, b.x, b.y, b.z);
      }
    }
  }
}

}  // namespace fss
