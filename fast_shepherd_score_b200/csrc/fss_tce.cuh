// fss_tce.cuh -- tensor-core exponents for the shape / ESP pairwise sums.
//
// The base-2 exponent of a term is
//     E_ji = A_j . B_i + P.w_i,   A_j = (b'_x, b'_y, b'_z, c_j),   B_i = (2k a_x, 2k a_y, 2k a_z, 2e c_i)
// (factored form: the per-fit-point part -k|b'|^2 - e c_j^2 is applied after the sum over i;
// shape modes have c = 0), i.e. a [fit rows x 4] x [4 x reference points] product per pose and
// step plus a per-column constant.  Here it runs on the tensor cores with tf32 operands in
// split precision (x_hi = tf32(x), x_lo = tf32(x - x_hi)):
//     E = P.w + A_hi B_lo                     mma.m16n8k4, accumulator initialised with P.w
//         + [A_hi | A_lo] [B_hi ; B_hi]       mma.m16n8k8 (K = 8 packs both cross terms)
// so the constant P.w enters exactly in FP32 and the three significant products take one k8 and
// one k4 instruction.  The dropped A_lo B_lo and the tf32 rounding of x_lo leave about
// 3 * 2^-22 |A_k B_k| per product, a few times the rounding of the FP32 path's chained FMAs on
// the same expanded form; the errors of the terms are independent, so a sum over many terms
// keeps fp32-level relative accuracy.  B is split once per work item, A once per pass of 16 fit
// rows; the MUFU ex2 and the value/gradient accumulation stay on the SM:
//     per term 1 ex2 + 4 FP32 lane-ops (f32x2 over the fragment's two reference columns),
// against 1 ex2 + 8 FP32 lane-ops on the FP32 path, where the FMA pipe is as busy as the MUFU.
//
// Fragment layouts (g = lane/4, t = lane%4).  k8: a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4],
// a3 = A[g+8][t+4]; b0 = B[t][g], b1 = B[t+4][g].  k4: a0 = A[g][t], a1 = A[g+8][t];
// b0 = B[t][g].  C/D: d0,d1 = E[g][2t, 2t+1], d2,d3 = E[g+8][2t, 2t+1].  With the packing
// above lane (g, t) holds component t of fit rows g and g+8 (hi and lo) and component t of
// reference point g of each block (hi and lo).  One warp owns one pose; lane t of row quad g
// keeps partial value/gradient sums of fit rows g and g+8 over its two columns of every block.
#pragma once
#include "fss_mma.cuh"

namespace fss {

// Shared memory per reference block of 8 points (in float2 units).
constexpr int kTceFragPerBlock = 32;  // float2 per lane: (B_hi[t][g], B_lo[t][g])
constexpr int kTceColPerBlock = 4;    // per t: float4 (PX_2t, PX_2t+1, PY_2t, PY_2t+1),
                                      // float4 (P.w_2t, P.w_2t+1, P.w_2t, P.w_2t+1),
                                      // float2 (PZ_2t, PZ_2t+1)
constexpr int kTceF2PerBlock = kTceFragPerBlock + kTceColPerBlock * 5;
// blocks in flight per lane: the HMMA -> MUFU -> FFMA chain of a block is latency bound, so
// the loop runs 4 independent blocks (measured: 1 -> 107.5 ms, 2 -> 102.3 ms, 4 -> 96.9 ms on
// 1024 surface pairs x 50 starts x 50 steps)
constexpr int kTceUnroll = 4;

// D = A (16x4, tf32) * B (4x8, tf32) + C
__device__ __forceinline__ void mma_tf32_k4(float d[4], float a0, float a1, float b,
                                            float4 c) {
  asm("mma.sync.aligned.m16n8k4.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%7,%8,%9,%10};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(__float_as_uint(a0)), "r"(__float_as_uint(a1)), "r"(__float_as_uint(b)),
        "f"(c.x), "f"(c.y), "f"(c.z), "f"(c.w));
}

// Staged layout of one reference cloud: nb blocks; per block 32 fragment float2, then the
// column tables of the 4 quad members.
struct TceRef {
  const float2* frag;   // [nb][32]
  const float4* colxy;  // [nb][4]
  const float4* colw;   // [nb][4]
  const float2* colz;   // [nb][4]
};

__device__ __forceinline__ TceRef tce_ref(float4* base, int nbMax) {
  float2* f = reinterpret_cast<float2*>(base);
  TceRef r;
  r.frag = f;
  r.colxy = reinterpret_cast<const float4*>(f + kTceFragPerBlock * nbMax);
  r.colw = r.colxy + kTceColPerBlock * nbMax;
  r.colz = reinterpret_cast<const float2*>(r.colw + kTceColPerBlock * nbMax);
  return r;
}

// Stage a reference cloud (centred on c) for the tensor-core exponents.  Slots past n get
// B = 0 and P.w = -1e30 (a zero term).
template <bool ESP>
__device__ __forceinline__ void stage_ref_tce(const float4* __restrict__ g, int n, float3 c,
                                              float k, float e, float4* base, int nbMax) {
  const int nb = (n + 7) >> 3;
  const TceRef r = tce_ref(base, nbMax);
  float2* frag = const_cast<float2*>(r.frag);
  float4* colxy = const_cast<float4*>(r.colxy);
  float4* colw = const_cast<float4*>(r.colw);
  float2* colz = const_cast<float2*>(r.colz);
  // B fragments: one float2 per (block, lane)
  for (int idx = threadIdx.x; idx < nb * 32; idx += blockDim.x) {
    const int kb = idx >> 5, lane = idx & 31, gg = lane >> 2, t = lane & 3;
    const int i = 8 * kb + gg;  // reference point of column gg
    float b = 0.f;
    if (i < n) {
      const float4 p = g[i];
      b = t == 0 ? p.x - c.x : t == 1 ? p.y - c.y : t == 2 ? p.z - c.z : 0.f;
      b *= 2.f * k;
      if (ESP && t == 3) b = 2.f * e * p.w;
    }
    const float h = tf32_round(b);
    frag[idx] = make_float2(h, tf32_round(b - h));
  }
  // column tables for the accumulation: block kb, quad member t -> points 2t, 2t+1
  for (int idx = threadIdx.x; idx < nb * 4; idx += blockDim.x) {
    const int kb = idx >> 2, t = idx & 3;
    float v[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = 8 * kb + 2 * t + h;
      v[h][0] = v[h][1] = v[h][2] = 0.f;
      v[h][3] = -1e30f;
      if (i < n) {
        const float4 p = g[i];
        const float ax = p.x - c.x, ay = p.y - c.y, az = p.z - c.z;
        v[h][0] = 2.f * k * ax; v[h][1] = 2.f * k * ay; v[h][2] = 2.f * k * az;
        float w = -k * (ax * ax + ay * ay + az * az);
        if (ESP) w = fmaf(-e * p.w, p.w, w);
        v[h][3] = w;
      }
    }
    colxy[idx] = make_float4(v[0][0], v[1][0], v[0][1], v[1][1]);
    colw[idx] = make_float4(v[0][3], v[1][3], v[0][3], v[1][3]);
    colz[idx] = make_float2(v[0][2], v[1][2]);
  }
}

// Sums of rows g and g+8 of one pass over every reference block: this lane's columns 2t, 2t+1
// of each block.  FACT: exponents without the per-row part (applied after the sum); otherwise
// nw = (-W_g, -W_g, -W_g+8, -W_g+8) joins the accumulator's initial value.
template <bool FACT>
__device__ __forceinline__ void tce_pass(const TceRef& r, int lane, int t, int nb, float ah0,
                                         float ah1, float al0, float al1, float4 nw,
                                         float2 (&sg)[2], float2 (&sx)[2], float2 (&sy)[2],
                                         float2 (&sz)[2]) {
  const float2* fp = r.frag + lane;
  const float4* xp = r.colxy + t;
  const float4* wp = r.colw + t;
  const float2* zp = r.colz + t;
#pragma unroll kTceUnroll
  for (int kb = 0; kb < nb; ++kb) {
    const float2 bf = fp[kTceFragPerBlock * kb];
    const float4 col = xp[kTceColPerBlock * kb];
    float4 cw = wp[kTceColPerBlock * kb];
    const float2 colz = zp[kTceColPerBlock * kb];
    if constexpr (!FACT) {
      const float2 lo = __fadd2_rn(f2(cw.x, cw.y), f2(nw.x, nw.y));
      const float2 hi = __fadd2_rn(f2(cw.z, cw.w), f2(nw.z, nw.w));
      cw = make_float4(lo.x, lo.y, hi.x, hi.y);
    }
    float d[4];
    mma_tf32_k4(d, ah0, ah1, bf.y, cw);                  // P.w + A_hi B_lo
    mma_tf32(d, ah0, ah1, al0, al1, f2(bf.x, bf.x));     // + A_hi B_hi + A_lo B_hi
    const float2 g0 = f2(ex2(d[0]), ex2(d[1])), g1 = f2(ex2(d[2]), ex2(d[3]));
    const float2 PX = f2(col.x, col.y), PY = f2(col.z, col.w);
    sg[0] = __fadd2_rn(sg[0], g0); sg[1] = __fadd2_rn(sg[1], g1);
    sx[0] = __ffma2_rn(g0, PX, sx[0]); sx[1] = __ffma2_rn(g1, PX, sx[1]);
    sy[0] = __ffma2_rn(g0, PY, sy[0]); sy[1] = __ffma2_rn(g1, PY, sy[1]);
    sz[0] = __ffma2_rn(g0, colz, sz[0]); sz[1] = __ffma2_rn(g1, colz, sz[1]);
  }
}

// Shape / ESP sums of one pose with the whole warp; adds this lane's share to acc in the units
// of shape_pose (raw v, f_j = S_j inv2k - b'_j G_j).
template <bool ESP>
__device__ __forceinline__ void shape_pose_tce(const TceRef& ref, const float4* __restrict__ sB,
                                               int N, int M, int lane, const Rot& R, float tx,
                                               float ty, float tz, float k, float e,
                                               float inv2k, Moments& acc) {
  const int nb = (N + 7) >> 3;
  const int g = lane >> 2, t = lane & 3;
  for (int j0 = 0; j0 < M; j0 += 16) {
    // rows g and g+8 of this pass: posed fit point, factor exponent, A component t
    float bx[2], by[2], bz[2], W[2], ah[2], al[2];
    bool big = false;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int j = j0 + g + 8 * r;
      const bool ok = j < M;
      float x = 0.f, y = 0.f, z = 0.f, cj = 0.f;
      if (ok) {
        const float4 b = sB[j];
        const float3 p = rot_apply(R, b.x, b.y, b.z);
        x = p.x + tx; y = p.y + ty; z = p.z + tz; cj = b.w;
      }
      float w = k * (x * x + y * y + z * z);
      if (ESP) w = fmaf(e * cj, cj, w);
      big = big || (ok && w > kFactorMax);
      bx[r] = x; by[r] = y; bz[r] = z; W[r] = w;
      const float v = t == 0 ? x : t == 1 ? y : t == 2 ? z : (ESP ? cj : 0.f);
      ah[r] = tf32_round(v);
      al[r] = tf32_round(v - ah[r]);
    }
    const bool fact = !__any_sync(0xffffffffu, big);
    float2 sg[2], sx[2], sy[2], sz[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      sg[r] = f2(0.f, 0.f); sx[r] = f2(0.f, 0.f); sy[r] = f2(0.f, 0.f); sz[r] = f2(0.f, 0.f);
    }
    if (fact)
      tce_pass<true>(ref, lane, t, nb, ah[0], ah[1], al[0], al[1], make_float4(0, 0, 0, 0), sg,
                     sx, sy, sz);
    else
      tce_pass<false>(ref, lane, t, nb, ah[0], ah[1], al[0], al[1],
                      make_float4(-W[0], -W[0], -W[1], -W[1]), sg, sx, sy, sz);
    // this lane's partial sums of rows g and g+8 (linear: the pose-wide sum completes them)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int j = j0 + g + 8 * r;
      if (j < M) {
        const float s = fact ? ex2(-W[r]) : 1.f;
        const float G = (sg[r].x + sg[r].y) * s;
        const float X = (sx[r].x + sx[r].y) * s, Y = (sy[r].x + sy[r].y) * s,
                    Z = (sz[r].x + sz[r].y) * s;
        const float4 b = sB[j];
        acc.v += G;
        acc.add_force(fmaf(X, inv2k, -bx[r] * G), fmaf(Y, inv2k, -by[r] * G),
                      fmaf(Z, inv2k, -bz[r] * G), b.x, b.y, b.z);
      }
    }
  }
}

}  // namespace fss
