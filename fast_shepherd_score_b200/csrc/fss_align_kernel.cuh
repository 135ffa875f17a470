// fss_align_kernel.cuh -- the fused persistent alignment kernel (template) and its launcher.
//
// One launch runs every (pair, start) pose for all Adam steps.  Work item = (pair, block
// of starts); a persistent grid pulls items from a device counter in cost order (costliest
// pairs first), stages the pair's clouds in shared memory once and keeps every pose's
// optimiser state in registers for the whole loop.  LPP lanes cooperate on one pose; the
// poses of one CTA all belong to the same pair so the shared-memory reads of the reference
// cloud are warp-wide broadcasts and every loop bound is uniform.
//
// The template is instantiated per mode in fss_align_<mode>.cu (compiled in parallel);
// fss_align.cu holds the host-side validation, tiling and dispatch.
#pragma once
#include <algorithm>
#include <cmath>
#include <string>

#include "fss_internal.cuh"
#include "fss_mma.cuh"
#include "fss_tce.cuh"

namespace fss {


struct AlignParams {
  int mode, n_pairs, n_starts, steps, chunks, n_items;
  int maxN, maxM, maxNp, maxMp;
  const int* pair_ref;
  const int* pair_fit;
  const int* order;
  const float4* ref_pts; const int* ref_off;
  const float4* fit_pts; const int* fit_off;
  const float* ref_self; const float* fit_self;
  const float4* ref_anc; const float4* ref_vec; const int* ref_ph_off;
  const float4* fit_anc; const float4* fit_vec; const int* fit_ph_off;
  const float* ref_self_ph; const float* fit_self_ph;
  const float* seed_q; const float* seed_t;
  float alpha, k, e, inv2k, Kc, aKc, w, lr;
  float sigma;  // pharm mode: Tversky sigma (>= 0) or Tanimoto (< 0)
  // vol_and_surf_esp: atoms with H (x, y, z, q) + radii, surfaces (x, y, z, pe)
  const float4* ref_atoms; const float* ref_radii; const int* ref_atom_off;
  const float4* fit_atoms; const float* fit_radii; const int* fit_atom_off;
  const float4* ref_surf; const int* ref_surf_off;
  const float4* fit_surf; const int* fit_surf_off;
  int maxNa, maxMa, maxNs, maxMs;
  float coulomb, probe, nkl, esp_w;  // nkl = -log2(e) / (LAM_SCALING * lam)
  int esp_stride;
  int fit_f16;  // fit clouds / pharmacophores stored as float16 (x, y, z, w), widened in staging
  PharmTables tab;
  float* row_score; float* row_q; float* row_t;
  int* counter;
};

constexpr int kMaxThreads = 320;  // 10 warps

// Code variants of the FP32-lane hot loop (fss_align_desc.kernel_variant - 1):
//   0  4 fit points per lane, reference loop unrolled 2x, <= 96 registers (2 CTAs/SM)
//   1  6 fit points per lane, unrolled 4x, <= 96 registers: more independent ex2/FMA
//      chains per warp (large clouds)
//   2  4 fit points per lane, unrolled 4x, register budget of one 320-thread CTA per SM:
//      no spills, fewer resident warps (small clouds, whose poses are tail-heavy)
//   3  4 fit points per lane, unrolled 4x, <= 96 registers
//   4  8 fit points per lane, unrolled 2x, register budget of one 320-thread CTA per SM: one
//      pass over the reference cloud for every fit cloud of up to 8 x lanes-per-pose points
//      (small molecules, whose second pass would run mostly empty register tiles)
template <int VAR>
struct AlignVariant;
template <>
struct AlignVariant<0> { static constexpr int kJB2 = 2, kUnroll = 2, kMinCtas = 2; };
template <>
struct AlignVariant<1> { static constexpr int kJB2 = 3, kUnroll = 4, kMinCtas = 2; };
template <>
struct AlignVariant<2> { static constexpr int kJB2 = 2, kUnroll = 4, kMinCtas = 1; };
template <>
struct AlignVariant<3> { static constexpr int kJB2 = 2, kUnroll = 4, kMinCtas = 2; };
template <>
struct AlignVariant<4> { static constexpr int kJB2 = 4, kUnroll = 2, kMinCtas = 1; };

// ACC: where the shape/ESP sums run -- 0 FP32 lanes, 1 tensor-core value/gradient sums
// (fss_mma.cuh), 2 tensor-core exponents (fss_tce.cuh); 1 and 2 need LPP == 32 and a mode
// without a pharmacophore channel.  EXT: extended pharmacophore points (pharm_pose).
template <int LPP, int MODE, int ACC, int VAR, int EXT = 0>
__global__ void __launch_bounds__(kMaxThreads, AlignVariant<VAR>::kMinCtas)
    align_kernel(const AlignParams p) {
  using V = AlignVariant<VAR>;
  constexpr bool TC = ACC == 1;
  constexpr bool TCE = ACC == 2;
  constexpr bool kCombo = MODE == FSS_MODE_ESP_COMBO;
  constexpr bool kShape = MODE == FSS_MODE_SHAPE || MODE == FSS_MODE_ESP ||
                          MODE == FSS_MODE_SHAPE_PHARM || MODE == FSS_MODE_SHAPE_COLOR || kCombo;
  constexpr bool kEsp = MODE == FSS_MODE_ESP;
  constexpr bool kPharm = MODE == FSS_MODE_PHARM || MODE == FSS_MODE_SHAPE_PHARM ||
                          MODE == FSS_MODE_SHAPE_COLOR;
  static_assert(ACC == 0 || (LPP == 32 && !kPharm && (MODE == FSS_MODE_SHAPE || MODE == FSS_MODE_ESP)),
                "tensor-core paths: whole-warp shape/ESP poses");
  extern __shared__ __align__(16) float4 smem[];
  // FP32 path: sP = 2 * maxN duplicated expanded reference (+ sQc).  Tensor-core path:
  // sP = 8 * nbMax block-interleaved reference, sCm/sQm after the fit cloud.
  const int nbMax = (p.maxN + 7) >> 3;
  // parked optimiser state: kColdFields floats per thread (a multiple of 16 bytes per CTA)
  volatile float* sCold = reinterpret_cast<float*>(smem) + threadIdx.x;
  float4* sP = smem + kColdFields * blockDim.x / 4;
  float4* sB = sP + (TC ? kMmaP4PerBlock * nbMax : TCE ? kTceF2PerBlock / 2 * nbMax
                                                     : 2 * p.maxN);
  float4* sRA = sB + p.maxM;
  float4* sRV = sRA + p.maxNp;
  float4* sFA = sRV + p.maxNp;
  float4* sFV = sFA + p.maxMp;
  float2* sQc = reinterpret_cast<float2*>(sFV + p.maxMp);
  float2* sCm = reinterpret_cast<float2*>(sB + p.maxM);
  float2* sQm = sCm + kMmaC2PerBlock * nbMax;
  // vol_and_surf_esp channel: surfaces, atoms with H (negated, duplicated: 2 float4 each),
  // -(radius + probe)^2 duplicated (float2)
  float4* sSA = sFV + p.maxMp;
  float4* sSB = sSA + p.maxNs;
  float4* sAA = sSB + p.maxMs;
  float4* sAB = sAA + 2 * p.maxNa;
  float2* sRA2 = reinterpret_cast<float2*>(sAB + 2 * p.maxMa);
  float2* sRB2 = sRA2 + p.maxNa;
  __shared__ float red[96];
  __shared__ int s_item;
  __shared__ int s_toff[10];   // first reference pharmacophore of each type

  const int tid = threadIdx.x;
  const int grp = tid / LPP, lane = tid % LPP;
  const int ppc = blockDim.x / LPP;  // poses per CTA
  constexpr int kGroupsPerWarp = 32 / LPP;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(p.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= p.n_items) break;
    const int pidx = p.order ? p.order[item / p.chunks] : item / p.chunks;
    const int chunk = item % p.chunks;
    const int ri = p.pair_ref[pidx], fi = p.pair_fit[pidx];

    // ---- stage the pair's clouds -------------------------------------------------------
    int N = 0, M = 0, Np = 0, Mp = 0, r0 = 0, f0 = 0, rp0 = 0, fp0 = 0;
    if (kShape) {
      r0 = p.ref_off[ri]; f0 = p.fit_off[fi];
      N = p.ref_off[ri + 1] - r0;
      M = p.fit_off[fi + 1] - f0;
    }
    if (kPharm) {
      rp0 = p.ref_ph_off[ri]; fp0 = p.fit_ph_off[fi];
      Np = p.ref_ph_off[ri + 1] - rp0;
      Mp = p.fit_ph_off[fi + 1] - fp0;
    }
    int Na = 0, Ma = 0, Ns = 0, Ms = 0, ra0 = 0, fa0 = 0, rs0 = 0, fs0 = 0;
    if (kCombo) {
      ra0 = p.ref_atom_off[ri]; fa0 = p.fit_atom_off[fi];
      rs0 = p.ref_surf_off[ri]; fs0 = p.fit_surf_off[fi];
      Na = p.ref_atom_off[ri + 1] - ra0; Ma = p.fit_atom_off[fi + 1] - fa0;
      Ns = p.ref_surf_off[ri + 1] - rs0; Ms = p.fit_surf_off[fi + 1] - fs0;
    }
    if (N < 0 || M < 0 || Np < 0 || Mp < 0 || N > p.maxN || M > p.maxM || Np > p.maxNp ||
        Mp > p.maxMp || Na < 0 || Ma < 0 || Ns < 0 || Ms < 0 || Na > p.maxNa ||
        Ma > p.maxMa || Ns > p.maxNs || Ms > p.maxMs) {
      // larger than the tiles this launch was sized for: flag it, leave its rows untouched
      if (tid == 0) atomicOr(p.counter + 1, 1);
      __syncthreads();
      continue;
    }
    float3 c = make_float3(0.f, 0.f, 0.f);
    if (kShape) {
      c = block_centroid(p.ref_pts + r0, N, red);
      if constexpr (TC) stage_ref_mma<kEsp>(p.ref_pts + r0, N, c, p.k, p.e, sP, sQm, sCm);
      else if constexpr (TCE)
        stage_ref_tce<kEsp>(p.ref_pts + r0, N, c, p.k, p.e, sP, nbMax);
      else stage_ref<kEsp>(p.ref_pts + r0, N, c, p.k, p.e, sP, sQc);
      stage_copy(Pts(p.fit_pts, p.fit_f16) + f0, M, sB);
    }
    if (kCombo) {
      // reference-side arrays move into the centred frame of the shape channel
      for (int i = tid; i < Ns; i += blockDim.x) {
        const float4 v = p.ref_surf[rs0 + i];
        sSA[i] = make_float4(v.x - c.x, v.y - c.y, v.z - c.z, v.w);
      }
      stage_copy(p.fit_surf + fs0, Ms, sSB);
      for (int i = tid; i < Na; i += blockDim.x) {
        const float4 v = p.ref_atoms[ra0 + i];
        const float x = c.x - v.x, y = c.y - v.y, z = c.z - v.z;
        sAA[2 * i] = make_float4(x, x, y, y);
        sAA[2 * i + 1] = make_float4(z, z, v.w, v.w);
        const float r = p.ref_radii[ra0 + i] + p.probe;
        sRA2[i] = make_float2(-r * r, -r * r);
      }
      for (int i = tid; i < Ma; i += blockDim.x) {
        const float4 v = p.fit_atoms[fa0 + i];
        sAB[2 * i] = make_float4(-v.x, -v.x, -v.y, -v.y);
        sAB[2 * i + 1] = make_float4(-v.z, -v.z, v.w, v.w);
        const float r = p.fit_radii[fa0 + i] + p.probe;
        sRB2[i] = make_float2(-r * r, -r * r);
      }
    }
    if (kPharm) {
      if (!kShape) c = block_centroid(p.ref_anc + rp0, Np, red);
      stage_ref_pharm(p.ref_anc + rp0, p.ref_vec ? p.ref_vec + rp0 : nullptr, Np, c, sRA, sRV,
                      s_toff);
      stage_fit_pharm(Pts(p.fit_anc, p.fit_f16) + fp0, Pts(p.fit_vec, p.fit_f16) + fp0, Mp, sFA,
                      sFV);
    }
    __syncthreads();

    const float Us = p.ref_self[ri] + p.fit_self[fi];
    const float Dtv = p.sigma * p.ref_self[ri] + (1.f - p.sigma) * p.fit_self[fi];
    const float Uc = kShape && kPharm ? p.ref_self_ph[ri] + p.fit_self_ph[fi] : 0.f;
    const int start = chunk * ppc + grp;
    const int warp_first = chunk * ppc + (tid >> 5) * kGroupsPerWarp;
    if (warp_first < p.n_starts) {  // whole idle warps skip the loop; idle groups shadow one
      const bool active = start < p.n_starts;
      const size_t row = (size_t)pidx * p.n_starts + (active ? start : p.n_starts - 1);
      PoseState s;
      {
        float q0[4], t0[3];
#pragma unroll
        for (int i = 0; i < 4; ++i) q0[i] = p.seed_q[row * 4 + i];
        t0[0] = p.seed_t[row * 3 + 0] - c.x;
        t0[1] = p.seed_t[row * 3 + 1] - c.y;
        t0[2] = p.seed_t[row * 3 + 2] - c.z;
        pose_init(s, q0, t0);
        cold_store(s, sCold, blockDim.x);
      }
      for (int step = 0; step < p.steps; ++step) {
        const Rot R = quat_to_rot(s.q);
        Reduced rs;
        if (kShape) {
          Moments ms;
          ms.zero();
          if constexpr (TC)
            shape_pose_mma<kEsp>(sP, sQm, sCm, sB, N, M, lane, R, s.t[0], s.t[1], s.t[2], p.k,
                                 p.e, ms);
          else if constexpr (TCE)
            shape_pose_tce<kEsp>(tce_ref(sP, nbMax), sB, N, M, lane, R, s.t[0], s.t[1], s.t[2],
                                 p.k, p.e, p.inv2k, ms);
          else
            shape_pose<LPP, kEsp, V::kJB2, V::kUnroll>(sP, sQc, sB, N, M, lane, R, s.t[0],
                                                       s.t[1], s.t[2], p.k, p.e, p.inv2k, ms);
          rs.from(ms, s.q);
          rs.template group_sum<LPP>();
          rs.scale(p.Kc, p.aKc);
        }
        if (kPharm) {
          Moments mc;
          mc.zero();
          pharm_pose<LPP, EXT>(sRA, sRV, sFA, sFV, Np, Mp, lane, R, s.t[0], s.t[1], s.t[2], p.tab,
                               mc, s_toff);
          Reduced rc;
          rc.from(mc, s.q);
          rc.template group_sum<LPP>();
          cold_load(s, sCold, blockDim.x);
          if (kShape) step_combo(s, rs, Us, rc, Uc, p.w, p.lr);
          else if (p.sigma >= 0.f) step_tversky(s, rc, Dtv, p.lr);
          else step_single(s, rc, Us, p.lr);
          cold_store(s, sCold, blockDim.x);
        } else if (kCombo) {
          const bool scored = step % p.esp_stride == 0 || step == p.steps - 1;
          float esp = 0.f;
          if (scored) {
            esp = esp_side<LPP, true>(sSA, Ns, sAB, sRB2, Ma, lane, R, s.t[0], s.t[1], s.t[2],
                                      p.coulomb, p.nkl) +
                  esp_side<LPP, false>(sSB, Ms, sAA, sRA2, Na, lane, R, s.t[0], s.t[1],
                                       s.t[2], p.coulomb, p.nkl);
#pragma unroll
            for (int o = LPP / 2; o > 0; o >>= 1) esp += __shfl_xor_sync(0xffffffffu, esp, o);
          }
          cold_load(s, sCold, blockDim.x);
          step_esp_combo(s, rs, Us, esp, (float)(Ns + Ms), p.esp_w, scored, p.lr);
          cold_store(s, sCold, blockDim.x);
        } else {
          cold_load(s, sCold, blockDim.x);
          step_single(s, rs, Us, p.lr);
          cold_store(s, sCold, blockDim.x);
        }
      }
      cold_load(s, sCold, blockDim.x);
      if (active && lane == 0) {
        const size_t r = (size_t)pidx * p.n_starts + start;
        p.row_score[r] = s.best;
#pragma unroll
        for (int i = 0; i < 4; ++i) p.row_q[r * 4 + i] = s.bq[i];
        p.row_t[r * 3 + 0] = s.bt[0] + c.x;
        p.row_t[r * 3 + 1] = s.bt[1] + c.y;
        p.row_t[r * 3 + 2] = s.bt[2] + c.z;
      }
    }
    __syncthreads();  // shared memory is restaged for the next item
  }
}

template <int LPP, int MODE, int ACC, int VAR, int EXT = 0>
int launch_align(const AlignParams& prm, int threads, int cta_per_sm, size_t smem,
                 cudaStream_t st) {
  auto kern = align_kernel<LPP, MODE, ACC, VAR, EXT>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem);
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_align: shared-memory attribute: ") +
                                       cudaGetErrorString(ce));
  int occ = 0;
  ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
  if (ce != cudaSuccess || occ <= 0)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_align: the tile does not fit on an SM");
  if (cta_per_sm > 0) occ = std::min(occ, cta_per_sm);
  const int grid = std::max(1, std::min(prm.n_items, occ * num_sms()));
  kern<<<grid, threads, smem, st>>>(prm);
  return check_launch("fss_align");
}

template <int MODE, int VAR, int EXT = 0>
int dispatch_lanes(int lpp, const AlignParams& prm, int threads, int cps, size_t smem,
                   cudaStream_t st) {
  switch (lpp) {
    case 1: return launch_align<1, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    case 2: return launch_align<2, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    case 4: return launch_align<4, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    case 8: return launch_align<8, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    case 16: return launch_align<16, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    case 32: return launch_align<32, MODE, 0, VAR, EXT>(prm, threads, cps, smem, st);
    default: return set_error(FSS_ERR_INVALID, "fss_align: lanes_per_pose must be 1, 2, 4, 8, 16 or 32");
  }
}

// Per-mode launchers (one translation unit each).  var: as AlignVariant; acc: 0 FP32 lanes,
// 1 tensor-core sums, 2 tensor-core exponents (shape and ESP modes only).
int launch_align_shape(int lpp, int acc, int var, const AlignParams& prm, int threads, int cps,
                       size_t smem, cudaStream_t st);
int launch_align_esp(int lpp, int acc, int var, const AlignParams& prm, int threads, int cps,
                     size_t smem, cudaStream_t st);
int launch_align_pharm(int mode, int lpp, int ext, const AlignParams& prm, int threads,
                       int cps, size_t smem, cudaStream_t st);
int launch_align_combo(int lpp, int var, const AlignParams& prm, int threads, int cps,
                       size_t smem, cudaStream_t st);

}  // namespace fss
