// fss_align.cu -- host side of the fused alignment (validation, tiling, dispatch) and the
// small helper kernels (per-pair argmax, self overlaps).  The fused kernel itself lives in
// fss_align_kernel.cuh and is instantiated per mode in fss_align_<mode>.cu.
#include <algorithm>
#include <cmath>

#include "fss_align_kernel.cuh"

namespace fss {

// Per-pair argmax over starts (first index wins ties, as torch.argmax).
__global__ void pick_best_kernel(const float* __restrict__ rs, const float* __restrict__ rq,
                                 const float* __restrict__ rt, int P, int S, float* os, float* oq,
                                 float* ot) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int bi = 0;
  float bs = rs[(size_t)p * S];
  for (int s = 1; s < S; ++s) {
    const float v = rs[(size_t)p * S + s];
    if (v > bs) { bs = v; bi = s; }
  }
  const size_t r = (size_t)p * S + bi;
  os[p] = bs;
#pragma unroll
  for (int i = 0; i < 4; ++i) oq[(size_t)p * 4 + i] = rq[r * 4 + i];
#pragma unroll
  for (int i = 0; i < 3; ++i) ot[(size_t)p * 3 + i] = rt[r * 3 + i];
}

// ---------------------------------------------------------------------------------------
// Self overlaps of packed clouds at the identity pose (one CTA of 32 threads per molecule).
// ---------------------------------------------------------------------------------------
template <bool ESP>
__global__ void self_overlap_kernel(const Pts pts, const int* __restrict__ off,
                                    int n_mol, int max_n, float k, float e, float inv2k, float Kc,
                                    float* out) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float red[96];
  const int m = blockIdx.x;
  const int o0 = off[m], n = off[m + 1] - o0;
  if (n < 0 || n > max_n) {  // larger than the launch's tile: report NaN, touch nothing else
    if (threadIdx.x == 0) out[m] = __int_as_float(0x7fc00000);
    return;
  }
  float4* sP = smem;
  float4* sB = sP + 2 * n;
  float2* sQc = reinterpret_cast<float2*>(sB + n);
  const float3 c = block_centroid(pts + o0, n, red);
  stage_ref<ESP>(pts + o0, n, c, k, e, sP, sQc);
  stage_copy(pts + o0, n, sB);
  __syncthreads();
  Rot R;
#pragma unroll
  for (int i = 0; i < 9; ++i) R.r[i] = (i % 4 == 0) ? 1.f : 0.f;
  Moments acc;
  acc.zero();
  shape_pose<32, ESP>(sP, sQc, sB, n, n, threadIdx.x, R, -c.x, -c.y, -c.z, k, e, inv2k, acc);
  acc.group_sum<32>();
  if (threadIdx.x == 0) out[m] = acc.v * Kc;
}

template <int EXT>
__global__ void pharm_self_kernel(const Pts anc, const Pts vec, const int* __restrict__ off,
                                  int n_mol, int max_n, PharmTables tab, float* out) {
  extern __shared__ __align__(16) float4 smem[];
  __shared__ float red[96];
  const int m = blockIdx.x;
  const int o0 = off[m], n = off[m + 1] - o0;
  if (n < 0 || n > max_n) {
    if (threadIdx.x == 0) out[m] = __int_as_float(0x7fc00000);
    return;
  }
  float4* sRA = smem;
  float4* sRV = sRA + n;
  float4* sFA = sRV + n;
  float4* sFV = sFA + n;
  const float3 c = block_centroid(anc + o0, n, red);
  stage_ref_pharm(anc + o0, vec + o0, n, c, sRA, sRV);
  stage_fit_pharm(anc + o0, vec + o0, n, sFA, sFV);
  __syncthreads();
  Rot R;
#pragma unroll
  for (int i = 0; i < 9; ++i) R.r[i] = (i % 4 == 0) ? 1.f : 0.f;
  Moments acc;
  acc.zero();
  pharm_pose<32, EXT>(sRA, sRV, sFA, sFV, n, n, threadIdx.x, R, -c.x, -c.y, -c.z, tab, acc);
  acc.group_sum<32>();
  if (threadIdx.x == 0) out[m] = acc.v;
}

PharmTables make_pharm_tables(bool directional) {
  // P_TYPES order: Acceptor, Donor, Aromatic, Hydrophobe, Halogen, Cation, Anion, ZnBinder,
  // Dummy (score/constants.py:20); alphas from P_ALPHAS (constants.py:24-34).
  static const double alphas[9] = {1.0, 1.0, 0.7, 0.7, 1.0, 1.0, 1.0, 1.0, 1.0};
  static const int cats_dir[9] = {1, 1, 2, 0, 1, 0, 0, 0, 3};
  PharmTables t;
  for (int i = 0; i < 9; ++i) {
    t.alpha[i] = (float)alphas[i];
    t.K[i] = (float)std::pow(M_PI / (2.0 * alphas[i]), 1.5);
    t.cat[i] = directional ? cats_dir[i] : (i == 8 ? 3 : 0);
  }
  return t;
}

namespace {

// Default tiling (the Python autotuner overrides it with measured choices): lanes per pose
// so that each lane owns about 8 fit points -- enough pairwise work per lane to amortise
// the per-step group reduction and Adam tail -- and start blocks that waste the fewest pose
// slots.  Pharmacophore-only poses are tiny, so they get the narrowest groups.
void auto_tile(int mode, int max_fit, int n_starts, int* lpp, int* chunks) {
  int l = *lpp;
  if (l <= 0) {
    const int m = mode == FSS_MODE_PHARM ? 0 : max_fit;
    l = m < 64 ? 4 : (m < 128 ? 8 : (m < 256 ? 16 : 32));
  }
  *lpp = l;
  if (*chunks > 0) return;
  const int max_poses = kMaxThreads / l;
  int best_c = 1, best_waste = 1 << 30;
  for (int c = 1; c <= n_starts; ++c) {
    const int ppc = (n_starts + c - 1) / c;
    if (ppc > max_poses) continue;
    const int warps = (ppc * l + 31) / 32;
    const int waste = warps * 32 / l * c - n_starts;  // idle pose slots
    if (waste < best_waste) { best_waste = waste; best_c = c; }
    if (waste == 0) break;
  }
  *chunks = best_c;
}

}  // namespace

int align_launch(const fss_align_desc* d, cudaStream_t st) {
  if (!d) return set_error(FSS_ERR_INVALID, "fss_align: null descriptor");
  if (d->mode < FSS_MODE_SHAPE || d->mode > FSS_MODE_ESP_COMBO)
    return set_error(FSS_ERR_INVALID, "fss_align: unknown mode");
  if (d->n_pairs < 0 || d->n_starts <= 0 || d->steps < 0)
    return set_error(FSS_ERR_INVALID, "fss_align: needs n_pairs >= 0, n_starts > 0, steps >= 0");
  if (!d->scratch || !d->row_score || !d->row_q || !d->row_t || !d->seed_q || !d->seed_t ||
      !d->pair_ref || !d->pair_fit)
    return set_error(FSS_ERR_INVALID, "fss_align: missing pair, seed, row or scratch buffer");
  const bool shape = d->mode != FSS_MODE_PHARM;
  const bool pharm = d->mode == FSS_MODE_PHARM || d->mode == FSS_MODE_SHAPE_PHARM ||
                     d->mode == FSS_MODE_SHAPE_COLOR;
  const bool combo = d->mode == FSS_MODE_ESP_COMBO;
  if (combo && (!d->ref_atoms || !d->ref_radii || !d->ref_atom_off || !d->fit_atoms ||
                !d->fit_radii || !d->fit_atom_off || !d->ref_surf || !d->ref_surf_off ||
                !d->fit_surf || !d->fit_surf_off))
    return set_error(FSS_ERR_INVALID, "fss_align: ESP-comparison channel (atoms, radii, "
                                      "surfaces) missing");
  if (combo && (!(d->esp_inv_lam > 0.f) || !(d->probe_radius >= 0.f) || d->esp_stride < 0))
    return set_error(FSS_ERR_INVALID, "fss_align: ESP comparison needs esp_inv_lam > 0, "
                                      "probe_radius >= 0, esp_stride >= 0");
  if (shape && (!d->ref_pts || !d->ref_off || !d->fit_pts || !d->fit_off || !d->ref_self ||
                !d->fit_self))
    return set_error(FSS_ERR_INVALID, "fss_align: shape channel clouds / self overlaps missing");
  if (pharm && (!d->ref_anc || !d->ref_ph_off || !d->fit_anc || !d->fit_ph_off))
    return set_error(FSS_ERR_INVALID, "fss_align: pharmacophore channel missing");
  if (d->mode == FSS_MODE_PHARM && (!d->ref_self || !d->fit_self))
    return set_error(FSS_ERR_INVALID, "fss_align: pharm self overlaps missing");
  if (shape && pharm && (!d->ref_self_ph || !d->fit_self_ph))
    return set_error(FSS_ERR_INVALID, "fss_align: pharm-channel self overlaps missing");
  if ((d->mode == FSS_MODE_PHARM || d->mode == FSS_MODE_SHAPE_PHARM) && (!d->ref_vec || !d->fit_vec))
    return set_error(FSS_ERR_INVALID, "fss_align: directional pharm needs vectors");
  if (shape && !(d->alpha > 0.f)) return set_error(FSS_ERR_INVALID, "fss_align: alpha must be > 0");
  if (d->fit_f16 != 0 && d->fit_f16 != 1)
    return set_error(FSS_ERR_INVALID, "fss_align: fit_f16 must be 0 or 1");
  if (d->fit_f16 && combo)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_align: float16 fit clouds are not supported in "
                                          "mode ESP_COMBO");
  const int maxN = shape ? d->max_ref_points : 0, maxM = shape ? d->max_fit_points : 0;
  const int maxNp = pharm ? d->max_ref_features : 0, maxMp = pharm ? d->max_fit_features : 0;
  const int maxNa = combo ? d->max_ref_atoms : 0, maxMa = combo ? d->max_fit_atoms : 0;
  const int maxNs = combo ? d->max_ref_surf : 0, maxMs = combo ? d->max_fit_surf : 0;
  if (maxN < 0 || maxM < 0 || maxNp < 0 || maxMp < 0 || maxNa < 0 || maxMa < 0 || maxNs < 0 ||
      maxMs < 0)
    return set_error(FSS_ERR_INVALID, "fss_align: negative extents");
  if (maxN > kMaxPoints || maxM > kMaxPoints || maxNp > kMaxPoints || maxMp > kMaxPoints ||
      maxNa > kMaxPoints || maxMa > kMaxPoints || maxNs > kMaxPoints || maxMs > kMaxPoints)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_align: more than fss_max_points() points in a molecule");

  cudaError_t ce = cudaMemsetAsync(d->scratch, 0, 2 * sizeof(int32_t), st);
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_align: scratch reset: ") + cudaGetErrorString(ce));
  if (d->n_pairs == 0) return FSS_OK;

  const bool tc_mode = d->mode == FSS_MODE_SHAPE || d->mode == FSS_MODE_ESP;
  if (d->accumulate < 0 || d->accumulate > 3)
    return set_error(FSS_ERR_INVALID, "fss_align: accumulate must be 0, 1, 2 or 3");
  if (d->accumulate >= 2 && !tc_mode)
    return set_error(FSS_ERR_INVALID, "fss_align: tensor-core sums need mode SHAPE or ESP");
  // kernel accumulation path: 0 FP32 lanes, 1 tensor-core sums, 2 tensor-core exponents
  const int acc = d->accumulate >= 2 ? d->accumulate - 1 : 0;
  const bool tc = acc != 0;
  if (d->pharm_extended < 0 || d->pharm_extended > 2 ||
      (d->pharm_extended != 0 && d->mode != FSS_MODE_PHARM))
    return set_error(FSS_ERR_INVALID, "fss_align: pharm_extended must be 0, 1 or 2 (mode PHARM)");
  if (d->similarity < 0 || d->similarity > 1 || (d->similarity && d->mode != FSS_MODE_PHARM) ||
      (d->similarity && !(d->tversky_sigma >= 0.f && d->tversky_sigma <= 1.f)))
    return set_error(FSS_ERR_INVALID, "fss_align: similarity must be 0 (Tanimoto) or 1 (Tversky, "
                                      "mode PHARM, tversky_sigma in [0, 1])");
  if (tc && d->lanes_per_pose != 0 && d->lanes_per_pose != 32)
    return set_error(FSS_ERR_INVALID, "fss_align: tensor-core sums use 32 lanes per pose");
  if (d->kernel_variant < 0 || d->kernel_variant > 5 ||
      (pharm && d->kernel_variant > 1) ||
      (combo && (d->kernel_variant == 2 || d->kernel_variant >= 4)))
    return set_error(FSS_ERR_INVALID, "fss_align: kernel_variant must be 0..5 (0 or 1 for "
                                      "modes with a pharmacophore channel, 0, 1 or 3 for "
                                      "ESP_COMBO)");
  // automatic code variant: wide register tile for large clouds, roomy registers for small
  const int var = d->kernel_variant > 0 ? d->kernel_variant - 1
                  : pharm ? 0 : combo ? 2 : (maxM >= 64 ? 1 : 2);
  int lpp = tc ? 32 : d->lanes_per_pose, chunks = d->chunks;
  // the ESP comparison splits surface points over the lanes, so it sizes the lanes
  auto_tile(d->mode, combo ? std::max(maxNs, maxMs) : shape ? maxM : maxMp, d->n_starts, &lpp,
            &chunks);
  if (chunks < 1 || chunks > d->n_starts)
    return set_error(FSS_ERR_INVALID, "fss_align: chunks must be in [1, n_starts]");
  const int ppc = (d->n_starts + chunks - 1) / chunks;
  const int threads = ((ppc * lpp + 31) / 32) * 32;
  if (threads > kMaxThreads)
    return set_error(FSS_ERR_INVALID, "fss_align: too many starts per CTA for lanes_per_pose");
  // every start block must be non-empty
  chunks = (d->n_starts + ppc - 1) / ppc;

  AlignParams p{};
  p.mode = d->mode; p.n_pairs = d->n_pairs; p.n_starts = d->n_starts; p.steps = d->steps;
  p.chunks = chunks; p.n_items = d->n_pairs * chunks;
  p.maxN = maxN; p.maxM = maxM; p.maxNp = maxNp; p.maxMp = maxMp;
  p.pair_ref = d->pair_ref; p.pair_fit = d->pair_fit; p.order = d->order;
  p.ref_pts = reinterpret_cast<const float4*>(d->ref_pts); p.ref_off = d->ref_off;
  p.fit_pts = reinterpret_cast<const float4*>(d->fit_pts); p.fit_off = d->fit_off;
  p.ref_self = d->ref_self; p.fit_self = d->fit_self;
  p.ref_anc = reinterpret_cast<const float4*>(d->ref_anc);
  p.ref_vec = reinterpret_cast<const float4*>(d->ref_vec); p.ref_ph_off = d->ref_ph_off;
  p.fit_anc = reinterpret_cast<const float4*>(d->fit_anc);
  p.fit_vec = reinterpret_cast<const float4*>(d->fit_vec); p.fit_ph_off = d->fit_ph_off;
  p.ref_self_ph = d->ref_self_ph; p.fit_self_ph = d->fit_self_ph;
  p.seed_q = d->seed_q; p.seed_t = d->seed_t;
  const double alpha = shape ? (double)d->alpha : 1.0;
  p.alpha = (float)alpha;
  p.k = (float)(0.5 * alpha * 1.4426950408889634);
  p.e = (float)((double)d->inv_lam * 1.4426950408889634);
  p.inv2k = (float)(1.0 / (alpha * 1.4426950408889634));
  p.Kc = (float)(std::pow(M_PI, 1.5) / std::pow(2.0 * alpha, 1.5));
  p.aKc = (float)(alpha * std::pow(M_PI, 1.5) / std::pow(2.0 * alpha, 1.5));
  p.w = d->color_weight; p.lr = d->lr;
  p.sigma = d->similarity == 1 ? d->tversky_sigma : -1.f;
  if (combo) {
    p.ref_atoms = reinterpret_cast<const float4*>(d->ref_atoms); p.ref_radii = d->ref_radii;
    p.ref_atom_off = d->ref_atom_off;
    p.fit_atoms = reinterpret_cast<const float4*>(d->fit_atoms); p.fit_radii = d->fit_radii;
    p.fit_atom_off = d->fit_atom_off;
    p.ref_surf = reinterpret_cast<const float4*>(d->ref_surf); p.ref_surf_off = d->ref_surf_off;
    p.fit_surf = reinterpret_cast<const float4*>(d->fit_surf); p.fit_surf_off = d->fit_surf_off;
    p.maxNa = maxNa; p.maxMa = maxMa; p.maxNs = maxNs; p.maxMs = maxMs;
    p.coulomb = d->coulomb; p.probe = d->probe_radius;
    p.nkl = (float)(-(double)d->esp_inv_lam * 1.4426950408889634);
    p.esp_w = d->esp_weight;
    p.esp_stride = d->esp_stride > 0 ? d->esp_stride : 1;
  }
  p.fit_f16 = d->fit_f16;
  p.tab = make_pharm_tables(d->mode != FSS_MODE_SHAPE_COLOR);
  p.row_score = d->row_score; p.row_q = d->row_q; p.row_t = d->row_t;
  p.counter = d->scratch;

  const size_t nb = ((size_t)maxN + 7) / 8;
  const size_t smem = sizeof(float) * kColdFields * (size_t)threads +
      (acc == 2 ? sizeof(float2) * kTceF2PerBlock * nb + sizeof(float4) * maxM + 16
       : tc ? sizeof(float4) * (kMmaP4PerBlock * nb + maxM) +
               sizeof(float2) * (kMmaC2PerBlock + kMmaQ2PerBlock) * nb + 16
         : sizeof(float4) * (2 * (size_t)maxN + maxM + 2 * (size_t)maxNp + 2 * (size_t)maxMp) +
               sizeof(float2) * (d->mode == FSS_MODE_ESP ? (size_t)maxN : 0) +
               sizeof(float4) * ((size_t)maxNs + maxMs + 2 * ((size_t)maxNa + maxMa)) +
               sizeof(float2) * ((size_t)maxNa + maxMa) + 16);
  int rc;
  switch (d->mode) {
    case FSS_MODE_SHAPE: rc = launch_align_shape(lpp, acc, var, p, threads, d->cta_per_sm, smem, st); break;
    case FSS_MODE_ESP: rc = launch_align_esp(lpp, acc, var, p, threads, d->cta_per_sm, smem, st); break;
    case FSS_MODE_ESP_COMBO:
      rc = launch_align_combo(lpp, var, p, threads, d->cta_per_sm, smem, st);
      break;
    default:
      rc = launch_align_pharm(d->mode, lpp, d->pharm_extended, p, threads, d->cta_per_sm, smem,
                              st);
      break;
  }
  if (rc != FSS_OK) return rc;
  if (d->out_score && d->out_q && d->out_t)
    return pick_best_launch(d->row_score, d->row_q, d->row_t, d->n_pairs, d->n_starts,
                            d->out_score, d->out_q, d->out_t, st);
  return FSS_OK;
}

int pick_best_launch(const float* rs, const float* rq, const float* rt, int P, int S, float* os,
                     float* oq, float* ot, cudaStream_t st) {
  if (P < 0 || S <= 0 || !rs || !rq || !rt || !os || !oq || !ot)
    return set_error(FSS_ERR_INVALID, "fss_pick_best: bad arguments");
  if (P == 0) return FSS_OK;
  pick_best_kernel<<<(P + 255) / 256, 256, 0, st>>>(rs, rq, rt, P, S, os, oq, ot);
  return check_launch("fss_pick_best");
}

int self_overlap_launch(const float* pts, const int32_t* off, int n_mol, int max_n, float alpha,
                        int esp, float inv_lam, int f16, float* out, cudaStream_t st) {
  if (n_mol < 0 || !pts || !off || !out || !(alpha > 0.f))
    return set_error(FSS_ERR_INVALID, "fss_self_overlap: bad arguments");
  if (max_n > kMaxPoints) return set_error(FSS_ERR_UNSUPPORTED, "fss_self_overlap: molecule too large");
  if (n_mol == 0) return FSS_OK;
  const double a = alpha;
  const float k = (float)(0.5 * a * 1.4426950408889634);
  const float e = (float)((double)inv_lam * 1.4426950408889634);
  const float inv2k = (float)(1.0 / (a * 1.4426950408889634));
  const float Kc = (float)(std::pow(M_PI, 1.5) / std::pow(2.0 * a, 1.5));
  const size_t smem = sizeof(float4) * 3 * (size_t)max_n + sizeof(float2) * (size_t)max_n + 16;
  cudaError_t ce;
  if (esp) {
    ce = cudaFuncSetAttribute(self_overlap_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      self_overlap_kernel<true><<<n_mol, 32, smem, st>>>(Pts(pts, f16), off, n_mol, max_n, k, e, inv2k, Kc, out);
  } else {
    ce = cudaFuncSetAttribute(self_overlap_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess)
      self_overlap_kernel<false><<<n_mol, 32, smem, st>>>(Pts(pts, f16), off, n_mol, max_n, k, 0.f, inv2k, Kc, out);
  }
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_self_overlap: ") + cudaGetErrorString(ce));
  return check_launch("fss_self_overlap");
}

int pharm_self_launch(const float* anc, const float* vec, const int32_t* off, int n_mol, int max_n,
                      int directional, int extended, int f16, float* out, cudaStream_t st) {
  if (n_mol < 0 || !anc || !off || !out || (directional && !vec))
    return set_error(FSS_ERR_INVALID, "fss_pharm_self_overlap: bad arguments");
  if (extended < 0 || extended > 2 || (extended && !directional))
    return set_error(FSS_ERR_INVALID, "fss_pharm_self_overlap: extended must be 0, 1 or 2 "
                                      "(directional tables)");
  if (max_n > kMaxPoints) return set_error(FSS_ERR_UNSUPPORTED, "fss_pharm_self_overlap: molecule too large");
  if (n_mol == 0) return FSS_OK;
  const size_t smem = sizeof(float4) * 4 * (size_t)max_n + 16;
  auto kern = extended == 1 ? pharm_self_kernel<1>
              : extended == 2 ? pharm_self_kernel<2> : pharm_self_kernel<0>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) return set_error(FSS_ERR_CUDA, std::string("fss_pharm_self_overlap: ") + cudaGetErrorString(ce));
  kern<<<n_mol, 32, smem, st>>>(Pts(anc, f16), Pts(vec, f16), off, n_mol, max_n,
                                make_pharm_tables(directional != 0), out);
  return check_launch("fss_pharm_self_overlap");
}

}  // namespace fss
