/*
 * fss_cuda.h -- C ABI of libfss_cuda.so, the sm_100a (B200) backend of fast_shepherd_score_b200.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t passed as void*
 * (NULL = legacy default stream), launches asynchronously on that stream, and returns an
 * int status (FSS_OK or an FSS_ERR_* code; fss_last_error() gives the message of the
 * calling thread's last failure).  Nothing here allocates or frees caller memory.
 *
 * Array conventions
 *   float4 clouds      points packed as (x, y, z, w), 16-byte aligned; w = per-point charge
 *                      (ESP) or 0.  Pharmacophore anchors carry the int32 type in w's bits,
 *                      vectors are (x, y, z, 0).
 *   offsets            int32 (n_mol + 1) prefix offsets into a packed cloud array.
 *   padded (AoS)       the reference's (K, N_pad, 3) float32 layout with int32 real counts.
 *   q, t               quaternion (w, x, y, z) and translation; the fit cloud moves:
 *                      aligned = R(q) fit + t (row-vector form: fit @ R^T + t).
 *
 * Each declaration cites the reference (shepherd_score) interface it replaces.
 */
#ifndef FSS_CUDA_H
#define FSS_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FSS_ABI_VERSION 3

enum fss_status {
  FSS_OK = 0,
  FSS_ERR_INVALID = 1,     /* bad argument: maps to ValueError (reference ValueErrors) */
  FSS_ERR_CUDA = 2,        /* CUDA runtime / launch failure: RuntimeError */
  FSS_ERR_NOMEM = 3,       /* device allocation failure: MemoryError (caller halves the batch) */
  FSS_ERR_UNSUPPORTED = 4, /* size beyond a documented limit */
  FSS_ERR_TIMEOUT = 5      /* a bounded device-side wait gave up (status word set) */
};

enum fss_mode {
  FSS_MODE_SHAPE = 0,      /* vol / surf: Gaussian shape Tanimoto */
  FSS_MODE_ESP = 1,        /* vol_esp / surf_esp: charge-weighted shape Tanimoto */
  FSS_MODE_PHARM = 2,      /* pharm: directional typed pharmacophore Tanimoto */
  FSS_MODE_SHAPE_PHARM = 3,/* (1-w) shape + w directional pharm, one shared pose */
  FSS_MODE_SHAPE_COLOR = 4,/* vol_color: (1-w) shape + w directionless colour */
  FSS_MODE_ESP_COMBO = 5   /* vol_and_surf_esp: pose steered by the shape gradient, score
                            * w * ShaEP ESP comparison + (1-w) shape Tanimoto
                            * (accel/drivers/esp_combo.py:334-595) */
};

/* Library identification. */
int fss_abi_version(void);
const char *fss_last_error(void);
/* Largest point / feature count per molecule the fused kernels stage in shared memory. */
int fss_max_points(void);

/* ---------------------------------------------------------------------------------------
 * Single evaluation: overlap value + SE(3) gradient for K poses, padded AoS inputs.
 * Replaces overlap_score_grad_se3_batch (accel/kernels/shape_triton.py:191-249) when
 * CA == CB == NULL, and overlap_score_grad_esp_se3_batch (accel/kernels/esp_triton.py:174-262)
 * when charges are given (inv_lam = 1/lam, lam as the reference kernel receives it).
 * A (K,N_pad,3), B (K,M_pad,3), CA (K,N_pad), CB (K,M_pad), q (K,4), t (K,3),
 * N_real/M_real (K) int32 (NULL = fully real).  Outputs V (K), dQ (K,4) = dV/dq,
 * dT (K,3) = dV/dt; dQ/dT untouched when need_grad == 0.
 * ------------------------------------------------------------------------------------- */
int fss_overlap_grad(const float *A, const float *B, const float *CA, const float *CB,
                     const float *q, const float *t, const int32_t *N_real,
                     const int32_t *M_real, int32_t K, int32_t N_pad, int32_t M_pad,
                     float alpha, float inv_lam, int32_t need_grad, float *V, float *dQ,
                     float *dT, void *stream);

/* Typed pharmacophore overlap + dO/dq, dO/dt for K poses, padded AoS inputs.
 * directional = 1 replaces pharm_grad_dq_se3_batch (accel/kernels/pharm_triton.py:403-467);
 * directional = 0 replaces pharm_color_score_grad_se3_batch (pharm_triton.py:254-293,
 * directionless lookup tables).  Types int32 in 0..8 (8 = Dummy, skipped); RV/FV may be NULL
 * when directional == 0. */
int fss_pharm_grad(const float *A, const float *B, const float *RV, const float *FV,
                   const int32_t *At, const int32_t *Bt, const float *q, const float *t,
                   const int32_t *N_real, const int32_t *M_real, int32_t K, int32_t N_pad,
                   int32_t M_pad, int32_t directional, int32_t need_grad, float *O, float *dQ,
                   float *dT, void *stream);

/* One fine-loop step for K pose rows from already computed overlap value/gradients:
 * Tanimoto score, pre-update best tracking and tangent-projected Adam with renormalisation.
 * Replaces _GraphedFineSurf._tanimoto_adam_tail + fused_adam_qt_with_tangent_proj
 * (accel/drivers/shape.py:114-130, accel/kernels/shape_triton.py:383-406).
 * U (K) = V_AA + V_BB.  All state arrays are updated in place. */
int fss_tanimoto_adam_step(const float *V, const float *dQ, const float *dT, const float *U,
                           float *q, float *t, float *mq, float *vq, float *mt, float *vt,
                           float *best, float *bq, float *bt, int32_t K, float lr,
                           void *stream);

/* ---------------------------------------------------------------------------------------
 * Packed clouds (float4 + offsets) used by the fused alignment and the screening server.
 * ------------------------------------------------------------------------------------- */

/* Point formats.  A packed cloud is float32 (x, y, z, w) per point, 16 bytes.  Where an
 * argument is marked "f16-capable", a flag selects float16 (x, y, z, w) points instead,
 * 8 bytes each (a screening library kept in float16 on the device, as the ProfileStore
 * format's default dtype stores it); the kernels widen them to float32 in their staging
 * loads.  Pharmacophore anchors in float16 carry the type as a float16 value in w (float32
 * anchors carry the int32 type in w's bits); vectors are (vx, vy, vz, 0) in either format. */

/* Self overlap per molecule at the identity pose (shape, or ESP when esp != 0 with
 * inv_lam = 1/lam).  Replaces _batch_self_overlap / _batch_self_overlap_esp
 * (shape_triton.py:436-448, esp_triton.py:393-425).  out (n_mol); max_points bounds every
 * molecule's count (a larger molecule gets NaN).  pts is f16-capable (pts_f16 = 1). */
int fss_self_overlap(const float *pts, const int32_t *off, int32_t n_mol, int32_t max_points,
                     float alpha, int32_t esp, float inv_lam, int32_t pts_f16, float *out,
                     void *stream);

/* Pharmacophore self overlap per molecule (directional or colour tables); `extended` 0/1/2
 * as fss_align_desc.pharm_extended (directional tables only).
 * Replaces the identity-pose self overlaps of accel/drivers/pharm.py:336-346 and
 * batch_pharm_self_overlap (accel/drivers/pharm_overlap.py:413-439).  anc and vec are
 * f16-capable (pts_f16 = 1). */
int fss_pharm_self_overlap(const float *anc, const float *vec, const int32_t *off,
                           int32_t n_mol, int32_t max_features, int32_t directional,
                           int32_t extended, int32_t pts_f16, float *out, void *stream);

/* Multi-start seeds for P pairs: identity, 4 PCA alignments (fp64 closed-form eigensolver),
 * up to 6 structured +-90 degree axis swaps, then the Fibonacci set `fibo_q` (n_fibo,4)
 * supplied by the caller, each with a COM-aligning translation; degenerate pairs
 * (< 3 points or non-finite) take the fixed fallback set.  Replaces batched_seeds_torch
 * (accel/drivers/_common.py:281-441).  seed_q (P,S,4), seed_t (P,S,3).  fit_pts is
 * f16-capable (fit_f16 = 1). */
int fss_seeds(const float *ref_pts, const int32_t *ref_off, const float *fit_pts,
              const int32_t *fit_off, const int32_t *pair_ref, const int32_t *pair_fit,
              int32_t n_pairs, int32_t n_seeds, const float *fibo_q, int32_t n_fibo,
              int32_t fit_f16, float *seed_q, float *seed_t, void *stream);

/* Descriptor of one fused alignment launch (all pairs x starts x Adam steps). */
typedef struct fss_align_desc {
  int32_t mode;              /* enum fss_mode */
  int32_t n_pairs;
  int32_t n_starts;
  int32_t steps;
  const int32_t *pair_ref;   /* (n_pairs) molecule index into the ref clouds */
  const int32_t *pair_fit;   /* (n_pairs) molecule index into the fit clouds */
  const int32_t *order;      /* (n_pairs) processing order (costliest first) or NULL */
  /* shape / ESP channel */
  const float *ref_pts; const int32_t *ref_off;
  const float *fit_pts; const int32_t *fit_off;
  const float *ref_self; const float *fit_self;       /* per-molecule self overlaps */
  /* pharmacophore channel (modes PHARM, SHAPE_PHARM, SHAPE_COLOR) */
  const float *ref_anc; const float *ref_vec; const int32_t *ref_ph_off;
  const float *fit_anc; const float *fit_vec; const int32_t *fit_ph_off;
  const float *ref_self_ph; const float *fit_self_ph;
  /* seeds (n_pairs, n_starts, 4|3) */
  const float *seed_q; const float *seed_t;
  /* parameters */
  float alpha;               /* Gaussian width of the shape channel */
  float inv_lam;             /* 1/lam for ESP */
  float color_weight;        /* w of the two-channel modes */
  float lr;                  /* Adam learning rate */
  /* per-row results (n_pairs*n_starts [x4|x3]): best score and best (pre-update) pose */
  float *row_score; float *row_q; float *row_t;
  /* per-pair results (argmax over starts, first index on ties) */
  float *out_score; float *out_q; float *out_t;
  /* largest molecule any pair uses, per cloud (sizes the shared-memory tiles; a pair
   * exceeding them is skipped and flagged in scratch[1]) */
  int32_t max_ref_points, max_fit_points, max_ref_features, max_fit_features;
  /* tiling: 0 = choose automatically */
  int32_t lanes_per_pose;    /* 1, 2, 4, 8, 16 or 32 lanes cooperate on one pose */
  int32_t chunks;            /* start blocks per pair (CTA covers n_starts/chunks starts) */
  int32_t cta_per_sm;        /* persistent CTAs per SM */
  int32_t accumulate;        /* where the shape and ESP channels' pairwise work runs:
                              * 0 automatic, 1 FP32 lanes, 2 value/gradient sums on the tensor
                              * cores, 3 exponents on the tensor cores (both tf32 hi/lo split
                              * MMA, one warp per pose; modes SHAPE and ESP) */
  int32_t kernel_variant;    /* code variant of the FP32-lane loop: 0 automatic, 1 base (4 fit
                              * points per lane, 2 CTAs/SM register budget), 2 wide (6 fit
                              * points per lane, deeper unroll), 3 roomy (4 fit points, one
                              * CTA/SM register budget), 4 unrolled (4 fit points, 4x unroll,
                              * 2 CTAs/SM budget), 5 small-molecule tile (8 fit points, one
                              * CTA/SM budget); 2-5 for modes SHAPE and ESP, 3 also for
                              * ESP_COMBO */
  int32_t pharm_extended;    /* mode PHARM: 0 cosine-weighted directional features, 1 extended
                              * points (anchor + unit vector) plus anchors, 2 extended points
                              * only (extended_points / only_extended of
                              * analytical_gradients/_torch.py:223-355) */
  int32_t similarity;        /* mode PHARM: 0 Tanimoto, 1 Tversky */
  float tversky_sigma;       /* Tversky D = sigma V_AA + (1 - sigma) V_BB, sigma in [0, 1]
                              * (accel/drivers/pharm.py:40: tversky 0.95, tversky_ref 1.0,
                              * tversky_fit 0.05) */
  /* ShaEP ESP channel of mode ESP_COMBO: atoms with hydrogens (x, y, z, partial charge) with
   * van der Waals radii, and surface points (x, y, z, ESP at the point), packed per molecule
   * with int32 prefix offsets like the shape clouds (the shape channel uses ref_pts/fit_pts
   * as the volumetric centres) */
  const float *ref_atoms; const float *ref_radii; const int32_t *ref_atom_off;
  const float *fit_atoms; const float *fit_radii; const int32_t *fit_atom_off;
  const float *ref_surf; const int32_t *ref_surf_off;
  const float *fit_surf; const int32_t *fit_surf_off;
  int32_t max_ref_atoms, max_fit_atoms, max_ref_surf, max_fit_surf;
  float esp_inv_lam;         /* 1 / (LAM_SCALING * lam) (esp_triton.py:378) */
  float coulomb;             /* COULOMB_SCALING, score/constants.py:16 */
  float probe_radius;        /* a surface point within radius + probe of an atom is masked */
  float esp_weight;          /* w of the combo score */
  int32_t esp_stride;        /* the combo score is tracked on steps that are multiples of
                              * esp_stride and on the last step (0 or 1: every step) */
  /* scratch: two device int32 -- [0] work counter, [1] status flags (bit 0: a pair was
   * larger than the max_* extents).  The launch zeroes both on `stream`. */
  int32_t *scratch;
  /* 1: fit_pts, fit_anc and fit_vec are float16 points (f16-capable, see "Point formats");
   * not in mode ESP_COMBO.  0: float32. */
  int32_t fit_f16;
} fss_align_desc;

/* Fused persistent alignment: every (pair, start) pose runs all `steps` Adam steps inside
 * one kernel with the clouds of its pair staged in shared memory, then a pick kernel takes
 * the per-pair argmax.  Replaces coarse_fine_align_many (accel/drivers/shape.py:155-313),
 * coarse_fine_esp_align_many (accel/drivers/esp.py:139-367), the pharm fine loop
 * (accel/drivers/pharm.py:123-517) and coarse_fine_vol_color_align_many
 * (accel/drivers/vol_color.py:199-518) with early stop disabled (fixed step count). */
int fss_align(const fss_align_desc *desc, void *stream);

/* Allocation-free variant of fss_align.  It has no counterpart in the reference: it is for
 * callers that cannot allocate device memory where they align (a host runtime that only
 * hands over input and output buffers, code inside another framework's memory pool, or a
 * latency-critical loop that must not call cudaMalloc).  The descriptor is read as for
 * fss_align except that row_score/row_q/row_t and scratch are ignored (may be NULL): the
 * per-(pair, start) rows and the work counter live in one library-owned __device__ array
 * of FSS_STATIC_MAX_ROWS rows (about 4 MiB per device, held until the process exits), so
 * n_pairs * n_starts above FSS_STATIC_MAX_ROWS is rejected with FSS_ERR_UNSUPPORTED.
 * out_score/out_q/out_t are required.  The first call on a device (and the first after a
 * cudaDeviceReset, which gives the device a new context) resolves the array's address
 * (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture.  All calls share the array, so calls that overlap on the GPU race.  A pair
 * larger than the declared max_* extents returns a NaN score; when `scratch` is not NULL it
 * is read as ONE device int32 that receives the call's status flags (as fss_align's
 * scratch[1]: bit 0 set when a pair exceeded the extents), copied on `stream` after the
 * launch. */
#define FSS_STATIC_MAX_ROWS 131072
int fss_align_static(const fss_align_desc *desc, void *stream);

/* Per-pair argmax over starts of row results (shape.py:306-313). */
int fss_pick_best(const float *row_score, const float *row_q, const float *row_t,
                  int32_t n_pairs, int32_t n_starts, float *out_score, float *out_q,
                  float *out_t, void *stream);

/* ---------------------------------------------------------------------------------------
 * Differentiable scoring (coordinate / charge adjoint).
 * Replaces torch autograd through get_overlap / get_overlap_esp
 * (score/gaussian_overlap.py:73, score/electrostatic_scoring.py:69) for P pairs of packed
 * clouds: score_p = V_AB / (V_AA + V_BB - V_AB).  Forward writes score (P) and the three
 * overlaps (P,3) = (V_AB, V_AA, V_BB).  Backward takes d(loss)/d(score) (P) and ADDS
 * d(loss)/d(coords) into grad_ref / grad_fit (float4 arrays aligned with the inputs,
 * w = d/d(charge); zero them first -- molecules shared by several pairs accumulate).  Either
 * grad_ref or grad_fit (not both) may be NULL: that side's adjoint is then not computed.
 * esp != 0 adds the charge factor exp(-(c_i-c_j)^2 * inv_lam).  max_*_points bound the
 * molecules' sizes (a larger pair gets a NaN score and no gradient).
 * ------------------------------------------------------------------------------------- */
int fss_score_fwd(const float *ref_pts, const int32_t *ref_off, const float *fit_pts,
                  const int32_t *fit_off, const int32_t *pair_ref, const int32_t *pair_fit,
                  int32_t n_pairs, int32_t max_ref_points, int32_t max_fit_points, float alpha,
                  int32_t esp, float inv_lam, float *score, float *overlaps, void *stream);
int fss_score_bwd(const float *ref_pts, const int32_t *ref_off, const float *fit_pts,
                  const int32_t *fit_off, const int32_t *pair_ref, const int32_t *pair_fit,
                  int32_t n_pairs, int32_t max_ref_points, int32_t max_fit_points, float alpha,
                  int32_t esp, float inv_lam, const float *overlaps, const float *grad_score,
                  float *grad_ref, float *grad_fit, void *stream);

/* Dense-batch form of fss_score_fwd / fss_score_bwd for the reference's padded tensors: ref
 * molecule b is ref_xyz[b, 0:ref_points, :] of a (B_ref, ref_points, 3) array (every point
 * real) with charges ref_q[b, :] (B_ref, ref_points) when esp != 0 (NULL otherwise); likewise
 * the fit side.  Same math as get_overlap / get_overlap_esp (score/gaussian_overlap.py:62-117,
 * score/electrostatic_scoring.py:17-120) without packing.  Backward ADDS d(loss)/d(coords)
 * into grad_*_xyz (same shapes as the inputs) and d(loss)/d(charges) into grad_*_q (may be
 * NULL when esp == 0).  A NULL grad_ref_xyz or grad_fit_xyz (not both) skips that side. */
int fss_score_fwd_dense(const float *ref_xyz, const float *ref_q, int32_t ref_points,
                        const float *fit_xyz, const float *fit_q, int32_t fit_points,
                        const int32_t *pair_ref, const int32_t *pair_fit, int32_t n_pairs,
                        float alpha, int32_t esp, float inv_lam, float *score, float *overlaps,
                        void *stream);
int fss_score_bwd_dense(const float *ref_xyz, const float *ref_q, int32_t ref_points,
                        const float *fit_xyz, const float *fit_q, int32_t fit_points,
                        const int32_t *pair_ref, const int32_t *pair_fit, int32_t n_pairs,
                        float alpha, int32_t esp, float inv_lam, const float *overlaps,
                        const float *grad_score, float *grad_ref_xyz, float *grad_ref_q,
                        float *grad_fit_xyz, float *grad_fit_q, void *stream);

/* Forward with adjoint moments (no counterpart in the reference, which differentiates
 * get_overlap / get_overlap_esp by torch autograd): as fss_score_fwd_dense (with both moments
 * pointers NULL it computes only the scores and overlaps), and in the same pass, for each
 * side whose moments pointer is non-NULL, writes per pair p and point k of that side two
 * float4 rows (x, y, z, charge):
 *   moments[8 (p * points + k) + 0..3] = sum over the other cloud's points y of g (x_k - y)
 *   moments[8 (p * points + k) + 4..7] = sum over the own cloud's points y of g (x_k - y)
 * (charge component g (c_k - c_y)); ref_moments is (n_pairs, ref_points, 8) floats,
 * fit_moments (n_pairs, fit_points, 8).  fss_score_bwd_moments_dense then turns them into the
 * gradients without a second pass over the pairs.  The overlaps may differ from
 * fss_score_fwd_dense's in the last bits (other summation order).  Both clouds are staged in
 * shared memory at 48 bytes a point: when 48 (ref_points + fit_points) + 16 bytes exceed the
 * device's per-block limit the call returns FSS_ERR_UNSUPPORTED and writes nothing (the
 * two-pass fss_score_fwd_dense / fss_score_bwd_dense handle those sizes). */
int fss_score_fwd_moments_dense(const float *ref_xyz, const float *ref_q, int32_t ref_points,
                                const float *fit_xyz, const float *fit_q, int32_t fit_points,
                                const int32_t *pair_ref, const int32_t *pair_fit,
                                int32_t n_pairs, float alpha, int32_t esp, float inv_lam,
                                float *score, float *overlaps, float *ref_moments,
                                float *fit_moments, void *stream);
/* ADDS into grad_* what fss_score_bwd_dense adds, from the forward's overlaps and moments, for
 * each side whose moments and grad_*_xyz are both non-NULL (grad_*_q may be NULL when
 * esp == 0).  Same expressions as fss_score_bwd_dense, so equal moments and overlaps give
 * bit-identical gradients.  Bit 0 (ref) / bit 1 (fit) of `overwrite` STORE that side's
 * gradients instead of adding them (no zeroing needed): only valid when every molecule of the
 * side belongs to exactly one pair. */
int fss_score_bwd_moments_dense(const int32_t *pair_ref, const int32_t *pair_fit,
                                int32_t n_pairs, int32_t ref_points, int32_t fit_points,
                                float alpha, int32_t esp, float inv_lam, const float *overlaps,
                                const float *grad_score, const float *ref_moments,
                                const float *fit_moments, float *grad_ref_xyz,
                                float *grad_ref_q, float *grad_fit_xyz, float *grad_fit_q,
                                int32_t overwrite, void *stream);

/* ---------------------------------------------------------------------------------------
 * Roof probe (measurement support, no reference counterpart): launches a throughput kernel
 * of `which` = 0 (ex2 on the MUFU pipe) or 1 (FP32 FMA) with `blocks_per_sm` CTAs of 256
 * threads per SM, each thread running `iters` x 8 independent operations; *ops receives the
 * operation count so ops / elapsed time is the device's measured rate.  `out` (grid floats)
 * is never written in practice; it keeps the work observable to the compiler.
 * ------------------------------------------------------------------------------------- */
int fss_probe_peak(int32_t which, int32_t iters, int32_t blocks_per_sm, float *out,
                   long long *ops, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FSS_CUDA_H */
