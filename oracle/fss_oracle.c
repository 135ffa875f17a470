/*
 * fss_oracle.c -- CPU restatement of the reference's batched alignment path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline; the product (fast_shepherd_score_b200) never links or calls it.
 *
 * It restates, function by function, the numba CPU twins the reference runs when
 * its batched aligners get CPU tensors (shepherd_score/accel/kernels/cpu.py and
 * shepherd_score/accel/kernels/cpu_fused.py):
 *
 *   fsso_overlap_grad   <- cpu.py:38-87   (_overlap_grad_kernel)
 *                          cpu.py:158-200 (_overlap_grad_esp_kernel, when CA/CB given)
 *   fsso_pharm_dq       <- cpu.py:500-582 (_pharm_grad_dq_kernel, directional pharm)
 *   fsso_pharm_color    <- cpu.py:412-458 (_pharm_color_grad_kernel, directionless)
 *   tail_tanimoto       <- cpu_fused.py:54-108  (_tail_tanimoto)
 *   pose_pharm ext!=0   <- analytical_gradients/_torch.py:223-355 (extended_points /
 *                          only_extended of compute_overlap_and_grad_pharm)
 *   tail_tversky        <- accel/drivers/pharm.py:417-426 + pharm_overlap.py:36-59
 *   esp_compare         <- cpu.py:237-261 (_esp_comparison_kernel, ShaEP ESP comparison)
 *   fsso_esp_combo_loop <- accel/drivers/esp_combo.py:497-595 (vol_and_surf_esp fine loop)
 *   tail_combo          <- cpu_fused.py:111-167 (_tail_vol_color)
 *   fsso_fine_loop      <- cpu_fused.py:179-217 (fine_loop_cpu) + the per-mode glue
 *                          cpu_fused.py:225-338
 *
 * Precision follows the numba code: every overlap sum is accumulated in double and
 * rounded to float at the kernel boundary (the `.astype(np.float32)` in
 * cpu_fused.py:242); the optimiser state (q, t, Adam moments, best pose) is float
 * and each tail update is evaluated in double and stored as float, as numba does
 * when a float64 constant (beta1, beta2, eps) meets a float32 array element.
 * exp() is the C library exp, the same routine numba's math.exp lowers to.
 *
 * Poses are independent unless the batch-global early stop is on, so with early
 * stop disabled the loop runs pose-major (all steps of one pose, then the next),
 * which is bit-identical to the step-major order and parallelises over poses on
 * pthreads.  With early stop on it runs step-major exactly as fine_loop_cpu does.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

/* Minimal dynamic parallel-for over [0, n) on `nthreads` pthreads (the build image's
 * gcc has no usable OpenMP spec, so the oracle carries its own). */
typedef void (*range_fn)(void *ctx, int i);
typedef struct { range_fn fn; void *ctx; int n; int chunk; int next; pthread_mutex_t mu; } pfor_t;

static void *pfor_worker(void *arg) {
    pfor_t *p = (pfor_t *)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        const int i0 = p->next;
        p->next += p->chunk;
        pthread_mutex_unlock(&p->mu);
        if (i0 >= p->n) break;
        const int i1 = i0 + p->chunk < p->n ? i0 + p->chunk : p->n;
        for (int i = i0; i < i1; ++i) p->fn(p->ctx, i);
    }
    return NULL;
}

static void parallel_for(int n, int nthreads, int chunk, range_fn fn, void *ctx) {
    if (nthreads <= 1 || n <= 1) {
        for (int i = 0; i < n; ++i) fn(ctx, i);
        return;
    }
    if (nthreads > 256) nthreads = 256;
    pfor_t p = {fn, ctx, n, chunk > 0 ? chunk : 1, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t th[256];
    int started = 0;
    for (int i = 0; i < nthreads - 1; ++i)
        if (pthread_create(&th[started], NULL, pfor_worker, &p) == 0) ++started;
    pfor_worker(&p);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
}

#define B1 0.9
#define B2 0.999
#define ADAM_EPS 1e-8

/* Precision of the per-pose overlap sums.  The default build (libfss_oracle.so) evaluates
 * them in double as numba does.  Built with -DFSSO_ACC32 (libfss_oracle_f32.so), the terms,
 * exp and every accumulation of pose_overlap / pose_pharm run in float instead -- the
 * precision of the reference's Triton kernels, which accumulate their tiles in fp32
 * (accel/kernels/shape_triton.py:114-177, pharm_triton.py:296-400).  Comparing the two
 * builds measures how far two correct precisions of the same algorithm drift apart over a
 * fine loop; the parity tests use it as the floor for the CUDA path's own drift. */
#define ACC(x) ((acc_t)(x))
#ifdef FSSO_ACC32
typedef float acc_t;
#define ACC_EXP expf
#define ACC_ABS fabsf
#else
typedef double acc_t;
#define ACC_EXP exp
#define ACC_ABS fabs
#endif

enum { FSSO_SHAPE = 0, FSSO_ESP = 1, FSSO_PHARM = 2, FSSO_COMBO = 3, FSSO_COLOR_COMBO = 4 };

static const double K_PI15 = 5.568327996831708; /* pi ** 1.5 */

/* Rotation matrix from a (w,x,y,z) quaternion, as cpu.py:56-58 (q assumed unit). */
static inline void rotmat(const float *q, acc_t R[9]) {
    const float qr = q[0], qi = q[1], qj = q[2], qk = q[3];
    R[0] = ACC(1.0) - ACC(2.0) * (acc_t)(qj * qj + qk * qk);
    R[1] = ACC(2.0) * (acc_t)(qi * qj - qk * qr);
    R[2] = ACC(2.0) * (acc_t)(qi * qk + qj * qr);
    R[3] = ACC(2.0) * (acc_t)(qi * qj + qk * qr);
    R[4] = ACC(1.0) - ACC(2.0) * (acc_t)(qi * qi + qk * qk);
    R[5] = ACC(2.0) * (acc_t)(qj * qk - qi * qr);
    R[6] = ACC(2.0) * (acc_t)(qi * qk - qj * qr);
    R[7] = ACC(2.0) * (acc_t)(qj * qk + qi * qr);
    R[8] = ACC(1.0) - ACC(2.0) * (acc_t)(qi * qi + qj * qj);
}

/* d(R(q) b)/dq contracted with a force f, body-frame point b (cpu.py:80-83). */
static inline void quat_tail(const acc_t f[3], acc_t bx, acc_t by, acc_t bz,
                             const float *q, acc_t dQ[4]) {
    const acc_t qr = q[0], qi = q[1], qj = q[2], qk = q[3];
    const acc_t fx = f[0], fy = f[1], fz = f[2];
    dQ[0] += fx * (-ACC(2.0) * qk * by + ACC(2.0) * qj * bz) + fy * (ACC(2.0) * qk * bx - ACC(2.0) * qi * bz)
           + fz * (-ACC(2.0) * qj * bx + ACC(2.0) * qi * by);
    dQ[1] += fx * (ACC(2.0) * qj * by + ACC(2.0) * qk * bz) + fy * (ACC(2.0) * qj * bx - ACC(4.0) * qi * by - ACC(2.0) * qr * bz)
           + fz * (ACC(2.0) * qk * bx + ACC(2.0) * qr * by - ACC(4.0) * qi * bz);
    dQ[2] += fx * (-ACC(4.0) * qj * bx + ACC(2.0) * qi * by + ACC(2.0) * qr * bz) + fy * (ACC(2.0) * qi * bx + ACC(2.0) * qk * bz)
           + fz * (-ACC(2.0) * qr * bx + ACC(2.0) * qk * by - ACC(4.0) * qj * bz);
    dQ[3] += fx * (-ACC(4.0) * qk * bx - ACC(2.0) * qr * by + ACC(2.0) * qi * bz) + fy * (ACC(2.0) * qr * bx - ACC(4.0) * qk * by + ACC(2.0) * qj * bz)
           + fz * (ACC(2.0) * qi * bx + ACC(2.0) * qj * by);
}

/* One pose of the shape / ESP overlap with its SE(3) gradient.
 * A (N,3) ref, B (M,3) fit, optional charges CA (N) / CB (M) (ESP when non-NULL).
 * Mirrors cpu.py:52-86 and cpu.py:166-199. */
static void pose_overlap(const float *A, const float *B, const float *CA, const float *CB,
                         const float *q, const float *t, int n_real, int m_real,
                         double alpha_d, double inv_lam_d, int need_grad,
                         double *V, double dQ_out[4], double dT_out[3]) {
    const acc_t alpha = (acc_t)alpha_d, inv_lam = (acc_t)inv_lam_d;
    acc_t dQ[4], dT[3];
    const acc_t Kc = (acc_t)K_PI15 / (acc_t)pow(ACC(2.0) * (double)alpha, ACC(1.5));
    const acc_t a2 = alpha / ACC(2.0);
    acc_t R[9];
    rotmat(q, R);
    const acc_t tx = t[0], ty = t[1], tz = t[2];
    acc_t Vacc = ACC(0.0);
    dT[0] = dT[1] = dT[2] = ACC(0.0);
    dQ[0] = dQ[1] = dQ[2] = dQ[3] = ACC(0.0);
    for (int m = 0; m < m_real; ++m) {
        const acc_t bx0 = B[3 * m], by0 = B[3 * m + 1], bz0 = B[3 * m + 2];
        const acc_t bx = R[0] * bx0 + R[1] * by0 + R[2] * bz0 + tx;
        const acc_t by = R[3] * bx0 + R[4] * by0 + R[5] * bz0 + ty;
        const acc_t bz = R[6] * bx0 + R[7] * by0 + R[8] * bz0 + tz;
        acc_t f[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};
        const float cbm = CB ? CB[m] : 0.0f;
        for (int n = 0; n < n_real; ++n) {
            const acc_t dx = A[3 * n] - bx, dy = A[3 * n + 1] - by, dz = A[3 * n + 2] - bz;
            const acc_t r2 = dx * dx + dy * dy + dz * dz;
            acc_t g;
            if (CA) {
                const float dc = CA[n] - cbm; /* float32 subtraction, as numba */
                g = Kc * ACC_EXP(-a2 * r2 - (acc_t)(dc * dc) * inv_lam);
            } else {
                g = Kc * ACC_EXP(-a2 * r2);
            }
            Vacc += g;
            if (need_grad) {
                const acc_t c = alpha * g;
                f[0] += c * dx; f[1] += c * dy; f[2] += c * dz;
            }
        }
        if (need_grad) {
            dT[0] += f[0]; dT[1] += f[1]; dT[2] += f[2];
            quat_tail(f, bx0, by0, bz0, q, dQ);
        }
    }
    *V = Vacc;
    for (int c = 0; c < 4; ++c) dQ_out[c] = dQ[c];
    for (int c = 0; c < 3; ++c) dT_out[c] = dT[c];
}

/* Unit vector with the ACC(1e-12) norm floor of cpu.py:524-526. */
static inline void unit_vec(const float *v, acc_t out[3]) {
    const float nrm = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const acc_t inv = ACC(1.0) / (nrm > 1e-12f ? (acc_t)nrm : ACC(1e-12));
    out[0] = v[0] * inv; out[1] = v[1] * inv; out[2] = v[2] * inv;
}

/* One pose of the typed pharmacophore overlap with in-register dO/dq (cpu.py:506-581).
 * A/B anchors, RV/FV vectors, At/Bt int32 types; alphas/Ks/cats are the 9-entry
 * lookup tables.  directional==0 gives the directionless colour kernel (cpu.py:418-457),
 * which is the directional one with every real type in category 0.
 * ext: 0 cosine weights; 1 extended points -- acceptor and donor pairs get anchor weight 1
 * plus a Gaussian between the extended points anchor + unit vector; 2 extended points only
 * (anchor weight 0).  The extended types are EXTENDED_POINT_TYPES = {acceptor, donor} of
 * the typed overlap the batched fine loop differentiates (accel/drivers/pharm_overlap.py:33,
 * :185-200); halogen keeps its cosine weight. */
static void pose_pharm(const float *A, const float *B, const float *RV, const float *FV,
                       const int32_t *At, const int32_t *Bt, const float *q, const float *t,
                       int n_real, int m_real, const double *alphas, const double *Ks,
                       const int32_t *cats, int ext, int need_grad,
                       double *O, double dQ_out[4], double dT_out[3]) {
    acc_t dQ[4], dT[3];
    acc_t R[9];
    rotmat(q, R);
    const acc_t tx = t[0], ty = t[1], tz = t[2];
    acc_t Oacc = ACC(0.0);
    dT[0] = dT[1] = dT[2] = ACC(0.0);
    dQ[0] = dQ[1] = dQ[2] = dQ[3] = ACC(0.0);
    for (int i = 0; i < m_real; ++i) {
        const int ityp = Bt[i];
        const int icat = cats[ityp];
        if (icat == 3) continue;
        const acc_t ialpha = alphas[ityp], iK = Ks[ityp];
        const acc_t fax0 = B[3 * i], fay0 = B[3 * i + 1], faz0 = B[3 * i + 2];
        acc_t fv[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};
        if (FV) unit_vec(FV + 3 * i, fv);
        const acc_t fatx = R[0] * fax0 + R[1] * fay0 + R[2] * faz0 + tx;
        const acc_t faty = R[3] * fax0 + R[4] * fay0 + R[5] * faz0 + ty;
        const acc_t fatz = R[6] * fax0 + R[7] * fay0 + R[8] * faz0 + tz;
        const acc_t fvtx = R[0] * fv[0] + R[1] * fv[1] + R[2] * fv[2];
        const acc_t fvty = R[3] * fv[0] + R[4] * fv[1] + R[5] * fv[2];
        const acc_t fvtz = R[6] * fv[0] + R[7] * fv[1] + R[8] * fv[2];
        acc_t f[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};   /* positional force sum_j alpha*K*w*E*(ref - rotfit) */
        acc_t wf[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};  /* weight force sum_j coeff * ref_vn */
        acc_t fe[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};  /* force at the extended point (ext != 0) */
        const int use_ext = ext != 0 && (ityp == 0 || ityp == 1);
        for (int j = 0; j < n_real; ++j) {
            if (At[j] != ityp) continue;
            const acc_t dx = fatx - A[3 * j], dy = faty - A[3 * j + 1], dz = fatz - A[3 * j + 2];
            const acc_t r2 = dx * dx + dy * dy + dz * dz;
            const acc_t E = ACC_EXP(-ialpha * ACC(0.5) * r2);
            acc_t rv[3] = {ACC(0.0), ACC(0.0), ACC(0.0)};
            acc_t w = ACC(1.0), c = ACC(0.0);
            if (use_ext) {
                unit_vec(RV + 3 * j, rv);
                w = ext == 1 ? ACC(1.0) : ACC(0.0);
                /* (rotfit + R v_fit) - (ref + v_ref), the sign convention of dx */
                const acc_t ex = dx + fvtx - rv[0], ey = dy + fvty - rv[1], ez = dz + fvtz - rv[2];
                const acc_t Ee = iK * ACC_EXP(-ialpha * ACC(0.5) * (ex * ex + ey * ey + ez * ez));
                Oacc += Ee;
                if (need_grad) {
                    fe[0] += -ialpha * Ee * ex; fe[1] += -ialpha * Ee * ey;
                    fe[2] += -ialpha * Ee * ez;
                }
            } else if (icat == 1 || icat == 2) {
                unit_vec(RV + 3 * j, rv);
                const acc_t D = fvtx * rv[0] + fvty * rv[1] + fvtz * rv[2];
                if (icat == 1) {
                    const acc_t Dcl = D < ACC(0.0) ? ACC(0.0) : (D > ACC(1.0) ? ACC(1.0) : D);
                    w = (Dcl + ACC(2.0)) / ACC(3.0);
                    c = (D > ACC(0.0) && D < ACC(1.0)) ? ACC(1.0) : ACC(0.0);
                } else {
                    w = (ACC_ABS(D) + ACC(2.0)) / ACC(3.0);
                    c = D > ACC(0.0) ? ACC(1.0) : (D < ACC(0.0) ? -ACC(1.0) : ACC(0.0));
                }
            }
            const acc_t KwE = iK * w * E;
            Oacc += KwE;
            if (need_grad) {
                const acc_t aKwE = -ialpha * KwE;
                f[0] += aKwE * dx; f[1] += aKwE * dy; f[2] += aKwE * dz;
                const acc_t coeff = (ACC(1.0) / ACC(3.0)) * iK * E * c;
                wf[0] += coeff * rv[0]; wf[1] += coeff * rv[1]; wf[2] += coeff * rv[2];
            }
        }
        if (need_grad) {
            dT[0] += f[0]; dT[1] += f[1]; dT[2] += f[2];
            quat_tail(f, fax0, fay0, faz0, q, dQ);
            quat_tail(wf, fv[0], fv[1], fv[2], q, dQ);
            if (use_ext) {
                dT[0] += fe[0]; dT[1] += fe[1]; dT[2] += fe[2];
                quat_tail(fe, fax0 + fv[0], fay0 + fv[1], faz0 + fv[2], q, dQ);
            }
        }
    }
    *O = Oacc;
    for (int c = 0; c < 4; ++c) dQ_out[c] = dQ[c];
    for (int c = 0; c < 3; ++c) dT_out[c] = dT[c];
}

/* ------------------------------------------------------------------------- */
/* Public single-evaluation entry points (value + gradient per pose).          */
/* Arrays are padded: A (K,Npad,3), B (K,Mpad,3), charges (K,Npad)/(K,Mpad).   */
/* ------------------------------------------------------------------------- */
typedef struct {
    int Npad, Mpad;
    const float *A, *B, *CA, *CB, *q, *t;
    const int32_t *Nr, *Mr;
    double alpha, inv_lam;
    int need_grad;
    double *V, *dQ, *dT;
} overlap_args;

static void overlap_one(void *ctx, int k) {
    const overlap_args *a = (const overlap_args *)ctx;
    pose_overlap(a->A + (size_t)k * a->Npad * 3, a->B + (size_t)k * a->Mpad * 3,
                 a->CA ? a->CA + (size_t)k * a->Npad : NULL,
                 a->CB ? a->CB + (size_t)k * a->Mpad : NULL, a->q + 4 * (size_t)k,
                 a->t + 3 * (size_t)k, a->Nr[k], a->Mr[k], a->alpha, a->inv_lam,
                 a->need_grad, a->V + k, a->dQ + 4 * (size_t)k, a->dT + 3 * (size_t)k);
}

void fsso_overlap_grad(int K, int Npad, int Mpad, const float *A, const float *B,
                       const float *CA, const float *CB, const float *q, const float *t,
                       const int32_t *Nr, const int32_t *Mr, double alpha, double inv_lam,
                       int need_grad, double *V, double *dQ, double *dT, int nthreads) {
    overlap_args a = {Npad, Mpad, A, B, CA, CB, q, t, Nr, Mr, alpha, inv_lam, need_grad, V, dQ, dT};
    parallel_for(K, nthreads, 4, overlap_one, &a);
}

typedef struct {
    int Npad, Mpad;
    const float *A, *B, *RV, *FV;
    const int32_t *At, *Bt;
    const float *q, *t;
    const int32_t *Nr, *Mr;
    const double *alphas, *Ks;
    const int32_t *cats;
    int ext, need_grad;
    double *O, *dQ, *dT;
} pharm_args;

static void pharm_one(void *ctx, int k) {
    const pharm_args *a = (const pharm_args *)ctx;
    pose_pharm(a->A + (size_t)k * a->Npad * 3, a->B + (size_t)k * a->Mpad * 3,
               a->RV ? a->RV + (size_t)k * a->Npad * 3 : NULL,
               a->FV ? a->FV + (size_t)k * a->Mpad * 3 : NULL, a->At + (size_t)k * a->Npad,
               a->Bt + (size_t)k * a->Mpad, a->q + 4 * (size_t)k, a->t + 3 * (size_t)k,
               a->Nr[k], a->Mr[k], a->alphas, a->Ks, a->cats, a->ext, a->need_grad, a->O + k,
               a->dQ + 4 * (size_t)k, a->dT + 3 * (size_t)k);
}

void fsso_pharm_grad(int K, int Npad, int Mpad, const float *A, const float *B,
                     const float *RV, const float *FV, const int32_t *At, const int32_t *Bt,
                     const float *q, const float *t, const int32_t *Nr, const int32_t *Mr,
                     const double *alphas, const double *Ks, const int32_t *cats,
                     int need_grad, double *O, double *dQ, double *dT, int nthreads, int ext) {
    pharm_args a = {Npad, Mpad, A, B, RV, FV, At, Bt, q, t, Nr, Mr, alphas, Ks, cats,
                    ext, need_grad, O, dQ, dT};
    parallel_for(K, nthreads, 4, pharm_one, &a);
}

/* ------------------------------------------------------------------------- */
/* Tails (cpu_fused.py:54-167).  State is float; arithmetic as numba types it. */
/* ------------------------------------------------------------------------- */
static inline void adam_update(float *q, float *t, const double gq[4], const double gt[3],
                               float *mq, float *vq, float *mt, float *vt, float lr) {
    /* tangent projection dq = g - q (g.q) */
    const double radial = gq[0] * q[0] + gq[1] * q[1] + gq[2] * q[2] + gq[3] * q[3];
    double dq[4];
    for (int c = 0; c < 4; ++c) dq[c] = gq[c] - q[c] * radial;
    for (int c = 0; c < 4; ++c) {
        mq[c] = (float)(B1 * mq[c] + (1.0 - B1) * dq[c]);
        vq[c] = (float)(B2 * vq[c] + (1.0 - B2) * dq[c] * dq[c]);
    }
    for (int c = 0; c < 4; ++c) {
        const float lm = lr * mq[c]; /* float32 * float32 in numba */
        q[c] = (float)(q[c] - lm / sqrt(vq[c] + ADAM_EPS));
    }
    for (int c = 0; c < 3; ++c) {
        mt[c] = (float)(B1 * mt[c] + (1.0 - B1) * gt[c]);
        vt[c] = (float)(B2 * vt[c] + (1.0 - B2) * gt[c] * gt[c]);
    }
    for (int c = 0; c < 3; ++c) {
        const float lm = lr * mt[c];
        t[c] = (float)(t[c] - lm / sqrt(vt[c] + ADAM_EPS));
    }
    float qn = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double qnd = qn < 1e-12f ? 1e-12 : (double)qn;
    for (int c = 0; c < 4; ++c) q[c] = (float)(q[c] / qnd);
}

static inline void track_best(double score, const float *q, const float *t,
                              float *best, float *bq, float *bt) {
    if (score > (double)*best) {
        *best = (float)score;
        memcpy(bq, q, 4 * sizeof(float));
        memcpy(bt, t, 3 * sizeof(float));
    }
}

/* single-channel Tanimoto tail (cpu_fused.py:54-108) */
static void tail_tanimoto(float O, const float dQf[4], const float dTf[3], float norm,
                          float *q, float *t, float *mq, float *vq, float *mt, float *vt,
                          float *best, float *bq, float *bt, float lr) {
    float denom32 = norm - O;
    const double denom = denom32 == 0.0f ? 1e-12 : (double)denom32;
    const double score = O / denom;
    const double scale = norm / (denom * denom);
    track_best(score, q, t, best, bq, bt);
    double gq[4], gt[3];
    for (int c = 0; c < 4; ++c) gq[c] = -scale * dQf[c];
    for (int c = 0; c < 3; ++c) gt[c] = -scale * dTf[c];
    adam_update(q, t, gq, gt, mq, vq, mt, vt, lr);
}

/* Tversky tail (pharm.py:417-426, pharm_overlap.py:36-59): score = min(O/D, 1) (0 when
 * D <= 1e-8), gradient scale active/D with active = O < D. */
static void tail_tversky(float O, const float dQf[4], const float dTf[3], float D,
                         float *q, float *t, float *mq, float *vq, float *mt, float *vt,
                         float *best, float *bq, float *bt, float lr) {
    double score = D > 1e-8f ? (double)O / (double)D : 0.0;
    if (score > 1.0) score = 1.0;
    const double scale = O < D ? 1.0 / (double)D : 0.0;
    track_best(score, q, t, best, bq, bt);
    double gq[4], gt[3];
    for (int c = 0; c < 4; ++c) gq[c] = -scale * dQf[c];
    for (int c = 0; c < 3; ++c) gt[c] = -scale * dTf[c];
    adam_update(q, t, gq, gt, mq, vq, mt, vt, lr);
}

/* two-channel tail: (1-w)*shape Tanimoto + w*pharm Tanimoto (cpu_fused.py:111-167) */
static void tail_combo(float Vs, const float dQs[4], const float dTs[3], float Oc,
                       const float dQc[4], const float dTc[3], float norm_s, float norm_c,
                       float w, float *q, float *t, float *mq, float *vq, float *mt, float *vt,
                       float *best, float *bq, float *bt, float lr) {
    float ds32 = norm_s - Vs;
    const double ds = ds32 == 0.0f ? 1e-12 : (double)ds32;
    const double ss = Vs / ds, scale_s = norm_s / (ds * ds);
    float dc32 = norm_c - Oc;
    const double dc = dc32 == 0.0f ? 1e-12 : (double)dc32;
    const double sc = Oc / dc, scale_c = norm_c / (dc * dc);
    const double wd = (double)w;
    const double score = (1.0 - wd) * ss + wd * sc;
    track_best(score, q, t, best, bq, bt);
    const double cs = -(1.0 - wd) * scale_s, cc = -wd * scale_c;
    double gq[4], gt[3];
    for (int c = 0; c < 4; ++c) gq[c] = cs * dQs[c] + cc * dQc[c];
    for (int c = 0; c < 3; ++c) gt[c] = cs * dTs[c] + cc * dTc[c];
    adam_update(q, t, gq, gt, mq, vq, mt, vt, lr);
}

/* ------------------------------------------------------------------------- */
/* Fine loop (cpu_fused.py:179-217).                                           */
/* ------------------------------------------------------------------------- */
typedef struct {
    int mode;              /* FSSO_SHAPE .. FSSO_COLOR_COMBO */
    int K, Npad, Mpad;     /* shape (or ESP) channel: poses, padded ref/fit points */
    const float *A, *B, *CA, *CB;
    const int32_t *Nr, *Mr;
    int Ppad, Qpad;        /* pharm channel padding (ref, fit) */
    const float *PA, *PB, *PRV, *PFV;
    const int32_t *PAt, *PBt, *PNr, *PMr;
    const double *alphas, *Ks;
    const int32_t *cats;
    double alpha, inv_lam, w;
    const float *norm_s, *norm_c; /* per pose self-overlap sums (Tversky: D per pose) */
    int ext;               /* pharm: extended points 0/1/2 */
    int tversky;           /* pharm: norm_s holds the Tversky denominator D */
} fsso_problem;

/* Evaluate the channels of one pose and apply its tail (one optimisation step). */
static void pose_step(const fsso_problem *P, int k, float *q, float *t, float *mq, float *vq,
                      float *mt, float *vt, float *best, float *bq, float *bt, float lr) {
    double V, dQ[4], dT[3];
    float Vf = 0.0f, dQf[4] = {0, 0, 0, 0}, dTf[3] = {0, 0, 0};
    if (P->mode == FSSO_SHAPE || P->mode == FSSO_ESP || P->mode == FSSO_COMBO ||
        P->mode == FSSO_COLOR_COMBO) {
        pose_overlap(P->A + (size_t)k * P->Npad * 3, P->B + (size_t)k * P->Mpad * 3,
                     P->mode == FSSO_ESP ? P->CA + (size_t)k * P->Npad : NULL,
                     P->mode == FSSO_ESP ? P->CB + (size_t)k * P->Mpad : NULL, q, t,
                     P->Nr[k], P->Mr[k], P->alpha, P->inv_lam, 1, &V, dQ, dT);
        Vf = (float)V;
        for (int c = 0; c < 4; ++c) dQf[c] = (float)dQ[c];
        for (int c = 0; c < 3; ++c) dTf[c] = (float)dT[c];
    }
    if (P->mode == FSSO_SHAPE || P->mode == FSSO_ESP) {
        tail_tanimoto(Vf, dQf, dTf, P->norm_s[k], q, t, mq, vq, mt, vt, best, bq, bt, lr);
        return;
    }
    double O, dQp[4], dTp[3];
    float Of, dQpf[4], dTpf[3];
    pose_pharm(P->PA + (size_t)k * P->Ppad * 3, P->PB + (size_t)k * P->Qpad * 3,
               P->PRV ? P->PRV + (size_t)k * P->Ppad * 3 : NULL,
               P->PFV ? P->PFV + (size_t)k * P->Qpad * 3 : NULL,
               P->PAt + (size_t)k * P->Ppad, P->PBt + (size_t)k * P->Qpad, q, t,
               P->PNr[k], P->PMr[k], P->alphas, P->Ks, P->cats, P->ext, 1, &O, dQp, dTp);
    Of = (float)O;
    for (int c = 0; c < 4; ++c) dQpf[c] = (float)dQp[c];
    for (int c = 0; c < 3; ++c) dTpf[c] = (float)dTp[c];
    if (P->mode == FSSO_PHARM) {
        if (P->tversky)
            tail_tversky(Of, dQpf, dTpf, P->norm_s[k], q, t, mq, vq, mt, vt, best, bq, bt, lr);
        else
            tail_tanimoto(Of, dQpf, dTpf, P->norm_s[k], q, t, mq, vq, mt, vt, best, bq, bt, lr);
        return;
    }
    tail_combo(Vf, dQf, dTf, Of, dQpf, dTpf, P->norm_s[k], P->norm_c[k], (float)P->w, q, t,
               mq, vq, mt, vt, best, bq, bt, lr);
}

typedef struct {
    const fsso_problem *P;
    float *q, *t, *mq, *vq, *mt, *vt, *best, *bq, *bt;
    float lr;
    int nsteps;
} loop_args;

static void pose_all_steps(void *ctx, int k) {
    const loop_args *a = (const loop_args *)ctx;
    for (int s = 0; s < a->nsteps; ++s)
        pose_step(a->P, k, a->q + 4 * (size_t)k, a->t + 3 * (size_t)k, a->mq + 4 * (size_t)k,
                  a->vq + 4 * (size_t)k, a->mt + 3 * (size_t)k, a->vt + 3 * (size_t)k,
                  a->best + k, a->bq + 4 * (size_t)k, a->bt + 3 * (size_t)k, a->lr);
}

/* Runs the fine loop from the seeds (q_io, t_io: in = seed, out = current pose) and
 * writes best score / best pose per pose.  es_patience < 0 disables early stop;
 * es_patience >= 0 follows fine_loop_cpu exactly (0 = stop at the first plateau). */
int fsso_fine_loop(const fsso_problem *P, float *q_io, float *t_io, int steps, float lr,
                   int es_patience, double es_tol, float *best, float *bq, float *bt,
                   int nthreads) {
    const int K = P->K;
    float *mq = calloc((size_t)K * 4, sizeof(float));
    float *vq = calloc((size_t)K * 4, sizeof(float));
    float *mt = calloc((size_t)K * 3, sizeof(float));
    float *vt = calloc((size_t)K * 3, sizeof(float));
    if (!mq || !vq || !mt || !vt) { free(mq); free(vq); free(mt); free(vt); return -1; }
    for (int k = 0; k < K; ++k) {
        best[k] = -INFINITY;
        memcpy(bq + 4 * (size_t)k, q_io + 4 * (size_t)k, 4 * sizeof(float));
        memcpy(bt + 3 * (size_t)k, t_io + 3 * (size_t)k, 3 * sizeof(float));
    }
    int steps_run = steps;
    loop_args la = {P, q_io, t_io, mq, vq, mt, vt, best, bq, bt, lr, steps};
    if (es_patience < 0) {
        parallel_for(K, nthreads, 1, pose_all_steps, &la);
    } else {
        double prev = -INFINITY;
        int no_improve = 0;
        la.nsteps = 1;
        for (int s = 0; s < steps; ++s) {
            parallel_for(K, nthreads, 4, pose_all_steps, &la);
            if (s % 5 == 0) {
                double cur = -INFINITY;
                for (int k = 0; k < K; ++k) if (best[k] > cur) cur = best[k];
                if (cur - prev < es_tol) {
                    if (++no_improve >= es_patience) { steps_run = s + 1; break; }
                } else {
                    no_improve = 0;
                    prev = cur;
                }
            }
        }
    }
    free(mq); free(vq); free(mt); free(vt);
    return steps_run;
}

/* Flat-argument wrapper so ctypes callers need no struct layout. */
int fsso_fine_loop_flat(int mode, int K, int Npad, int Mpad, const float *A, const float *B,
                        const float *CA, const float *CB, const int32_t *Nr, const int32_t *Mr,
                        int Ppad, int Qpad, const float *PA, const float *PB, const float *PRV,
                        const float *PFV, const int32_t *PAt, const int32_t *PBt,
                        const int32_t *PNr, const int32_t *PMr, const double *alphas,
                        const double *Ks, const int32_t *cats, double alpha, double inv_lam,
                        double w, const float *norm_s, const float *norm_c, float *q_io,
                        float *t_io, int steps, float lr, int es_patience, double es_tol,
                        float *best, float *bq, float *bt, int nthreads, int ext, int tversky) {
    fsso_problem P = {mode, K, Npad, Mpad, A, B, CA, CB, Nr, Mr, Ppad, Qpad, PA, PB, PRV, PFV,
                      PAt, PBt, PNr, PMr, alphas, Ks, cats, alpha, inv_lam, w, norm_s, norm_c,
                      ext, tversky};
    return fsso_fine_loop(&P, q_io, t_io, steps, lr, es_patience, es_tol, best, bq, bt, nthreads);
}

int fsso_max_threads(void) {
    const long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* ------------------------------------------------------------------------- */
/* ShaEP ESP comparison and the vol_and_surf_esp fine loop.                   */
/* ------------------------------------------------------------------------- */
/* Sum over field points i of exp(-(pe_i - coulomb * sum_m q_m / max(d_im, 1e-6))^2 * inv_lam),
 * skipping every point within radius_m + probe of some atom (cpu.py:237-261).  P (n,3) field
 * points and A (m,3) atoms are in one frame (double), PE (n) the field points' ESP, Q/R (m)
 * the atoms' charges and radii. */
static double esp_compare(const double *P, const float *PE, int n, const double *A,
                          const float *Q, const float *Rr, int m, double inv_lam,
                          double coulomb, double probe) {
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        double esp = 0.0;
        int blocked = 0;
        for (int j = 0; j < m; ++j) {
            const double dx = P[3 * i] - A[3 * j], dy = P[3 * i + 1] - A[3 * j + 1],
                         dz = P[3 * i + 2] - A[3 * j + 2];
            double d = sqrt(dx * dx + dy * dy + dz * dz);
            if (d < 1e-6) d = 1e-6;
            esp += Q[j] / d;
            if (d < (double)Rr[j] + probe) blocked = 1;
        }
        esp *= coulomb;
        if (!blocked) {
            const double diff = PE[i] - esp;
            total += exp(-(diff * diff) * inv_lam);
        }
    }
    return total;
}

static void to_double(const float *X, int n, double *out) {
    for (int i = 0; i < 3 * n; ++i) out[i] = X[i];
}

static void transform(const float *X, int n, const float *q, const float *t, double *out) {
    acc_t R[9];
    rotmat(q, R);
    for (int i = 0; i < n; ++i) {
        const double x = X[3 * i], y = X[3 * i + 1], z = X[3 * i + 2];
        out[3 * i] = R[0] * x + R[1] * y + R[2] * z + t[0];
        out[3 * i + 1] = R[3] * x + R[4] * y + R[5] * z + t[1];
        out[3 * i + 2] = R[6] * x + R[7] * y + R[8] * z + t[2];
    }
}

/* Batched comparison (esp_comparison_batch): K rows of padded field points / atoms. */
void fsso_esp_compare(int K, int Npad, int Mpad, const float *P, const float *PE,
                      const float *A, const float *Q, const float *Rr, const int32_t *Nr,
                      const int32_t *Mr, double inv_lam, double coulomb, double probe,
                      double *out) {
    double *pd = malloc(sizeof(double) * 3 * (size_t)(Npad > 0 ? Npad : 1));
    double *ad = malloc(sizeof(double) * 3 * (size_t)(Mpad > 0 ? Mpad : 1));
    for (int k = 0; k < K; ++k) {
        to_double(P + (size_t)k * Npad * 3, Nr[k], pd);
        to_double(A + (size_t)k * Mpad * 3, Mr[k], ad);
        out[k] = esp_compare(pd, PE + (size_t)k * Npad, Nr[k], ad, Q + (size_t)k * Mpad,
                             Rr + (size_t)k * Mpad, Mr[k], inv_lam, coulomb, probe);
    }
    free(pd);
    free(ad);
}

typedef struct {
    int K;
    int Cn, Cm; const float *CA, *CB; const int32_t *CNr, *CMr;     /* shape centres */
    int An, Am; const float *AA, *AB, *QA, *QB, *RA, *RB;           /* atoms with H */
    const int32_t *ANr, *AMr;
    int Sn, Sm; const float *SA, *SB, *PEA, *PEB;                   /* surfaces + ESP */
    const int32_t *SNr, *SMr;
    double alpha, inv_lam, coulomb, probe, w;
    int stride, steps;
    const float *norm;                                              /* V_AA + V_BB */
    float *q, *t, *best, *bq, *bt;
    float lr;
} combo_args;

/* One row of the vol_and_surf_esp fine loop: the pose follows the shape gradient scaled by
 * (1 - w); the tracked score w * ESP similarity + (1 - w) * shape Tanimoto is evaluated on
 * steps that are multiples of `stride` and on the last step (esp_combo.py:497-595). */
static void combo_row(void *ctx, int k) {
    const combo_args *a = (const combo_args *)ctx;
    float *q = a->q + 4 * (size_t)k, *t = a->t + 3 * (size_t)k;
    float mq[4] = {0, 0, 0, 0}, vq[4] = {0, 0, 0, 0}, mt[3] = {0, 0, 0}, vt[3] = {0, 0, 0};
    float *best = a->best + k, *bq = a->bq + 4 * (size_t)k, *bt = a->bt + 3 * (size_t)k;
    *best = -INFINITY;
    memcpy(bq, q, 4 * sizeof(float));
    memcpy(bt, t, 3 * sizeof(float));
    const int na = a->ANr[k], ma = a->AMr[k], ns = a->SNr[k], ms = a->SMr[k];
    double *sa = malloc(sizeof(double) * 3 * (size_t)(ns > 0 ? ns : 1));
    double *aa = malloc(sizeof(double) * 3 * (size_t)(na > 0 ? na : 1));
    double *sb = malloc(sizeof(double) * 3 * (size_t)(ms > 0 ? ms : 1));
    double *ab = malloc(sizeof(double) * 3 * (size_t)(ma > 0 ? ma : 1));
    to_double(a->SA + (size_t)k * a->Sn * 3, ns, sa);
    to_double(a->AA + (size_t)k * a->An * 3, na, aa);
    const float U = a->norm[k];
    const float wf = (float)a->w;
    for (int step = 0; step < a->steps; ++step) {
        double V, dQ[4], dT[3];
        pose_overlap(a->CA + (size_t)k * a->Cn * 3, a->CB + (size_t)k * a->Cm * 3, NULL, NULL,
                     q, t, a->CNr[k], a->CMr[k], a->alpha, 0.0, 1, &V, dQ, dT);
        const float Vf = (float)V;
        const float denom = U - Vf;
        const float scale = U / (denom * denom);
        if (step % a->stride == 0 || step == a->steps - 1) {
            transform(a->AB + (size_t)k * a->Am * 3, ma, q, t, ab);
            transform(a->SB + (size_t)k * a->Sm * 3, ms, q, t, sb);
            const double e1 = esp_compare(sa, a->PEA + (size_t)k * a->Sn, ns, ab,
                                          a->QB + (size_t)k * a->Am, a->RB + (size_t)k * a->Am,
                                          ma, a->inv_lam, a->coulomb, a->probe);
            const double e2 = esp_compare(sb, a->PEB + (size_t)k * a->Sm, ms, aa,
                                          a->QA + (size_t)k * a->An, a->RA + (size_t)k * a->An,
                                          na, a->inv_lam, a->coulomb, a->probe);
            const float es = ((float)e1 + (float)e2) / (float)(ns + ms);
            const float vs = Vf / denom;
            const float score = wf * es + (1.0f - wf) * vs;
            track_best(score, q, t, best, bq, bt);
        }
        const float c = -scale * (1.0f - wf);
        double gq[4], gt[3];
        for (int i = 0; i < 4; ++i) gq[i] = c * (float)dQ[i];
        for (int i = 0; i < 3; ++i) gt[i] = c * (float)dT[i];
        adam_update(q, t, gq, gt, mq, vq, mt, vt, a->lr);
    }
    free(sa); free(aa); free(sb); free(ab);
}

void fsso_esp_combo_loop(int K, int Cn, int Cm, const float *CA, const float *CB,
                         const int32_t *CNr, const int32_t *CMr, int An, int Am,
                         const float *AA, const float *AB, const float *QA, const float *QB,
                         const float *RA, const float *RB, const int32_t *ANr,
                         const int32_t *AMr, int Sn, int Sm, const float *SA, const float *SB,
                         const float *PEA, const float *PEB, const int32_t *SNr,
                         const int32_t *SMr, double alpha, double inv_lam, double coulomb,
                         double probe, double w, int stride, const float *norm, float *q_io,
                         float *t_io, int steps, float lr, float *best, float *bq, float *bt,
                         int nthreads) {
    combo_args a = {K, Cn, Cm, CA, CB, CNr, CMr, An, Am, AA, AB, QA, QB, RA, RB, ANr, AMr,
                    Sn, Sm, SA, SB, PEA, PEB, SNr, SMr, alpha, inv_lam, coulomb, probe, w,
                    stride > 0 ? stride : 1, steps, norm, q_io, t_io, best, bq, bt, lr};
    parallel_for(K, nthreads, 1, combo_row, &a);
}
