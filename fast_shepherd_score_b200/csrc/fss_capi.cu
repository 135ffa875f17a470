// fss_capi.cu -- the extern "C" surface of libfss_cuda.so (declared in include/fss_cuda.h).
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "fss_internal.cuh"

namespace fss {

namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_launch(const char* what) {
  const cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) return FSS_OK;
  const int code = ce == cudaErrorMemoryAllocation ? FSS_ERR_NOMEM : FSS_ERR_CUDA;
  return set_error(code, std::string(what) + ": " + cudaGetErrorString(ce));
}

int num_sms() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
  return n > 0 ? n : 1;
}

int align_launch(const fss_align_desc* d, cudaStream_t st);
int pick_best_launch(const float* rs, const float* rq, const float* rt, int P, int S, float* os,
                     float* oq, float* ot, cudaStream_t st);
int self_overlap_launch(const float* pts, const int32_t* off, int n_mol, int max_n, float alpha,
                        int esp, float inv_lam, float* out, cudaStream_t st);
int pharm_self_launch(const float* anc, const float* vec, const int32_t* off, int n_mol, int max_n,
                      int directional, float* out, cudaStream_t st);
int overlap_eval_launch(const float* A, const float* B, const float* CA, const float* CB,
                        const float* q, const float* t, const int32_t* Nr, const int32_t* Mr,
                        int K, int Npad, int Mpad, float alpha, float inv_lam, int need_grad,
                        float* V, float* dQ, float* dT, cudaStream_t st);
int pharm_eval_launch(const float* A, const float* B, const float* RV, const float* FV,
                      const int32_t* At, const int32_t* Bt, const float* q, const float* t,
                      const int32_t* Nr, const int32_t* Mr, int K, int Npad, int Mpad,
                      int directional, int need_grad, float* O, float* dQ, float* dT,
                      cudaStream_t st);
int tanimoto_adam_launch(const float* V, const float* dQ, const float* dT, const float* U,
                         float* q, float* t, float* mq, float* vq, float* mt, float* vt,
                         float* best, float* bq, float* bt, int K, float lr, cudaStream_t st);
int seeds_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                 const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                 int P, int S, const float* fibo, int n_fibo, int fit_f16, float* sq, float* st,
                 cudaStream_t stream);
int score_fwd_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                     const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                     int P, int maxN, int maxM, float alpha, int esp, float inv_lam, float* score,
                     float* overlaps, cudaStream_t st);
int score_bwd_launch(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                     const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                     int P, int maxN, int maxM, float alpha, int esp, float inv_lam,
                     const float* overlaps, const float* grad_score, float* grad_ref,
                     float* grad_fit, cudaStream_t st);
int score_fwd_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                           const float* fit_xyz, const float* fit_q, int fit_n,
                           const int32_t* pair_ref, const int32_t* pair_fit, int P, float alpha,
                           int esp, float inv_lam, float* score, float* overlaps,
                           cudaStream_t st);
int score_bwd_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                           const float* fit_xyz, const float* fit_q, int fit_n,
                           const int32_t* pair_ref, const int32_t* pair_fit, int P, float alpha,
                           int esp, float inv_lam, const float* overlaps, const float* grad_score,
                           float* grad_ref_xyz, float* grad_ref_q, float* grad_fit_xyz,
                           float* grad_fit_q, cudaStream_t st);

int score_fwd_mom_dense_launch(const float* ref_xyz, const float* ref_q, int ref_n,
                               const float* fit_xyz, const float* fit_q, int fit_n,
                               const int32_t* pair_ref, const int32_t* pair_fit, int P,
                               float alpha, int esp, float inv_lam, float* score, float* overlaps,
                               float* ref_mom, float* fit_mom, cudaStream_t st);
int score_bwd_mom_dense_launch(const int32_t* pair_ref, const int32_t* pair_fit, int P,
                               int ref_n, int fit_n, float alpha, int esp, float inv_lam,
                               const float* overlaps, const float* grad_score,
                               const float* ref_mom, const float* fit_mom, float* grad_ref_xyz,
                               float* grad_ref_q, float* grad_fit_xyz, float* grad_fit_q,
                               int overwrite, cudaStream_t st);

int probe_launch(int which, int iters, int blocks_per_sm, float* out, long long* ops,
                 cudaStream_t st);
int align_static_launch(const fss_align_desc* d, cudaStream_t st);

}  // namespace fss

#define FSS_GUARD(expr)                                                   \
  try {                                                                   \
    return (expr);                                                        \
  } catch (const std::exception& ex) {                                    \
    return fss::set_error(FSS_ERR_CUDA, std::string("host exception: ") + ex.what()); \
  } catch (...) {                                                         \
    return fss::set_error(FSS_ERR_CUDA, "unknown host exception");       \
  }

static inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

int fss_abi_version(void) { return FSS_ABI_VERSION; }

const char* fss_last_error(void) { return fss::g_last_error.c_str(); }

int fss_max_points(void) { return fss::kMaxPoints; }

int fss_overlap_grad(const float* A, const float* B, const float* CA, const float* CB,
                     const float* q, const float* t, const int32_t* N_real,
                     const int32_t* M_real, int32_t K, int32_t N_pad, int32_t M_pad,
                     float alpha, float inv_lam, int32_t need_grad, float* V, float* dQ,
                     float* dT, void* stream) {
  FSS_GUARD(fss::overlap_eval_launch(A, B, CA, CB, q, t, N_real, M_real, K, N_pad, M_pad, alpha,
                                     inv_lam, need_grad, V, dQ, dT, S(stream)));
}

int fss_pharm_grad(const float* A, const float* B, const float* RV, const float* FV,
                   const int32_t* At, const int32_t* Bt, const float* q, const float* t,
                   const int32_t* N_real, const int32_t* M_real, int32_t K, int32_t N_pad,
                   int32_t M_pad, int32_t directional, int32_t need_grad, float* O, float* dQ,
                   float* dT, void* stream) {
  FSS_GUARD(fss::pharm_eval_launch(A, B, RV, FV, At, Bt, q, t, N_real, M_real, K, N_pad, M_pad,
                                   directional, need_grad, O, dQ, dT, S(stream)));
}

int fss_tanimoto_adam_step(const float* V, const float* dQ, const float* dT, const float* U,
                           float* q, float* t, float* mq, float* vq, float* mt, float* vt,
                           float* best, float* bq, float* bt, int32_t K, float lr,
                           void* stream) {
  FSS_GUARD(fss::tanimoto_adam_launch(V, dQ, dT, U, q, t, mq, vq, mt, vt, best, bq, bt, K, lr,
                                      S(stream)));
}

int fss_self_overlap(const float* pts, const int32_t* off, int32_t n_mol, int32_t max_points,
                     float alpha, int32_t esp, float inv_lam, int32_t pts_f16, float* out,
                     void* stream) {
  if (pts_f16 != 0 && pts_f16 != 1)
    return fss::set_error(FSS_ERR_INVALID, "fss_self_overlap: pts_f16 must be 0 or 1");
  FSS_GUARD(fss::self_overlap_launch(pts, off, n_mol, max_points, alpha, esp, inv_lam, pts_f16,
                                     out, S(stream)));
}

int fss_pharm_self_overlap(const float* anc, const float* vec, const int32_t* off,
                           int32_t n_mol, int32_t max_features, int32_t directional,
                           int32_t extended, int32_t pts_f16, float* out, void* stream) {
  if (pts_f16 != 0 && pts_f16 != 1)
    return fss::set_error(FSS_ERR_INVALID, "fss_pharm_self_overlap: pts_f16 must be 0 or 1");
  FSS_GUARD(fss::pharm_self_launch(anc, vec, off, n_mol, max_features, directional, extended,
                                   pts_f16, out, S(stream)));
}

int fss_seeds(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
              const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
              int32_t n_pairs, int32_t n_seeds, const float* fibo_q, int32_t n_fibo,
              int32_t fit_f16, float* seed_q, float* seed_t, void* stream) {
  if (fit_f16 != 0 && fit_f16 != 1)
    return fss::set_error(FSS_ERR_INVALID, "fss_seeds: fit_f16 must be 0 or 1");
  FSS_GUARD(fss::seeds_launch(ref_pts, ref_off, fit_pts, fit_off, pair_ref, pair_fit, n_pairs,
                              n_seeds, fibo_q, n_fibo, fit_f16, seed_q, seed_t, S(stream)));
}

int fss_align(const fss_align_desc* desc, void* stream) {
  FSS_GUARD(fss::align_launch(desc, S(stream)));
}

int fss_align_static(const fss_align_desc* desc, void* stream) {
  FSS_GUARD(fss::align_static_launch(desc, S(stream)));
}

int fss_pick_best(const float* row_score, const float* row_q, const float* row_t,
                  int32_t n_pairs, int32_t n_starts, float* out_score, float* out_q,
                  float* out_t, void* stream) {
  FSS_GUARD(fss::pick_best_launch(row_score, row_q, row_t, n_pairs, n_starts, out_score, out_q,
                                  out_t, S(stream)));
}

int fss_score_fwd(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                  const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                  int32_t n_pairs, int32_t max_ref_points, int32_t max_fit_points, float alpha,
                  int32_t esp, float inv_lam, float* score, float* overlaps, void* stream) {
  FSS_GUARD(fss::score_fwd_launch(ref_pts, ref_off, fit_pts, fit_off, pair_ref, pair_fit,
                                  n_pairs, max_ref_points, max_fit_points, alpha, esp, inv_lam,
                                  score, overlaps, S(stream)));
}

int fss_score_bwd(const float* ref_pts, const int32_t* ref_off, const float* fit_pts,
                  const int32_t* fit_off, const int32_t* pair_ref, const int32_t* pair_fit,
                  int32_t n_pairs, int32_t max_ref_points, int32_t max_fit_points, float alpha,
                  int32_t esp, float inv_lam, const float* overlaps, const float* grad_score,
                  float* grad_ref, float* grad_fit, void* stream) {
  FSS_GUARD(fss::score_bwd_launch(ref_pts, ref_off, fit_pts, fit_off, pair_ref, pair_fit,
                                  n_pairs, max_ref_points, max_fit_points, alpha, esp, inv_lam,
                                  overlaps, grad_score, grad_ref, grad_fit, S(stream)));
}

int fss_score_fwd_dense(const float* ref_xyz, const float* ref_q, int32_t ref_points,
                        const float* fit_xyz, const float* fit_q, int32_t fit_points,
                        const int32_t* pair_ref, const int32_t* pair_fit, int32_t n_pairs,
                        float alpha, int32_t esp, float inv_lam, float* score, float* overlaps,
                        void* stream) {
  FSS_GUARD(fss::score_fwd_dense_launch(ref_xyz, ref_q, ref_points, fit_xyz, fit_q, fit_points,
                                        pair_ref, pair_fit, n_pairs, alpha, esp, inv_lam, score,
                                        overlaps, S(stream)));
}

int fss_score_bwd_dense(const float* ref_xyz, const float* ref_q, int32_t ref_points,
                        const float* fit_xyz, const float* fit_q, int32_t fit_points,
                        const int32_t* pair_ref, const int32_t* pair_fit, int32_t n_pairs,
                        float alpha, int32_t esp, float inv_lam, const float* overlaps,
                        const float* grad_score, float* grad_ref_xyz, float* grad_ref_q,
                        float* grad_fit_xyz, float* grad_fit_q, void* stream) {
  FSS_GUARD(fss::score_bwd_dense_launch(ref_xyz, ref_q, ref_points, fit_xyz, fit_q, fit_points,
                                        pair_ref, pair_fit, n_pairs, alpha, esp, inv_lam,
                                        overlaps, grad_score, grad_ref_xyz, grad_ref_q,
                                        grad_fit_xyz, grad_fit_q, S(stream)));
}

int fss_score_fwd_moments_dense(const float* ref_xyz, const float* ref_q, int32_t ref_points,
                                const float* fit_xyz, const float* fit_q, int32_t fit_points,
                                const int32_t* pair_ref, const int32_t* pair_fit,
                                int32_t n_pairs, float alpha, int32_t esp, float inv_lam,
                                float* score, float* overlaps, float* ref_moments,
                                float* fit_moments, void* stream) {
  FSS_GUARD(fss::score_fwd_mom_dense_launch(ref_xyz, ref_q, ref_points, fit_xyz, fit_q,
                                            fit_points, pair_ref, pair_fit, n_pairs, alpha, esp,
                                            inv_lam, score, overlaps, ref_moments, fit_moments,
                                            S(stream)));
}

int fss_score_bwd_moments_dense(const int32_t* pair_ref, const int32_t* pair_fit,
                                int32_t n_pairs, int32_t ref_points, int32_t fit_points,
                                float alpha, int32_t esp, float inv_lam, const float* overlaps,
                                const float* grad_score, const float* ref_moments,
                                const float* fit_moments, float* grad_ref_xyz,
                                float* grad_ref_q, float* grad_fit_xyz, float* grad_fit_q,
                                int32_t overwrite, void* stream) {
  FSS_GUARD(fss::score_bwd_mom_dense_launch(pair_ref, pair_fit, n_pairs, ref_points, fit_points,
                                            alpha, esp, inv_lam, overlaps, grad_score,
                                            ref_moments, fit_moments, grad_ref_xyz, grad_ref_q,
                                            grad_fit_xyz, grad_fit_q, overwrite, S(stream)));
}

int fss_probe_peak(int32_t which, int32_t iters, int32_t blocks_per_sm, float* out,
                   long long* ops, void* stream) {
  FSS_GUARD(fss::probe_launch(which, iters, blocks_per_sm, out, ops, S(stream)));
}

}  // extern "C"
