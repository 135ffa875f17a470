"""Oracle drivers: the reference's batched alignment restated on CPU (test infrastructure only).

Each ``align_*`` function follows one reference driver on its CPU (numba, fused) branch:

* :func:`align_shape` -- ``coarse_fine_align_many`` (shepherd_score/accel/drivers/shape.py:155-313)
  through ``cpu_fused_shape`` (accel/kernels/cpu_fused.py:225)
* :func:`align_esp`   -- ``coarse_fine_esp_align_many`` (accel/drivers/esp.py:139-367) through
  ``cpu_fused_esp`` (cpu_fused.py:251)
* :func:`align_pharm` -- ``coarse_fine_pharm_align_many`` (accel/drivers/pharm.py:123-517) through
  ``cpu_fused_pharm`` (cpu_fused.py:278), including the anchor centring (pharm.py:205-225)
  and the translation fold-back (pharm.py:509-517)
* :func:`align_combo` -- shape + directional pharmacophore with one shared pose, composed from
  ``cpu._overlap_grad_kernel`` + ``cpu._pharm_grad_dq_kernel`` and the two-channel tail
  ``cpu_fused._tail_vol_color`` (cpu_fused.py:112); with ``directional=False`` it is
  ``coarse_fine_vol_color_align_many`` (accel/drivers/vol_color.py:199) on its CPU branch.

Early stop: ``es_patience=None`` disables it (the alignment configs run fixed steps);
an integer follows ``fine_loop_cpu``'s batch-global schedule (cpu_fused.py:208-215).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .seeds import batched_seeds, quat_to_rotmat

P_TYPES = ('Acceptor', 'Donor', 'Aromatic', 'Hydrophobe', 'Halogen', 'Cation', 'Anion',
           'ZnBinder', 'Dummy')
_P_ALPHAS = {'acceptor': 1.0, 'donor': 1.0, 'aromatic': 0.7, 'hydrophobe': 0.7, 'cation': 1.0,
             'anion': 1.0, 'znbinder': 1.0, 'halogen': 1.0, 'dummy': 1.0}
_NONDIR = {'hydrophobe', 'znbinder', 'anion', 'cation'}
_DIR = {'acceptor', 'donor', 'halogen'}
_AROM = {'aromatic'}
DUMMY_TYPE = P_TYPES.index('Dummy')
LAM_SCALING = (1e4 / (4 * 55.263 * np.pi)) ** 2


def lookup_tables(directionless: bool = False):
    """(alphas, Ks, cats) per pharmacophore type (analytical_gradients/_torch.py:177-220).

    The reference builds these as float32 tensors and the numba path widens them to float64
    (cpu_fused.py:285-286), so the float32 rounding is kept here.
    """
    al, ks, cats = [], [], []
    for p in P_TYPES:
        pl = p.lower()
        a = _P_ALPHAS.get(pl, 1.0)
        al.append(a)
        ks.append((math.pi / (2.0 * a)) ** 1.5)
        if pl == 'dummy':
            cats.append(3)
        elif directionless or pl in _NONDIR:
            cats.append(0)
        elif pl in _DIR:
            cats.append(1)
        elif pl in _AROM:
            cats.append(2)
        else:
            cats.append(3)
    return (np.asarray(al, np.float32).astype(np.float64),
            np.asarray(ks, np.float32).astype(np.float64),
            np.asarray(cats, np.int32))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _threads(n):
    return _lib.max_threads() if n is None else int(n)


def overlap_grad(A, B, q, t, N_real=None, M_real=None, *, alpha=0.81, CA=None, CB=None,
                 lam=None, need_grad=True, nthreads=None):
    """Shape (or ESP when CA/CB given) overlap and dV/dq, dV/dt per pose, float64.

    cpu.py:38-109 (shape) and cpu.py:158-225 (ESP; ``lam`` is the kernel's lambda).
    """
    A, B, q, t = _f32(A), _f32(B), _f32(q), _f32(t)
    K, Npad, _ = A.shape
    Mpad = B.shape[1]
    Nr = _i32(np.full(K, Npad) if N_real is None else N_real)
    Mr = _i32(np.full(K, Mpad) if M_real is None else M_real)
    CA, CB = _f32(CA), _f32(CB)
    V = np.zeros(K, np.float64)
    dQ = np.zeros((K, 4), np.float64)
    dT = np.zeros((K, 3), np.float64)
    inv_lam = 0.0 if CA is None else 1.0 / float(lam)
    P = _lib.ptr
    _lib.lib().fsso_overlap_grad(K, Npad, Mpad, P(A), P(B), P(CA), P(CB), P(q), P(t), P(Nr),
                                 P(Mr), float(alpha), inv_lam, int(bool(need_grad)), P(V),
                                 P(dQ), P(dT), _threads(nthreads))
    return V, dQ, dT


def pharm_grad(A, B, RV, FV, At, Bt, q, t, N_real=None, M_real=None, *, directionless=False,
               need_grad=True, nthreads=None, ext=0):
    """Typed pharmacophore overlap and dO/dq, dO/dt per pose, float64 (cpu.py:412-612);
    ``ext`` 1/2 adds the extended points of analytical_gradients/_torch.py:288-355."""
    A, B, q, t = _f32(A), _f32(B), _f32(q), _f32(t)
    RV, FV = _f32(RV), _f32(FV)
    At, Bt = _i32(At), _i32(Bt)
    K, Npad, _ = A.shape
    Mpad = B.shape[1]
    Nr = _i32(np.full(K, Npad) if N_real is None else N_real)
    Mr = _i32(np.full(K, Mpad) if M_real is None else M_real)
    al, ks, cats = lookup_tables(directionless)
    O = np.zeros(K, np.float64)
    dQ = np.zeros((K, 4), np.float64)
    dT = np.zeros((K, 3), np.float64)
    P = _lib.ptr
    _lib.lib().fsso_pharm_grad(K, Npad, Mpad, P(A), P(B), P(RV), P(FV), P(At), P(Bt), P(q),
                               P(t), P(Nr), P(Mr), P(al), P(ks), P(cats),
                               int(bool(need_grad)), P(O), P(dQ), P(dT), _threads(nthreads),
                               int(ext))
    return O, dQ, dT


def _identity_pose(K):
    q = np.zeros((K, 4), np.float32)
    q[:, 0] = 1.0
    return q, np.zeros((K, 3), np.float32)


def self_overlap(X, N_real, *, alpha=0.81, C=None, lam=None, nthreads=None):
    """V_XX at the identity pose, float32 as the reference returns it (cpu.py:140-148, :615-624)."""
    q, t = _identity_pose(X.shape[0])
    V, _, _ = overlap_grad(X, X, q, t, N_real, N_real, alpha=alpha, CA=C, CB=C, lam=lam,
                           need_grad=False, nthreads=nthreads)
    return V.astype(np.float32)


def pharm_self_overlap(X, V, T, N_real, *, directionless=False, nthreads=None, ext=0):
    """Pharmacophore self-overlap via the dq kernel at identity (pharm.py:336-346)."""
    q, t = _identity_pose(X.shape[0])
    O, _, _ = pharm_grad(X, X, V, V, T, T, q, t, N_real, N_real, directionless=directionless,
                         need_grad=False, nthreads=nthreads, ext=ext)
    return O.astype(np.float32)


def fine_loop(mode, q_seed, t_seed, norm_s, *, steps, lr, es_patience=None, es_tol=1e-5,
              A=None, B=None, CA=None, CB=None, Nr=None, Mr=None, alpha=0.81, lam=None,
              PA=None, PB=None, PRV=None, PFV=None, PAt=None, PBt=None, PNr=None, PMr=None,
              directionless=False, norm_c=None, w=0.5, nthreads=None, ext=0, tversky=False):
    """Run the fused fine loop over K pose rows (cpu_fused.py:179-217).

    All per-row arrays are already expanded to K = pairs x starts rows.  Returns
    (best score (K,), best q (K,4), best t (K,3), final q, final t, steps run).
    """
    q = np.array(q_seed, np.float32, copy=True, order='C')
    t = np.array(t_seed, np.float32, copy=True, order='C')
    K = q.shape[0]
    best = np.empty(K, np.float32)
    bq = np.empty((K, 4), np.float32)
    bt = np.empty((K, 3), np.float32)
    A, B, CA, CB = _f32(A), _f32(B), _f32(CA), _f32(CB)
    PA, PB, PRV, PFV = _f32(PA), _f32(PB), _f32(PRV), _f32(PFV)
    Nr, Mr, PAt, PBt, PNr, PMr = _i32(Nr), _i32(Mr), _i32(PAt), _i32(PBt), _i32(PNr), _i32(PMr)
    norm_s = _f32(norm_s)
    norm_c = _f32(norm_c)
    Npad = A.shape[1] if A is not None else 0
    Mpad = B.shape[1] if B is not None else 0
    Ppad = PA.shape[1] if PA is not None else 0
    Qpad = PB.shape[1] if PB is not None else 0
    al, ks, cats = lookup_tables(directionless)
    inv_lam = 0.0 if lam is None else 1.0 / float(lam)
    P = _lib.ptr
    n = _lib.lib().fsso_fine_loop_flat(
        int(mode), K, Npad, Mpad, P(A), P(B), P(CA), P(CB), P(Nr), P(Mr), Ppad, Qpad, P(PA),
        P(PB), P(PRV), P(PFV), P(PAt), P(PBt), P(PNr), P(PMr), P(al), P(ks), P(cats),
        float(alpha), inv_lam, float(w), P(norm_s), P(norm_c), P(q), P(t), int(steps),
        float(np.float32(lr)), -1 if es_patience is None else int(es_patience), float(es_tol),
        P(best), P(bq), P(bt), _threads(nthreads), int(ext), int(bool(tversky)))
    if n < 0:
        raise MemoryError("oracle fine loop could not allocate its Adam state")
    return best, bq, bt, q, t, n


def _rep(x, S):
    return np.repeat(np.asarray(x), S, axis=0)


def _pick(best, bq, bt, nb, S):
    """Per-pair argmax over starts (shape.py:306-313)."""
    sc = best.reshape(nb, S)
    i = sc.argmax(1)
    ar = np.arange(nb)
    return sc[ar, i], bq.reshape(nb, S, 4)[ar, i], bt.reshape(nb, S, 3)[ar, i]


def align_shape(A, B, N_real, M_real, *, alpha=0.81, num_seeds=50, steps=100, lr=0.075,
                seeds=None, es_patience=None, es_tol=1e-5, nthreads=None, return_rows=False):
    """Batched shape alignment (vol / surf): shape.py:155-313 on its CPU fused branch."""
    A, B = _f32(A), _f32(B)
    nb = A.shape[0]
    if seeds is None:
        seeds = batched_seeds(A, B, N_real, M_real, num_seeds)
    qs, ts = seeds
    S = qs.shape[1]
    norm = (self_overlap(A, N_real, alpha=alpha, nthreads=nthreads)
            + self_overlap(B, M_real, alpha=alpha, nthreads=nthreads)).astype(np.float32)
    best, bq, bt, _, _, n = fine_loop(
        0, qs.reshape(-1, 4), ts.reshape(-1, 3), _rep(norm, S), steps=steps, lr=lr,
        es_patience=es_patience, es_tol=es_tol, A=_rep(A, S), B=_rep(B, S),
        Nr=_rep(N_real, S), Mr=_rep(M_real, S), alpha=alpha, nthreads=nthreads)
    out = _pick(best, bq, bt, nb, S)
    return (out + ((best, bq, bt),)) if return_rows else out


def align_esp(A, B, CA, CB, N_real, M_real, *, alpha=0.81, lam=0.3, num_seeds=50, steps=100,
              lr=0.075, seeds=None, es_patience=None, es_tol=1e-5, nthreads=None,
              return_rows=False):
    """Batched ESP alignment (surf_esp / vol_esp): esp.py:139-367 on its CPU fused branch.

    ``lam`` is the kernel lambda (surf_esp callers pass LAM_SCALING * lam, aligners.py:383).
    """
    A, B = _f32(A), _f32(B)
    nb = A.shape[0]
    if seeds is None:
        seeds = batched_seeds(A, B, N_real, M_real, num_seeds)
    qs, ts = seeds
    S = qs.shape[1]
    norm = (self_overlap(A, N_real, alpha=alpha, C=CA, lam=lam, nthreads=nthreads)
            + self_overlap(B, M_real, alpha=alpha, C=CB, lam=lam, nthreads=nthreads)
            ).astype(np.float32)
    best, bq, bt, _, _, n = fine_loop(
        1, qs.reshape(-1, 4), ts.reshape(-1, 3), _rep(norm, S), steps=steps, lr=lr,
        es_patience=es_patience, es_tol=es_tol, A=_rep(A, S), B=_rep(B, S), CA=_rep(CA, S),
        CB=_rep(CB, S), Nr=_rep(N_real, S), Mr=_rep(M_real, S), alpha=alpha, lam=lam,
        nthreads=nthreads)
    out = _pick(best, bq, bt, nb, S)
    return (out + ((best, bq, bt),)) if return_rows else out


def center_anchors(X, N_real):
    """Centroid over real points and the centred cloud (pharm.py:205-225)."""
    X = _f32(X)
    npad = X.shape[1]
    mask = (np.arange(npad)[None] < np.asarray(N_real)[:, None]).astype(np.float32)
    c = (X * mask[..., None]).sum(1, dtype=np.float32) / np.maximum(
        np.asarray(N_real, np.float32), 1)[:, None]
    return c.astype(np.float32), (X - c[:, None, :]).astype(np.float32)


TVERSKY_SIGMA = {"tversky": 0.95, "tversky_ref": 1.0, "tversky_fit": 0.05}  # pharm.py:40


def align_pharm(A, B, RV, FV, At, Bt, N_real, M_real, *, num_seeds=50, steps=100, lr=0.075,
                seeds=None, es_patience=None, es_tol=1e-5, nthreads=None, return_rows=False,
                similarity="tanimoto", extended_points=False, only_extended=False):
    """Batched directional pharmacophore alignment: pharm.py:123-517, CPU fused branch for
    Tanimoto without extended points, and the same step arithmetic for the eager branch the
    reference takes otherwise (Tversky tail pharm.py:417-426; extended points via
    compute_overlap_and_grad_pharm, self overlaps with the same flags pharm.py:732-748).

    Anchors are centred per cloud before seeding and the optimum translation is folded back
    into the original frame at the end.  ``seeds`` (if given) are for the centred clouds.
    """
    ext = 0 if not extended_points else (2 if only_extended else 1)
    nb = np.asarray(A).shape[0]
    c_ref, A_c = center_anchors(A, N_real)
    c_fit, B_c = center_anchors(B, M_real)
    if seeds is None:
        seeds = batched_seeds(A_c, B_c, N_real, M_real, num_seeds)
    qs, ts = seeds
    S = qs.shape[1]
    VAA = pharm_self_overlap(A_c, RV, At, N_real, nthreads=nthreads, ext=ext)
    VBB = pharm_self_overlap(B_c, FV, Bt, M_real, nthreads=nthreads, ext=ext)
    if similarity == "tanimoto":
        norm = (VAA + VBB).astype(np.float32)
    else:
        sg = np.float32(TVERSKY_SIGMA[similarity])
        norm = (sg * VAA + (np.float32(1) - sg) * VBB).astype(np.float32)
    best, bq, bt, _, _, n = fine_loop(
        2, qs.reshape(-1, 4), ts.reshape(-1, 3), _rep(norm, S), steps=steps, lr=lr,
        es_patience=es_patience, es_tol=es_tol, PA=_rep(A_c, S), PB=_rep(B_c, S),
        PRV=_rep(_f32(RV), S), PFV=_rep(_f32(FV), S), PAt=_rep(At, S), PBt=_rep(Bt, S),
        PNr=_rep(N_real, S), PMr=_rep(M_real, S), nthreads=nthreads, ext=ext,
        tversky=similarity != "tanimoto")
    sc, q, t = _pick(best, bq, bt, nb, S)
    R = quat_to_rotmat(q.astype(np.float32))
    t = (t - np.einsum('bij,bj->bi', R, c_fit) + c_ref).astype(np.float32)
    out = (sc, q, t)
    return (out + ((best, bq, bt),)) if return_rows else out


def align_combo(A, B, N_real, M_real, PA, PB, PRV, PFV, PAt, PBt, PN_real, PM_real, *,
                alpha=0.81, w=0.5, directional=True, num_seeds=50, steps=100, lr=0.075,
                seeds=None, es_patience=None, es_tol=1e-5, nthreads=None, return_rows=False):
    """Shape + pharmacophore alignment with one shared pose and the two-channel tail.

    Seeds come from the atom clouds (vol_color.py:248).  ``directional=False`` reproduces the
    reference vol_color mode (directionless colour channel).
    """
    A, B = _f32(A), _f32(B)
    nb = A.shape[0]
    if seeds is None:
        seeds = batched_seeds(A, B, N_real, M_real, num_seeds)
    qs, ts = seeds
    S = qs.shape[1]
    norm_s = (self_overlap(A, N_real, alpha=alpha, nthreads=nthreads)
              + self_overlap(B, M_real, alpha=alpha, nthreads=nthreads)).astype(np.float32)
    dl = not directional
    norm_c = (pharm_self_overlap(PA, PRV, PAt, PN_real, directionless=dl, nthreads=nthreads)
              + pharm_self_overlap(PB, PFV, PBt, PM_real, directionless=dl, nthreads=nthreads)
              ).astype(np.float32)
    best, bq, bt, _, _, n = fine_loop(
        3 if directional else 4, qs.reshape(-1, 4), ts.reshape(-1, 3), _rep(norm_s, S),
        steps=steps, lr=lr, es_patience=es_patience, es_tol=es_tol, A=_rep(A, S), B=_rep(B, S),
        Nr=_rep(N_real, S), Mr=_rep(M_real, S), alpha=alpha, PA=_rep(_f32(PA), S),
        PB=_rep(_f32(PB), S), PRV=None if PRV is None else _rep(_f32(PRV), S),
        PFV=None if PFV is None else _rep(_f32(PFV), S), PAt=_rep(PAt, S), PBt=_rep(PBt, S),
        PNr=_rep(PN_real, S), PMr=_rep(PM_real, S), directionless=dl, norm_c=_rep(norm_c, S),
        w=w, nthreads=nthreads)
    out = _pick(best, bq, bt, nb, S)
    return (out + ((best, bq, bt),)) if return_rows else out


# --------------------------------------------------------------------------------------------
# vol_and_surf_esp (ShaEP ESP comparison + volumetric shape), accel/drivers/esp_combo.py
# --------------------------------------------------------------------------------------------
COULOMB_SCALING = 1e4 / (4 * 55.263 * np.pi)     # score/constants.py:16
LAM_SCALING = COULOMB_SCALING ** 2               # score/constants.py:17


def esp_compare(P, PE, A, Q, R, N_real, M_real, *, lam=0.001, probe_radius=1.0):
    """esp_comparison_batch (cpu.py:264-285): per row, the masked Gaussian-of-ESP-difference
    sum over the field points P (K,N,3) with ESP PE (K,N) against atoms A (K,M,3) with charges
    Q and radii R (K,M), all in one frame."""
    P, PE, A, Q, R = _f32(P), _f32(PE), _f32(A), _f32(Q), _f32(R)
    K, Npad, _ = P.shape
    Mpad = A.shape[1]
    out = np.zeros(K, np.float64)
    L = _lib.ptr
    _lib.lib().fsso_esp_compare(K, Npad, Mpad, L(P), L(PE), L(A), L(Q), L(R),
                                L(_i32(N_real)), L(_i32(M_real)),
                                1.0 / (LAM_SCALING * float(lam)), float(COULOMB_SCALING),
                                float(probe_radius), L(out))
    return out


def align_esp_combo(C1, C2, CN, CM, A1, A2, Q1, Q2, R1, R2, AN, AM, S1, S2, PE1, PE2, SN, SM,
                    *, alpha=0.81, lam=0.001, probe_radius=1.0, esp_weight=0.5, num_seeds=8,
                    steps=60, lr=0.1, stride=5, seeds=None, nthreads=None, return_rows=False):
    """coarse_fine_esp_combo_align_many (esp_combo.py:334-595) without the coarse grid: seeds
    on the shape centres, the shape gradient scaled by (1 - esp_weight) steers the pose, and the
    combo score is tracked every `stride` steps and on the last one (the reference's eager loop
    uses 5; its CUDA-graph loop scores every step, i.e. 1)."""
    nb = np.asarray(C1).shape[0]
    if seeds is None:
        seeds = batched_seeds(C1, C2, CN, CM, num_seeds)
    qs, ts = seeds
    S = qs.shape[1]
    norm = (self_overlap(C1, CN, alpha=alpha, nthreads=nthreads)
            + self_overlap(C2, CM, alpha=alpha, nthreads=nthreads)).astype(np.float32)
    rep = lambda x, f=_f32: f(_rep(x, S))
    q = np.array(qs.reshape(-1, 4), np.float32, copy=True, order="C")
    t = np.array(ts.reshape(-1, 3), np.float32, copy=True, order="C")
    K = q.shape[0]
    best = np.empty(K, np.float32)
    bq = np.empty((K, 4), np.float32)
    bt = np.empty((K, 3), np.float32)
    arrs = dict(C1=rep(C1), C2=rep(C2), CN=rep(CN, _i32), CM=rep(CM, _i32), A1=rep(A1),
                A2=rep(A2), Q1=rep(Q1), Q2=rep(Q2), R1=rep(R1), R2=rep(R2), AN=rep(AN, _i32),
                AM=rep(AM, _i32), S1=rep(S1), S2=rep(S2), PE1=rep(PE1), PE2=rep(PE2),
                SN=rep(SN, _i32), SM=rep(SM, _i32), norm=_rep(norm, S).astype(np.float32))
    a = arrs
    L = _lib.ptr
    _lib.lib().fsso_esp_combo_loop(
        K, a["C1"].shape[1], a["C2"].shape[1], L(a["C1"]), L(a["C2"]), L(a["CN"]), L(a["CM"]),
        a["A1"].shape[1], a["A2"].shape[1], L(a["A1"]), L(a["A2"]), L(a["Q1"]), L(a["Q2"]),
        L(a["R1"]), L(a["R2"]), L(a["AN"]), L(a["AM"]), a["S1"].shape[1], a["S2"].shape[1],
        L(a["S1"]), L(a["S2"]), L(a["PE1"]), L(a["PE2"]), L(a["SN"]), L(a["SM"]),
        float(alpha), 1.0 / (LAM_SCALING * float(lam)), float(COULOMB_SCALING),
        float(probe_radius), float(esp_weight), int(stride), L(a["norm"]), L(q), L(t),
        int(steps), float(np.float32(lr)), L(best), L(bq), L(bt), _threads(nthreads))
    out = _pick(best, bq, bt, nb, S)
    return (out + ((best, bq, bt),)) if return_rows else out


# --------------------------------------------------------------------------------------------
# translation-seeded starts (trans_init=True): accel/drivers/esp.py:228-262 and its twins in
# pharm.py:244-283, vol_color.py:253-291, esp_combo.py:407-460
# --------------------------------------------------------------------------------------------
def select_top(scores, G, topk):
    """Indices (K, topk) of the best-scoring start poses per pair (``coarse_score.topk``),
    rows at or past a pair's pose count G excluded."""
    sc = np.array(scores, np.float64, copy=True)
    Gm = sc.shape[1]
    if topk > int(np.min(G)):
        raise ValueError("topk exceeds a pair's pose count")
    sc[np.arange(Gm)[None, :] >= np.asarray(G)[:, None]] = -np.inf
    return np.argsort(-sc, axis=1, kind="stable")[:, :topk]


def align_trans(align_fn, args, grid_q, grid_t, G, *, topk=30, steps=100, **kw):
    """Coarse grid + top-k + fine: every grid pose scored once (the row scores of a one-step
    run are the seeds' own scores), the ``topk`` best per pair refined for ``steps``.
    ``align_fn`` is one of the align_* drivers above, called with ``args`` and ``kw``."""
    grid_q, grid_t = _f32(grid_q), _f32(grid_t)
    K, Gm = grid_q.shape[:2]
    *_, (best, _, _) = align_fn(*args, seeds=(grid_q, grid_t), steps=1, return_rows=True, **kw)
    idx = select_top(best.reshape(K, Gm), G, topk)
    sq = np.take_along_axis(grid_q, idx[..., None], 1)
    st = np.take_along_axis(grid_t, idx[..., None], 1)
    return align_fn(*args, seeds=(sq, st), steps=steps, **kw)
