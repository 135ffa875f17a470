"""numpy restatement of the reference seed generator (test infrastructure only).

Follows ``batched_seeds_torch`` (shepherd_score/accel/drivers/_common.py:281-441) step by
step: identity, 4 PCA-alignment quaternions (fp64 closed-form eigensolver,
``_analytic_sym3x3_axes`` :207-255 / ``_masked_principal_axes`` :258-278), up to 6
structured +/-90 degree axis-swap seeds (:401-413), a Fibonacci fill
(``_quats_from_fibo``, shepherd_score/alignment/_torch.py:173-195 with
``_get_points_fibonacci``, generate_point_cloud.py:234-261), COM-aligning translations
(:425-428) and the fixed fallback set for degenerate pairs (:189-204, :430-439).
Dtypes follow the reference: the PCA in float64, everything else in float32.
"""
from __future__ import annotations

import math

import numpy as np

_TWO_PI_3 = 2.0 * math.pi / 3.0


def quat_mul(q, r):
    """Hamilton product, (w,x,y,z) convention (_common.py:35-56)."""
    w1, x1, y1, z1 = np.moveaxis(q, -1, 0)
    w2, x2, y2, z2 = np.moveaxis(r, -1, 0)
    return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
                     w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                     w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], axis=-1)


def _normalize(v, eps=1e-12):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.maximum(n, eps)


def quat_to_rotmat(q):
    """(...,4) -> (...,3,3) after normalising q (_common.py:59-97)."""
    q = _normalize(q)
    w, x, y, z = np.moveaxis(q, -1, 0)
    R = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                  2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                  2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], axis=-1)
    return R.reshape(q.shape[:-1] + (3, 3)).astype(q.dtype)


def fibonacci_points(n: int) -> np.ndarray:
    """Golden-spiral points on the unit sphere (generate_point_cloud.py:234-261)."""
    offset = 2.0 / n
    increment = np.pi * (3.0 - np.sqrt(5.0))
    i = np.arange(n)
    y = ((i * offset) - 1) + (offset / 2)
    r = np.sqrt(1 - np.square(y))
    phi = np.mod((i + 1), n) * increment
    return np.column_stack((np.cos(phi) * r, y, np.sin(phi) * r))


def quats_from_fibo(n: int) -> np.ndarray:
    """Quaternions rotating +x onto each Fibonacci point, float32 (alignment/_torch.py:173-195)."""
    fibo = fibonacci_points(n).astype(np.float32)
    unit = np.tile(np.array([1.0, 0.0, 0.0], np.float32), (n, 1))
    ang = np.arccos(np.clip((unit * fibo).sum(1), -1.0, 1.0)).astype(np.float32)[:, None]
    same = np.isclose(unit, fibo).sum(1) == 3
    axes = np.zeros((n, 3), np.float32)
    axes[:, 0] = 1.0
    cr = np.cross(unit, fibo).astype(np.float32)
    axes[~same] = cr[~same]
    axes = _normalize(axes).astype(np.float32)
    half = ang / np.float32(2.0)
    return np.concatenate([np.cos(half), axes * np.sin(half)], axis=1).astype(np.float32)


def fallback_quats(num: int) -> np.ndarray:
    """Deterministic rotations for degenerate pairs (_common.py:189-204)."""
    s2 = math.sqrt(0.5)
    base = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1], [s2, s2, 0, 0],
                     [s2, 0, s2, 0], [s2, 0, 0, s2], [0, s2, s2, 0], [0, s2, 0, s2],
                     [0, 0, s2, s2]], np.float32)
    reps = (num + len(base) - 1) // len(base)
    return _normalize(np.tile(base, (reps, 1))[:num]).astype(np.float32)


def sym3x3_axes(M: np.ndarray, eps: float = 1e-12) -> np.ndarray:
    """Rows = eigenvectors, descending eigenvalue, of symmetric 3x3 (K,3,3) (_common.py:207-255)."""
    a00, a11, a22 = M[:, 0, 0], M[:, 1, 1], M[:, 2, 2]
    a01, a02, a12 = M[:, 0, 1], M[:, 0, 2], M[:, 1, 2]
    q = (a00 + a11 + a22) / 3.0
    p1 = a01 * a01 + a02 * a02 + a12 * a12
    p2 = (a00 - q) ** 2 + (a11 - q) ** 2 + (a22 - q) ** 2 + 2.0 * p1
    p = np.sqrt(np.maximum(p2 / 6.0, eps))
    ip = 1.0 / p
    b00, b11, b22 = (a00 - q) * ip, (a11 - q) * ip, (a22 - q) * ip
    b01, b02, b12 = a01 * ip, a02 * ip, a12 * ip
    detB = (b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02)
            + b02 * (b01 * b12 - b11 * b02))
    r = np.clip(detB * 0.5, -1.0, 1.0)
    phi = np.arccos(r) / 3.0
    e1 = q + 2.0 * p * np.cos(phi)
    e3 = q + 2.0 * p * np.cos(phi + _TWO_PI_3)
    e2 = 3.0 * q - e1 - e3
    I = np.broadcast_to(np.eye(3, dtype=M.dtype), M.shape)
    ar = np.arange(M.shape[0])

    def evec(lj, lk):
        P = np.matmul(M - lj[:, None, None] * I, M - lk[:, None, None] * I)
        idx = np.linalg.norm(P, axis=1).argmax(axis=1)
        col = P[ar, :, idx]
        nrm = np.linalg.norm(col, axis=1, keepdims=True)
        return col / np.maximum(nrm, eps), nrm[:, 0]

    v1, n1 = evec(e2, e3)
    v3, n3 = evec(e1, e2)
    v2 = _normalize(np.cross(v3, v1), eps)
    v1 = _normalize(np.cross(v2, v3), eps)
    R = np.stack([v1, v2, v3], axis=1)
    bad = (n1 < 1e-9) | (n3 < 1e-9) | ~np.isfinite(R).all(axis=(1, 2))
    return np.where(bad[:, None, None], I, R)


def masked_principal_axes(points: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Principal axes of the masked points (_common.py:258-278)."""
    n = np.maximum(mask.sum(1), 1.0)
    com = (points * mask[..., None]).sum(1) / n[:, None]
    centered = (points - com[:, None, :]) * mask[..., None]
    A = (centered ** 2).sum((1, 2))
    Bm = np.matmul(centered.transpose(0, 2, 1), centered)
    inertia = A[:, None, None] * np.eye(3) - Bm
    return sym3x3_axes(inertia)


def batched_seeds(A: np.ndarray, B: np.ndarray, N_real, M_real, num_seeds: int = 50):
    """Seeds (K,S,4) float32 and translations (K,S,3) float32 (_common.py:281-441).

    A (K,Npad,3), B (K,Mpad,3) float32 padded clouds; N_real/M_real (K,) counts.
    """
    A = np.asarray(A, np.float32)
    B = np.asarray(B, np.float32)
    K, Npad, _ = A.shape
    Mpad = B.shape[1]
    N_real = np.asarray(N_real).astype(np.int64)
    M_real = np.asarray(M_real).astype(np.int64)
    if num_seeds == 1:
        q = np.zeros((K, 1, 4), np.float32)
        q[:, :, 0] = 1.0
        return q, np.zeros((K, 1, 3), np.float32)
    if num_seeds < 5:
        num_seeds = 5
    mask_n = (np.arange(Npad)[None] < N_real[:, None]).astype(np.float32)
    mask_m = (np.arange(Mpad)[None] < M_real[:, None]).astype(np.float32)
    nreal = np.maximum(mask_n.sum(1), 1.0).astype(np.float32)
    mreal = np.maximum(mask_m.sum(1), 1.0).astype(np.float32)
    ref_com = ((A * mask_n[..., None]).sum(1, dtype=np.float32) / nreal[:, None]).astype(np.float32)
    fit_com = ((B * mask_m[..., None]).sum(1, dtype=np.float32) / mreal[:, None]).astype(np.float32)

    A64 = np.nan_to_num(A.astype(np.float64))
    B64 = np.nan_to_num(B.astype(np.float64))
    mn64 = mask_n.astype(np.float64)
    mm64 = mask_m.astype(np.float64)
    ref_axes = masked_principal_axes(A64, mn64)
    ref_axes4 = np.repeat(ref_axes[:, None], 4, axis=1).copy()
    ref_axes4[:, 1, 0] *= -1
    ref_axes4[:, 2, 1] *= -1
    ref_axes4[:, 3, 0] *= -1
    ref_axes4[:, 3, 1] *= -1
    ref_axes_f = ref_axes4.reshape(4 * K, 3, 3)
    fit_c = (B64 - fit_com.astype(np.float64)[:, None, :]) * mm64[..., None]
    fit4 = np.repeat(fit_c[:, None], 4, axis=1).reshape(4 * K, Mpad, 3)
    mask_m4 = np.repeat(mm64[:, None], 4, axis=1).reshape(4 * K, Mpad)
    quat_order = [None, None]
    for ax in range(2):
        fit_axes = masked_principal_axes(fit4, mask_m4)
        v1 = fit_axes[:, ax]
        v2 = ref_axes_f[:, ax]
        cos = np.clip((v1 * v2).sum(1, keepdims=True), -1.0, 1.0)
        angle = np.arccos(cos)
        axis = np.cross(v1, v2)
        an = np.linalg.norm(axis, axis=1, keepdims=True)
        axis = np.where(an < 1e-8, np.array([1.0, 0.0, 0.0]), axis / np.maximum(an, 1e-12))
        half = angle * 0.5
        q = np.concatenate([np.cos(half), axis * np.sin(half)], axis=1)
        quat_order[ax] = q
        R = quat_to_rotmat(q)
        fit4 = np.einsum('kni,kji->knj', fit4, R) * mask_m4[..., None]
    pca = quat_mul(quat_order[1], quat_order[0]).reshape(K, 4, 4).astype(np.float32)

    identity = np.zeros((K, 1, 4), np.float32)
    identity[:, :, 0] = 1.0
    n_struct = min(max(num_seeds - 5, 0), 6)
    if n_struct > 0:
        base = pca[:, 0]
        axes = ref_axes.astype(np.float32)
        ch = np.float32(math.cos(math.pi / 4))
        sgn = np.array([math.sin(math.pi / 4), -math.sin(math.pi / 4)], np.float32)
        w = np.full((K, 3, 2, 1), ch, np.float32)
        xyz = sgn.reshape(1, 1, 2, 1) * axes.reshape(K, 3, 1, 3)
        q_ax = np.concatenate([w, xyz], axis=-1).reshape(K, 6, 4)[:, :n_struct]
        base_rep = np.broadcast_to(base[:, None], (K, n_struct, 4)).reshape(-1, 4)
        struct = quat_mul(q_ax.reshape(-1, 4), base_rep).reshape(K, n_struct, 4).astype(np.float32)
    else:
        struct = np.zeros((K, 0, 4), np.float32)
    n_fibo = max(num_seeds - 5 - n_struct, 0)
    fibo = (np.broadcast_to(quats_from_fibo(n_fibo)[None], (K, n_fibo, 4)) if n_fibo > 0
            else np.zeros((K, 0, 4), np.float32))
    quats = np.concatenate([identity, pca, struct, fibo], axis=1)[:, :num_seeds]
    quats = _normalize(quats).astype(np.float32)

    R_all = quat_to_rotmat(quats.reshape(-1, 4)).reshape(K, num_seeds, 3, 3)
    rot_fit_com = np.einsum('ksij,kj->ksi', R_all, fit_com).astype(np.float32)
    trans = (ref_com[:, None, :] - rot_fit_com).astype(np.float32)

    valid = ((N_real >= 3) & (M_real >= 3) & np.isfinite(A).all(axis=(1, 2))
             & np.isfinite(B).all(axis=(1, 2)))
    if not valid.all():
        fb_q = np.broadcast_to(fallback_quats(num_seeds)[None], (K, num_seeds, 4))
        fb_t = np.broadcast_to((ref_com - fit_com)[:, None, :], (K, num_seeds, 3))
        quats = np.where(valid[:, None, None], quats, fb_q).astype(np.float32)
        trans = np.where(valid[:, None, None], trans, fb_t).astype(np.float32)
    return quats, trans
