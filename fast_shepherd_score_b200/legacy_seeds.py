"""Start poses of the translation-seeded (``trans_init=True``) alignment path.

The reference builds them per pair on the host (accel/drivers/_common.py:156-186 calling
alignment/_torch.py:329-399): pose 0 is the identity with the centres of mass matched; poses
1-4 rotate the fit cloud's principal axes onto the reference's in the four sign combinations of
the two longest axes (alignment/utils/pca_np.py:111-166); then, for every translation centre c,
``per_trans`` Fibonacci-sphere rotations R with t = c - R com_fit.  G = 5 + per_trans * n_c.

The principal axes are eigenvectors of the float64 inertia tensor from ``np.linalg.eigh``,
exactly as the reference computes them, so the eigenvector signs LAPACK picks carry over
unchanged (a closed-form eigensolver would flip some of them and change poses 1-4).  The
translations and rotation matrices use float32 torch arithmetic on the host like the
reference's.  This is seed construction only; the candidate poses are scored and refined by the
CUDA kernels.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch
import torch.nn.functional as F

from .kernels import _fibo_host


def _inertia_axes(points: np.ndarray) -> np.ndarray:
    """Rows = principal axes, largest inertia moment first (pca_np.py:12-33)."""
    x = points - np.mean(points, axis=0)
    trace = np.sum(x ** 2)
    tensor = (trace * np.eye(3) - x.T @ x) / x.shape[0]
    vals, vecs = np.linalg.eigh(tensor)
    return vecs[:, np.argsort(-vals)].T


def _axis_angle_quat(v_from: np.ndarray, v_to: np.ndarray) -> np.ndarray:
    """Quaternion (w, x, y, z) of the rotation taking direction v_from onto v_to about their
    common normal (pca_np.py:36-76); parallel inputs give the x axis and angle 0."""
    u = v_from / np.linalg.norm(v_from)
    w = v_to / np.linalg.norm(v_to)
    angle = np.arccos(np.clip(np.dot(u, w), -1.0, 1.0))
    if np.allclose(v_from, v_to):
        axis = np.array([1, 0, 0])
    else:
        n = np.cross(v_from, v_to)
        axis = n / np.linalg.norm(n)
    sq = np.dot(axis, axis)
    if abs(1.0 - sq) > 1e-12:
        axis = axis / np.sqrt(sq)
    h = angle / 2.0
    return np.array([np.cos(h), *(axis * np.sin(h))])


def _quat_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrix of a quaternion (normalised first), row-major (se3_np.py:13-50)."""
    q = q / np.linalg.norm(q)
    r, i, j, k = q
    s = 2.0 / (q * q).sum()
    return np.array([[1 - s * (j * j + k * k), s * (i * j - k * r), s * (i * k + j * r)],
                     [s * (i * j + k * r), 1 - s * (i * i + k * k), s * (j * k - i * r)],
                     [s * (i * k - j * r), s * (j * k + i * r), 1 - s * (i * i + j * j)]])


def _quat_mul(p: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Hamilton product p * q (rotation q first, then p)."""
    pw, px, py, pz = p
    return np.array([[pw, -px, -py, -pz], [px, pw, -pz, py], [py, pz, pw, -px],
                     [pz, -py, px, pw]]) @ q


def pca_quats(ref: np.ndarray, fit: np.ndarray) -> np.ndarray:
    """The four principal-axis quaternions (4, 4) for the centred fit cloud."""
    axes_ref = _inertia_axes(ref)
    out = np.zeros((4, 4))
    # sign patterns of (longest, second) reference axes: (+,+), (-,+), (+,-), (-,-)
    for idx, (s0, s1) in enumerate(((1, 1), (-1, 1), (1, -1), (-1, -1))):
        target = axes_ref.copy()
        target[0] = s0 * axes_ref[0]
        target[1] = s1 * axes_ref[1]
        cur = fit - np.mean(fit, axis=0)
        steps = []
        for ax in range(2):
            axes_fit = _inertia_axes(cur)
            qa = _axis_angle_quat(axes_fit[ax], target[ax])
            steps.append(qa)
            cur = (_quat_matrix(qa) @ cur.T).T
        out[idx] = _quat_mul(steps[1], steps[0])
    return out


def _rot32(q: torch.Tensor, normalise: bool = True) -> torch.Tensor:
    """(n,4) float32 -> (n,3,3) rotation matrices (quaternions normalised first unless they
    already are, as the reference's SE(3) builder does)."""
    if normalise:
        q = F.normalize(q, p=2, dim=1)
    r, i, j, k = q.unbind(1)
    s = torch.tensor([2.0]) / (q ** 2).sum(1)
    return torch.stack((1 - s * (j * j + k * k), s * (i * j - k * r), s * (i * k + j * r),
                        s * (i * j + k * r), 1 - s * (i * i + k * k), s * (j * k - i * r),
                        s * (i * k - j * r), s * (j * k + i * r), 1 - s * (i * i + j * j)),
                       1).reshape(-1, 3, 3)


def _rotate_point(R: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
    """R (n,3,3) applied to one point p (3,) -> (n,3), as the reference's batched transform."""
    n = R.shape[0]
    pts = p.reshape(1, 1, 3).expand(n, 1, 3)
    return torch.baddbmm(torch.zeros(n, 1, 3), pts, R.transpose(1, 2))[:, 0, :]


def pair_grid(ref: np.ndarray, fit: np.ndarray, centres: np.ndarray, per_trans: int = 10):
    """Legacy start poses of one pair: q (G,4), t (G,3) float32 torch (CPU), G = 5 + per_trans
    * len(centres).  ``ref``/``fit``/``centres`` are the real points (float32)."""
    ref_t = torch.as_tensor(np.ascontiguousarray(ref, dtype=np.float32))
    fit_t = torch.as_tensor(np.ascontiguousarray(fit, dtype=np.float32))
    ctr = torch.as_tensor(np.ascontiguousarray(centres, dtype=np.float32)).reshape(-1, 3)
    com_ref, com_fit = ref_t.mean(0), fit_t.mean(0)
    n_c = ctr.shape[0]
    G = 5 + per_trans * n_c
    q = torch.zeros(G, 4)
    t = torch.zeros(G, 3)
    q[0, 0] = 1.0
    t[0] = com_ref - com_fit
    q[1:5] = torch.from_numpy(pca_quats(ref_t.numpy(), fit_t.numpy())).to(torch.float32)
    t[1:5] = com_ref - _rotate_point(_rot32(q[1:5]), com_fit)
    if per_trans > 0 and n_c > 0:
        qf = F.normalize(torch.from_numpy(_fibo_host(per_trans)), p=2, dim=1)
        Tf = _rotate_point(_rot32(qf, normalise=False), com_fit)
        q[5:] = qf.repeat(n_c, 1)
        t[5:] = torch.repeat_interleave(ctr, per_trans, 0) - Tf.repeat(n_c, 1)
    return F.normalize(q, dim=1), t


def grid_packed(ref, fit, centres, pair_ref, pair_fit, per_trans: int = 10,
                centre_shift: Optional[torch.Tensor] = None):
    """Padded legacy grids of a batch of pairs over packed clouds (``layout.CloudSet``):
    q (P,Gmax,4), t (P,Gmax,3) on the clouds' device and the per-pair pose counts G (P,) numpy.
    ``centres`` is a CloudSet indexed like ``ref`` (one centre list per reference molecule);
    ``centre_shift`` (n_ref,3), if given, is subtracted from each molecule's centres (the
    pharmacophore path works on centred clouds).  Rows past a pair's G repeat its first pose."""
    def host(cs):
        off = np.concatenate([[0], np.cumsum(cs.counts)]).astype(np.int64)
        return cs.pts[:, :3].detach().cpu().numpy(), off, np.asarray(cs.counts, np.int64)

    rp, ro, rn = host(ref)
    fp, fo, fn = host(fit)
    cp, co, cn = host(centres)
    shift = None if centre_shift is None else centre_shift.detach().cpu().numpy()
    pr = torch.as_tensor(pair_ref).cpu().numpy().astype(np.int64)
    pf = torch.as_tensor(pair_fit).cpu().numpy().astype(np.int64)
    qs, ts = [], []
    for i, j in zip(pr, pf):
        if rn[i] < 1 or fn[j] < 1:
            raise ValueError("translation-seeded starts need non-empty clouds")
        c = cp[co[i]:co[i] + cn[i]]
        if shift is not None:
            c = (c - shift[i]).astype(np.float32)
        q, t = pair_grid(rp[ro[i]:ro[i] + rn[i]], fp[fo[j]:fo[j] + fn[j]], c, per_trans)
        qs.append(q)
        ts.append(t)
    P = len(qs)
    G = np.array([q.shape[0] for q in qs], dtype=np.int64)
    Gm = int(G.max()) if P else 0
    qp = torch.zeros(P, Gm, 4)
    tp = torch.zeros(P, Gm, 3)
    for k in range(P):
        qp[k, :G[k]] = qs[k]
        tp[k, :G[k]] = ts[k]
        qp[k, G[k]:] = qs[k][0]
        tp[k, G[k]:] = ts[k][0]
    dev = ref.pts.device
    return qp.to(dev), tp.to(dev), G


def select(scores: torch.Tensor, q: torch.Tensor, t: torch.Tensor, G, topk: int):
    """The top-k start poses per pair by their scored value (padded rows excluded):
    (K,topk,4), (K,topk,3)."""
    K, Gm = q.shape[0], q.shape[1]
    Gt = torch.as_tensor(G, device=q.device)
    if K and topk > int(Gt.min()):
        raise ValueError(f"topk={topk} exceeds the {int(Gt.min())} translation-seeded poses "
                         "of a pair")
    sc = scores.reshape(K, Gm).clone()
    sc[torch.arange(Gm, device=q.device)[None, :] >= Gt[:, None]] = -float("inf")
    idx = sc.topk(k=topk, dim=1).indices
    return (torch.gather(q, 1, idx.unsqueeze(-1).expand(-1, -1, 4)).contiguous(),
            torch.gather(t, 1, idx.unsqueeze(-1).expand(-1, -1, 3)).contiguous())
