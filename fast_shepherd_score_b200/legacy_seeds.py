"""Start poses of the translation-seeded (``trans_init=True``) alignment path.

The reference builds them per pair on the host (accel/drivers/_common.py:156-186 calling
alignment/_torch.py:329-399): pose 0 is the identity with the centres of mass matched; poses
1-4 rotate the fit cloud's principal axes onto the reference's in the four sign combinations of
the two longest axes (alignment/utils/pca_np.py:111-166); then, for every translation centre c,
``per_trans`` Fibonacci-sphere rotations R with t = c - R com_fit.  G = 5 + per_trans * n_c.

The principal axes are eigenvectors of the float64 inertia tensor from ``np.linalg.eigh``,
as the reference computes them, so the eigenvector signs LAPACK picks carry over unchanged (a
closed-form eigensolver would flip some of them and change poses 1-4).  Translations and
rotation matrices use float32 arithmetic like the reference's.  Everything here runs over a
whole batch of pairs at once on the clouds' device (padded tensors; only the batched 3x3
``eigh`` of each axis step goes to the host) instead of the reference's per-pair Python loop;
the results agree with it to float32 rounding.  This is seed construction only: the candidate
poses are scored and refined by the fused CUDA kernel.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch
import torch.nn.functional as F

from .kernels import _fibo_host

def _inertia_axes(X: torch.Tensor, mask: torch.Tensor, n: torch.Tensor) -> np.ndarray:
    """Principal axes of padded clouds X (P,L,3) (any device) with real-point mask (P,L):
    numpy (P,3,3), rows = axes, largest inertia moment first (pca_np.py:12-33: recentre,
    (tr(x^T x) I - x^T x) / n in float64, eigh, descending order).  The sums run where X lives;
    the 3x3 eigenproblems go to LAPACK on the host, as in the reference."""
    dt = X.dtype
    mean = X.sum(1) / n.to(dt)[:, None]
    x = (X - mean[:, None, :]) * mask[..., None].to(dt)
    trace = (x * x).sum((1, 2))
    B = torch.bmm(x.transpose(1, 2), x)
    eye = torch.eye(3, dtype=torch.float64, device=X.device)
    T = (trace.double()[:, None, None] * eye - B.double()) / n.double()[:, None, None]
    vals, vecs = np.linalg.eigh(T.cpu().numpy())
    order = np.argsort(-vals, axis=1)
    return np.take_along_axis(vecs, order[:, None, :], axis=2).transpose(0, 2, 1)


def _axis_angle_quat(v_from: np.ndarray, v_to: np.ndarray) -> np.ndarray:
    """(P,4) quaternions (w, x, y, z) turning directions v_from onto v_to (P,3) about their
    common normal (pca_np.py:36-76); parallel inputs give the x axis and angle 0."""
    nrm = lambda v: np.sqrt((v * v).sum(1, keepdims=True))
    u = v_from / nrm(v_from)
    w = v_to / nrm(v_to)
    angle = np.arccos(np.clip((u * w).sum(1), -1.0, 1.0))
    same = np.all(np.abs(v_from - v_to) <= 1e-8 + 1e-5 * np.abs(v_to), axis=1)
    cr = np.cross(v_from, v_to)
    cn = nrm(cr)
    # antiparallel directions have no common normal (the reference's axis would be 0/0):
    # turn half way round an axis perpendicular to v_from instead
    perp = np.cross(v_from, np.where(np.abs(u[:, :1]) < 0.9, np.array([1.0, 0.0, 0.0]),
                                     np.array([0.0, 1.0, 0.0])))
    cr = np.where(cn > 0, cr, perp)
    cn = nrm(cr)
    axis = np.where(same[:, None], np.array([1.0, 0.0, 0.0]), cr / np.where(cn > 0, cn, 1.0))
    sq = (axis * axis).sum(1, keepdims=True)
    axis = np.where(np.abs(1.0 - sq) > 1e-12, axis / np.sqrt(np.where(sq > 0, sq, 1.0)), axis)
    h = angle / 2.0
    return np.concatenate([np.cos(h)[:, None], axis * np.sin(h)[:, None]], 1)


def _quat_matrix(q: np.ndarray) -> np.ndarray:
    """(P,3,3) rotation matrices of quaternions (P,4), normalised first (se3_np.py:13-50)."""
    q = q / np.sqrt((q * q).sum(1, keepdims=True))
    r, i, j, k = q.T
    s = 2.0 / (q * q).sum(1)
    return np.stack([1 - s * (j * j + k * k), s * (i * j - k * r), s * (i * k + j * r),
                     s * (i * j + k * r), 1 - s * (i * i + k * k), s * (j * k - i * r),
                     s * (i * k - j * r), s * (j * k + i * r), 1 - s * (i * i + j * j)],
                    1).reshape(-1, 3, 3)


def _quat_mul(p: np.ndarray, q: np.ndarray) -> np.ndarray:
    """Hamilton products p * q of (P,4) batches (rotation q first, then p)."""
    pw, px, py, pz = p.T
    qw, qx, qy, qz = q.T
    return np.stack([pw * qw - px * qx - py * qy - pz * qz,
                     px * qw + pw * qx - pz * qy + py * qz,
                     py * qw + pz * qx + pw * qy - px * qz,
                     pz * qw - py * qx + px * qy + pw * qz], 1)


def pca_quats(R: torch.Tensor, nr: torch.Tensor, Fp: torch.Tensor,
              nf: torch.Tensor) -> np.ndarray:
    """The four principal-axis quaternions, numpy (P,4,4), of padded float32 clouds R (P,Lr,3)
    / Fp (P,Lf,3) (zero padding) with real counts nr / nf (tensors on the clouds' device)."""
    dev = R.device
    mr = torch.arange(R.shape[1], device=dev)[None, :] < nr[:, None]
    mf = torch.arange(Fp.shape[1], device=dev)[None, :] < nf[:, None]
    axes_ref = _inertia_axes(R, mr, nr)
    fit0 = (Fp - (Fp.sum(1) / nf.to(Fp.dtype)[:, None])[:, None, :]) * mf[..., None]
    axes_fit0 = _inertia_axes(fit0, mf, nf)   # identical for the four sign patterns
    out = np.zeros((R.shape[0], 4, 4))
    # sign patterns of the (longest, second) reference axes: (+,+), (-,+), (+,-), (-,-)
    for idx, (s0, s1) in enumerate(((1, 1), (-1, 1), (1, -1), (-1, -1))):
        q0 = _axis_angle_quat(axes_fit0[:, 0], s0 * axes_ref[:, 0])
        rot = torch.from_numpy(_quat_matrix(q0)).to(dev)
        cur = torch.bmm(fit0.double(), rot.transpose(1, 2))      # (rot x^T)^T per pair
        axes_fit1 = _inertia_axes(cur, mf, nf)
        q1 = _axis_angle_quat(axes_fit1[:, 1], s1 * axes_ref[:, 1])
        out[:, idx] = _quat_mul(q1, q0)
    return out


def _rot32(q: torch.Tensor, normalise: bool = True) -> torch.Tensor:
    """(n,4) float32 -> (n,3,3) rotation matrices (quaternions normalised first unless they
    already are, as the reference's SE(3) builder does)."""
    if normalise:
        q = F.normalize(q, p=2, dim=1)
    r, i, j, k = q.unbind(1)
    s = 2.0 / (q ** 2).sum(1)
    return torch.stack((1 - s * (j * j + k * k), s * (i * j - k * r), s * (i * k + j * r),
                        s * (i * j + k * r), 1 - s * (i * i + k * k), s * (j * k - i * r),
                        s * (i * k - j * r), s * (j * k + i * r), 1 - s * (i * i + j * j)),
                       1).reshape(-1, 3, 3)


def _rotate(R: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
    """R (n,3,3) applied to points p (n,3) -> (n,3), as the reference's batched transform."""
    n = R.shape[0]
    z = torch.zeros(n, 1, 3, dtype=p.dtype, device=p.device)
    return torch.baddbmm(z, p.reshape(n, 1, 3), R.transpose(1, 2))[:, 0, :]


def grid_padded(R: torch.Tensor, nr, Fp: torch.Tensor, nf, C: torch.Tensor, nc,
                per_trans: int = 10):
    """Legacy start grids of P pairs from padded float32 tensors (any device): reference clouds
    R (P,Lr,3), fit clouds Fp (P,Lf,3), translation centres C (P,Lc,3), zero padding, real
    counts nr / nf / nc.  Returns q (P,Gmax,4), t (P,Gmax,3) float32 on R's device and G (P,)
    numpy int64; rows past a pair's G repeat its pose 0."""
    dev = R.device
    nr, nf, nc = (torch.as_tensor(x, device=dev).to(torch.int64).reshape(-1)
                  for x in (nr, nf, nc))
    P = R.shape[0]
    ncn = nc.cpu().numpy()
    if P and (int(nr.min()) < 1 or int(nf.min()) < 1):
        raise ValueError("translation-seeded starts need non-empty clouds")
    R, Fp = R.to(torch.float32), Fp.to(torch.float32)
    C = C.to(torch.float32).reshape(P, C.shape[-2] if C.dim() == 3 else -1, 3)
    G = 5 + per_trans * ncn
    Gm = int(G.max()) if P else 5
    if P == 0:
        return torch.zeros(0, Gm, 4, device=dev), torch.zeros(0, Gm, 3, device=dev), G
    com_ref = R.sum(1) / nr.to(torch.float32)[:, None]
    com_fit = Fp.sum(1) / nf.to(torch.float32)[:, None]
    q = torch.zeros(P, Gm, 4, device=dev)
    t = torch.zeros(P, Gm, 3, device=dev)
    q[:, 0, 0] = 1.0
    t[:, 0] = com_ref - com_fit
    q[:, 1:5] = torch.from_numpy(pca_quats(R, nr, Fp, nf)).to(dev, torch.float32)
    Tp = _rotate(_rot32(q[:, 1:5].reshape(-1, 4)), com_fit.repeat_interleave(4, 0))
    t[:, 1:5] = com_ref[:, None, :] - Tp.reshape(P, 4, 3)
    if Gm > 5:
        qf = F.normalize(torch.from_numpy(_fibo_host(per_trans)).to(dev), p=2, dim=1)
        Tf = _rotate(_rot32(qf, normalise=False).repeat(P, 1, 1),
                     com_fit.repeat_interleave(per_trans, 0)).reshape(P, per_trans, 3)
        j = torch.arange(Gm - 5, device=dev)
        ci, r = j // per_trans, j % per_trans            # centre, rotation of pose 5 + j
        pad = ci[None, :] >= nc[:, None]
        qg = qf[r].expand(P, -1, -1)
        tg = C[:, ci.clamp(max=C.shape[1] - 1)] - Tf[:, r]
        q[:, 5:] = torch.where(pad[..., None], q[:, :1], qg)
        t[:, 5:] = torch.where(pad[..., None], t[:, :1], tg)
    return F.normalize(q, dim=2), t, G


def pair_grid(ref, fit, centres, per_trans: int = 10):
    """Legacy start poses of one pair: q (G,4), t (G,3) float32 CPU tensors."""
    f = lambda a: torch.as_tensor(np.asarray(a, np.float32)).reshape(1, -1, 3)
    R, Fp, C = f(ref), f(fit), f(centres)
    q, t, G = grid_padded(R, [R.shape[1]], Fp, [Fp.shape[1]], C, [C.shape[1]], per_trans)
    return q[0, :G[0]], t[0, :G[0]]


def _gather_padded(cs, idx: torch.Tensor, shift: Optional[torch.Tensor] = None):
    """Padded (len(idx), L, 3) float32 points (on the set's device) of molecules idx of a packed
    CloudSet and their counts; ``shift`` (n_mol,3) is subtracted from each molecule's points."""
    dev = cs.pts.device
    cnt = torch.as_tensor(np.asarray(cs.counts, np.int64), device=dev)
    off = torch.cumsum(cnt, 0) - cnt
    n = cnt[idx]
    L = max(int(n.max()) if len(n) else 0, 1)
    ar = torch.arange(L, device=dev)[None, :]
    mask = ar < n[:, None]
    if cs.pts.shape[0] == 0:
        return torch.zeros(len(idx), L, 3, device=dev), n
    rows = torch.where(mask, off[idx][:, None] + ar, torch.zeros_like(ar))
    X = cs.pts[:, :3][rows]
    if shift is not None:
        X = X - shift.to(dev, torch.float32)[idx][:, None, :]
    return torch.where(mask[..., None], X, torch.zeros_like(X)), n


def grid_packed(ref, fit, centres, pair_ref, pair_fit, per_trans: int = 10,
                centre_shift: Optional[torch.Tensor] = None):
    """Padded legacy grids of a batch of pairs over packed clouds (``layout.CloudSet``):
    q (P,Gmax,4), t (P,Gmax,3) on the clouds' device and the per-pair pose counts G (P,) numpy.
    ``centres`` is a CloudSet indexed like ``ref`` (one centre list per reference molecule);
    ``centre_shift`` (n_ref,3), if given, is subtracted from each molecule's centres (the
    pharmacophore path works on centred clouds).  Rows past a pair's G repeat its pose 0."""
    dev = ref.pts.device
    pr = torch.as_tensor(pair_ref, device=dev).to(torch.int64)
    pf = torch.as_tensor(pair_fit, device=dev).to(torch.int64)
    R, nr = _gather_padded(ref, pr)
    Fp, nf = _gather_padded(fit, pf)
    C, nc = _gather_padded(centres, pr, centre_shift)
    return grid_padded(R, nr, Fp, nf, C, nc, per_trans)


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
