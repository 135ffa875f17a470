"""float64 numpy restatement of the reference scoring functions (test infrastructure only).

* :func:`vab` / :func:`shape_tanimoto`  -- VAB_2nd_order / shape_tanimoto
  (shepherd_score/score/gaussian_overlap.py:16-70)
* :func:`esp_tanimoto`  -- VAB_2nd_order_esp / get_overlap_esp (score/electrostatic_scoring.py:17-120)
* :func:`pharm_tanimoto` -- get_overlap_pharm with similarity='tanimoto', no extended points
  (score/pharmacophore_scoring.py:422-913): per-type Gaussian overlaps, cosine weight
  (clamp(cos,0,1)+2)/3 for acceptor/donor/halogen, (|cos|+2)/3 for aromatic, isotropic for
  the rest (all isotropic with ``directionless=True``), totals summed over types
* :func:`combo_score` -- get_pharm_combo_score (pharmacophore_scoring.py:915-974)
* the analytic coordinate / charge gradients of the shape and ESP Tanimoto scores, which
  the reference obtains by torch autograd (checked against its autograd in the golden
  fixtures and against central finite differences in the tests).
"""
from __future__ import annotations

import numpy as np

P_ALPHA = np.array([1.0, 1.0, 0.7, 0.7, 1.0, 1.0, 1.0, 1.0, 1.0])
DIRECTIONAL = {0: False, 1: False, 4: False, 2: True}   # type -> allow_antiparallel


def _d2(x, y):
    return ((x[:, None, :] - y[None, :, :]) ** 2).sum(-1)


def _kc(alpha):
    return np.pi ** 1.5 / (2.0 * alpha) ** 1.5


def vab(x, y, alpha, cx=None, cy=None, lam=None):
    """Gaussian overlap sum_ij K exp(-alpha/2 r^2) [* exp(-(cx-cy)^2/lam)] in float64."""
    x = np.asarray(x, np.float64); y = np.asarray(y, np.float64)
    g = np.exp(-(alpha / 2.0) * _d2(x, y))
    if cx is not None:
        dc = np.asarray(cx, np.float64)[:, None] - np.asarray(cy, np.float64)[None, :]
        g = g * np.exp(-(dc * dc) / lam)
    return _kc(alpha) * g.sum()


def shape_tanimoto(x, y, alpha):
    ab, aa, bb = vab(x, y, alpha), vab(x, x, alpha), vab(y, y, alpha)
    return ab / (aa + bb - ab)


def esp_tanimoto(x, y, cx, cy, alpha, lam):
    ab = vab(x, y, alpha, cx, cy, lam)
    aa = vab(x, x, alpha, cx, cx, lam)
    bb = vab(y, y, alpha, cy, cy, lam)
    return ab / (aa + bb - ab)


def _vab_grads(x, y, alpha, cx=None, cy=None, lam=None):
    """d V_xy / d x (N,3), d V_xy / d y (M,3), and charge grads (N,), (M,)."""
    x = np.asarray(x, np.float64); y = np.asarray(y, np.float64)
    diff = x[:, None, :] - y[None, :, :]
    g = np.exp(-(alpha / 2.0) * (diff ** 2).sum(-1))
    dc = None
    if cx is not None:
        dc = np.asarray(cx, np.float64)[:, None] - np.asarray(cy, np.float64)[None, :]
        g = g * np.exp(-(dc * dc) / lam)
    g = _kc(alpha) * g
    gx = -alpha * (g[..., None] * diff).sum(1)
    gy = alpha * (g[..., None] * diff).sum(0)
    if dc is None:
        return gx, gy, None, None
    gcx = (-2.0 / lam) * (g * dc).sum(1)
    gcy = (2.0 / lam) * (g * dc).sum(0)
    return gx, gy, gcx, gcy


def _tanimoto_grads(x, y, alpha, cx=None, cy=None, lam=None):
    ab = vab(x, y, alpha, cx, cy, lam)
    aa = vab(x, x, alpha, cx, cx, lam)
    bb = vab(y, y, alpha, cy, cy, lam)
    U = aa + bb
    D = U - ab
    dAB, dSelf = U / D ** 2, -ab / D ** 2
    gx_ab, gy_ab, gcx_ab, gcy_ab = _vab_grads(x, y, alpha, cx, cy, lam)
    gx_aa, gx_aa2, gcx_aa, gcx_aa2 = _vab_grads(x, x, alpha, cx, cx, lam)
    gy_bb, gy_bb2, gcy_bb, gcy_bb2 = _vab_grads(y, y, alpha, cy, cy, lam)
    gx = dAB * gx_ab + dSelf * (gx_aa + gx_aa2)
    gy = dAB * gy_ab + dSelf * (gy_bb + gy_bb2)
    if cx is None:
        return gx, gy, None, None
    gcx = dAB * gcx_ab + dSelf * (gcx_aa + gcx_aa2)
    gcy = dAB * gcy_ab + dSelf * (gcy_bb + gcy_bb2)
    return gx, gy, gcx, gcy


def shape_tanimoto_grad(x, y, alpha):
    gx, gy, _, _ = _tanimoto_grads(x, y, alpha)
    return gx, gy


def esp_tanimoto_grad(x, y, cx, cy, alpha, lam):
    return _tanimoto_grads(x, y, alpha, cx, cy, lam)


def _unit(v):
    v = np.asarray(v, np.float64)
    return v / np.maximum(np.linalg.norm(v, axis=-1, keepdims=True), 1e-12)


def _pharm_overlaps(t1, t2, a1, a2, v1, v2, directionless):
    """Total (VAB, VAA, VBB) summed over pharmacophore types."""
    t1 = np.asarray(t1); t2 = np.asarray(t2)
    tot = np.zeros(3)
    for ty in np.unique(np.concatenate([t1, t2])):
        ty = int(ty)
        if ty == 8:
            continue
        m1, m2 = t1 == ty, t2 == ty
        alpha = P_ALPHA[ty]
        K = _kc(alpha)

        def ov(xa, xv, ya, yv):
            g = np.exp(-(alpha / 2.0) * _d2(xa, ya))
            if not directionless and ty in DIRECTIONAL:
                c = _unit(xv) @ _unit(yv).T
                c = np.abs(c) if DIRECTIONAL[ty] else np.clip(c, 0.0, 1.0)
                g = g * (c + 2.0) / 3.0
            return K * g.sum()

        A1, A2 = np.asarray(a1, np.float64)[m1], np.asarray(a2, np.float64)[m2]
        V1, V2 = np.asarray(v1, np.float64)[m1], np.asarray(v2, np.float64)[m2]
        tot += [ov(A1, V1, A2, V2), ov(A1, V1, A1, V1), ov(A2, V2, A2, V2)]
    return tot


def pharm_tanimoto(t1, t2, a1, a2, v1, v2, directionless=False):
    ab, aa, bb = _pharm_overlaps(t1, t2, a1, a2, v1, v2, directionless)
    return ab / (aa + bb - ab)


def combo_score(c1, c2, t1, t2, a1, a2, v1, v2, alpha=0.81, w=0.5, directionless=False):
    return (1 - w) * shape_tanimoto(c1, c2, alpha) + w * pharm_tanimoto(t1, t2, a1, a2, v1, v2,
                                                                        directionless)
