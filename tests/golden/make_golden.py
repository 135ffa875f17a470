"""Generate the golden fixtures in this directory by running the REFERENCE implementation.

Run from the repository root on a machine that has the reference source tree:

    python tests/golden/make_golden.py --reference /path/to/fast_shepherd_score

It imports ``shepherd_score`` from that tree (a tiny import-only ``rdkit`` stub is written
to a temporary directory, because ``shepherd_score.alignment`` imports RDKit at module
level but the paths used here never call it), runs the reference's own CPU (numba) path
and its torch scoring functions on small seeded inputs, and writes ``*.npz`` fixtures.
The fixtures pin the oracle (``tests/test_oracle_golden.py``) and the CUDA path
(``tests/test_gpu_parity.py``); neither test needs the reference at run time.

Inputs come from ``fast_shepherd_score_b200.synthetic`` with fixed seeds.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fast_shepherd_score_b200 import synthetic as syn  # noqa: E402

_STUB = {
    "rdkit/__init__.py": "",
    "rdkit/Chem/__init__.py": ("from . import rdchem, rdMolDescriptors, rdMolAlign, AllChem\n"
                               "def GetPeriodicTable():\n    return None\n"
                               "def __getattr__(name):\n    return type(name, (), {})\n"),
    "rdkit/Chem/rdchem.py": "def __getattr__(name):\n    return type(name, (), {})\n",
    "rdkit/Chem/rdMolDescriptors.py": "def __getattr__(name):\n    return type(name, (), {})\n",
    "rdkit/Chem/rdMolAlign.py": "def __getattr__(name):\n    return type(name, (), {})\n",
    "rdkit/Chem/AllChem.py": "def __getattr__(name):\n    return type(name, (), {})\n",
    "rdkit/Geometry/__init__.py": "",
    "rdkit/Geometry/rdGeometry.py": "class Point3D:\n    pass\n",
}


def _install_stub():
    d = tempfile.mkdtemp(prefix="rdkit_stub_")
    for rel, txt in _STUB.items():
        p = os.path.join(d, rel)
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            f.write(txt)
    sys.path.insert(0, d)


def pad(clouds, width=None, fill=0.0, dtype=np.float32):
    """Pad a list of (n_i, ...) arrays into (K, width, ...) plus counts."""
    n = np.array([len(c) for c in clouds], np.int32)
    w = int(width or max(n.max(), 1))
    tail = clouds[0].shape[1:]
    out = np.full((len(clouds), w) + tail, fill, dtype)
    for i, c in enumerate(clouds):
        out[i, :len(c)] = c
    return out, n


def rand_quat(rng, K):
    q = rng.standard_normal((K, 4)).astype(np.float32)
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def rotated_copy(rng, X, shift=1.0):
    R = syn.random_rotation(rng)
    return ((X @ R.T) + shift * rng.standard_normal(3)).astype(np.float32), R


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FSS_REFERENCE"),
                    help="the reference source tree (default: $FSS_REFERENCE)")
    ap.add_argument("--only", default="", help="write only this fixture (e.g. pharm_ext)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference source tree with --reference or $FSS_REFERENCE")
    _install_stub()
    sys.path.insert(0, args.reference)
    if args.only == "pharm_ext":
        return make_pharm_ext()
    if args.only == "esp_combo":
        return make_esp_combo()
    if args.only == "trans_init":
        return make_trans_init()
    import torch
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    from shepherd_score.accel.kernels import cpu as rk
    from shepherd_score.accel.drivers._common import batched_seeds_torch
    from shepherd_score.accel.drivers.shape import coarse_fine_align_many
    from shepherd_score.accel.drivers.esp import coarse_fine_esp_align_many
    from shepherd_score.accel.drivers.pharm import coarse_fine_pharm_align_many
    from shepherd_score.accel.drivers.vol_color import coarse_fine_vol_color_align_many
    from shepherd_score.score.analytical_gradients._torch import build_lookup_tables
    from shepherd_score.score.constants import LAM_SCALING
    from shepherd_score.score.gaussian_overlap import get_overlap
    from shepherd_score.score.electrostatic_scoring import get_overlap_esp
    from shepherd_score.score.pharmacophore_scoring import get_overlap_pharm, get_pharm_combo_score

    T = lambda a: torch.as_tensor(np.ascontiguousarray(a))
    rng = np.random.default_rng(1234)

    # ---------------- single-evaluation kernels -------------------------------------
    sizes = [(1, 1), (2, 3), (3, 2), (15, 17), (17, 15), (31, 33), (33, 31), (50, 48)]
    refs = syn.ball_clouds(rng, [a for a, _ in sizes])
    fits = syn.ball_clouds(rng, [b for _, b in sizes])
    A, Nr = pad(refs)
    B, Mr = pad(fits)
    K = len(sizes)
    q = rand_quat(rng, K)
    t = (0.8 * rng.standard_normal((K, 3))).astype(np.float32)
    CA = (0.3 * rng.standard_normal(A.shape[:2])).astype(np.float32)
    CB = (0.3 * rng.standard_normal(B.shape[:2])).astype(np.float32)
    out = dict(A=A, B=B, N=Nr, M=Mr, q=q, t=t, CA=CA, CB=CB)
    V, dQ, dT = rk.overlap_score_grad_se3_batch(T(A), T(B), T(q), T(t), alpha=0.81,
                                                N_real=T(Nr), M_real=T(Mr))
    out.update(shape_V=V.numpy(), shape_dQ=dQ.numpy(), shape_dT=dT.numpy())
    for tag, lam in (("esp_surf", 0.3 * LAM_SCALING), ("esp_raw", 0.3)):
        V, dQ, dT = rk.overlap_score_grad_esp_se3_batch(
            T(A), T(B), T(CA), T(CB), T(q), T(t), alpha=0.81, lam=lam, N_real=T(Nr), M_real=T(Mr))
        out.update({f"{tag}_lam": np.float64(lam), f"{tag}_V": V.numpy(),
                    f"{tag}_dQ": dQ.numpy(), f"{tag}_dT": dT.numpy()})
    out["self_shape_A"] = rk._batch_self_overlap(T(A), T(Nr), 0.81).numpy()
    out["self_esp_A"] = rk._batch_self_overlap_esp(T(A), T(CA), T(Nr), 0.81, 0.3).numpy()

    # pharmacophore kernels (directional + directionless colour)
    psz = [(1, 1), (3, 4), (7, 5), (12, 20), (20, 12), (20, 20)]
    PA_l, PB_l, PRV_l, PFV_l, PAt_l, PBt_l = [], [], [], [], [], []
    for na, nb in psz:
        fr = syn.pharm_features(rng, [refs[-1]], [na])[0]
        ff = syn.pharm_features(rng, [fits[-1]], [nb])[0]
        PAt_l.append(fr[0]); PA_l.append(fr[1]); PRV_l.append(fr[2])
        PBt_l.append(ff[0]); PB_l.append(ff[1]); PFV_l.append(ff[2])
    PA, PN = pad(PA_l); PB, PM = pad(PB_l)
    PRV, _ = pad(PRV_l); PFV, _ = pad(PFV_l)
    PAt, _ = pad(PAt_l, fill=8, dtype=np.int64); PBt, _ = pad(PBt_l, fill=8, dtype=np.int64)
    Kp = len(psz)
    pq = rand_quat(rng, Kp)
    pt = (0.5 * rng.standard_normal((Kp, 3))).astype(np.float32)
    out.update(PA=PA, PB=PB, PRV=PRV, PFV=PFV, PAt=PAt, PBt=PBt, PN=PN, PM=PM, pq=pq, pt=pt)
    al, ks, cats = build_lookup_tables(torch.device("cpu"), torch.float32)
    O, dQ, dT = rk.pharm_grad_dq_se3_batch(T(pq), T(pt), T(PAt), T(PBt), T(PA), T(PB), T(PRV),
                                           T(PFV), al, ks, cats, N_real=T(PN), M_real=T(PM))
    out.update(pharm_O=O.numpy(), pharm_dQ=dQ.numpy(), pharm_dT=dT.numpy())
    al0, ks0, cats0 = build_lookup_tables(torch.device("cpu"), torch.float32, directionless=True)
    O, dQ, dT = rk.pharm_color_score_grad_se3_batch(T(PA), T(PB), T(pq), T(pt), T(PAt), T(PBt),
                                                    al0, ks0, cats0, N_real=T(PN), M_real=T(PM))
    out.update(color_O=O.numpy(), color_dQ=dQ.numpy(), color_dT=dT.numpy())
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **out)
    print("kernels.npz", {k: v.shape for k, v in out.items()})

    # ---------------- seeds ----------------------------------------------------------
    out = {}
    srefs = syn.ball_clouds(rng, [20, 2, 35, 9, 50, 1])
    sfits = syn.ball_clouds(rng, [25, 18, 3, 40, 12, 30])
    SA, SN = pad(srefs); SB, SM = pad(sfits)
    out.update(A=SA, B=SB, N=SN, M=SM)
    for ns in (1, 3, 8, 10, 16, 32, 50):
        qq, tt = batched_seeds_torch(T(SA), T(SB), T(SN), T(SM), num_seeds=ns)
        out[f"q_{ns}"] = qq.numpy(); out[f"t_{ns}"] = tt.numpy()
    np.savez_compressed(os.path.join(HERE, "seeds.npz"), **out)
    print("seeds.npz")

    # ---------------- batched alignment drivers (numba CPU path, early stop off) --------
    ES = 10 ** 9
    out = {}
    arefs, afits = syn.shape_pairs(6, seed=11)
    # two self-copies (rotated + shifted): the optimum is a Tanimoto of 1
    for i in (0, 1):
        afits[i], _ = rotated_copy(rng, arefs[i])
    AA, AN = pad(arefs); AB, AM = pad(afits)
    VAA = rk._batch_self_overlap(T(AA), T(AN), 0.81)
    VBB = rk._batch_self_overlap(T(AB), T(AM), 0.81)
    qs, ts = batched_seeds_torch(T(AA), T(AB), T(AN), T(AM), num_seeds=20)
    sc, bq, bt = coarse_fine_align_many(T(AA), T(AB), VAA, VBB, alpha=0.81, num_seeds=20,
                                        steps_fine=80, lr=0.1, N_real=T(AN), M_real=T(AM),
                                        early_stop_patience=ES, seeds=(qs, ts))
    out.update(shape_A=AA, shape_B=AB, shape_N=AN, shape_M=AM, shape_seeds_q=qs.numpy(),
               shape_seeds_t=ts.numpy(), shape_score=sc.numpy(), shape_q=bq.numpy(),
               shape_t=bt.numpy())

    erefs, efits = syn.esp_surface_pairs(4, seed=12, lo=40, hi=90)
    efits[0] = (rotated_copy(rng, erefs[0][0])[0], erefs[0][1].copy())
    EA, EN = pad([p for p, _ in erefs]); EB, EM = pad([p for p, _ in efits])
    ECA, _ = pad([c for _, c in erefs]); ECB, _ = pad([c for _, c in efits])
    lam_s = 0.3 * LAM_SCALING
    VAA = rk._batch_self_overlap_esp(T(EA), T(ECA), T(EN), 0.81, lam_s)
    VBB = rk._batch_self_overlap_esp(T(EB), T(ECB), T(EM), 0.81, lam_s)
    sc, bq, bt = coarse_fine_esp_align_many(
        T(EA), T(EB), T(ECA), T(ECB), VAA, VBB, alpha=0.81, lam=lam_s, num_seeds=10,
        steps_fine=60, lr=0.1, N_real=T(EN), M_real=T(EM), early_stop_patience=ES)
    qs, ts = batched_seeds_torch(T(EA), T(EB), T(EN), T(EM), num_seeds=10)
    out.update(esp_A=EA, esp_B=EB, esp_CA=ECA, esp_CB=ECB, esp_N=EN, esp_M=EM,
               esp_lam=np.float64(lam_s), esp_seeds_q=qs.numpy(), esp_seeds_t=ts.numpy(),
               esp_score=sc.numpy(), esp_q=bq.numpy(), esp_t=bt.numpy())

    prefs, pfits = syn.shape_pharm_pairs(5, seed=13)
    pfits[0] = dict(prefs[0])
    Rr = syn.random_rotation(rng)
    sh = rng.standard_normal(3)
    pfits[0]["pharm_ancs"] = (prefs[0]["pharm_ancs"] @ Rr.T + sh).astype(np.float32)
    pfits[0]["pharm_vecs"] = (prefs[0]["pharm_vecs"] @ Rr.T).astype(np.float32)
    pfits[0]["atom_pos"] = (prefs[0]["atom_pos"] @ Rr.T + sh).astype(np.float32)
    PA, PN = pad([m["pharm_ancs"] for m in prefs]); PB, PM = pad([m["pharm_ancs"] for m in pfits])
    PRV, _ = pad([m["pharm_vecs"] for m in prefs]); PFV, _ = pad([m["pharm_vecs"] for m in pfits])
    PAt, _ = pad([m["pharm_types"] for m in prefs], fill=0, dtype=np.int64)
    PBt, _ = pad([m["pharm_types"] for m in pfits], fill=0, dtype=np.int64)
    dummyV = torch.zeros(len(prefs))
    sc, bq, bt = coarse_fine_pharm_align_many(
        T(PA), T(PB), T(PRV), T(PFV), T(PAt), T(PBt), dummyV, dummyV, num_seeds=16,
        steps_fine=60, lr=0.1, N_real=T(PN), M_real=T(PM), early_stop_patience=ES)
    out.update(pharm_A=PA, pharm_B=PB, pharm_RV=PRV, pharm_FV=PFV, pharm_At=PAt, pharm_Bt=PBt,
               pharm_N=PN, pharm_M=PM, pharm_score=sc.numpy(), pharm_q=bq.numpy(),
               pharm_t=bt.numpy())

    CA_, CN = pad([m["atom_pos"] for m in prefs]); CB_, CM = pad([m["atom_pos"] for m in pfits])
    PAt8, _ = pad([m["pharm_types"] for m in prefs], fill=8, dtype=np.int64)
    PBt8, _ = pad([m["pharm_types"] for m in pfits], fill=8, dtype=np.int64)
    VAA = rk._batch_self_overlap(T(CA_), T(CN), 0.81)
    VBB = rk._batch_self_overlap(T(CB_), T(CM), 0.81)
    sc, bq, bt = coarse_fine_vol_color_align_many(
        T(CA_), T(CB_), T(PAt8), T(PBt8), T(PA), T(PB), VAA, VBB, alpha=0.81, color_weight=0.5,
        num_seeds=16, steps_fine=60, lr=0.1, N_real_centers=T(CN), M_real_centers=T(CM),
        N_real_pharm=T(PN), M_real_pharm=T(PM), early_stop_patience=ES)
    out.update(color_A=CA_, color_B=CB_, color_N=CN, color_M=CM, color_At=PAt8, color_Bt=PBt8,
               color_score=sc.numpy(), color_q=bq.numpy(), color_t=bt.numpy())
    np.savez_compressed(os.path.join(HERE, "align.npz"), **out)
    print("align.npz")

    # ---------------- fp64 torch scoring + autograd coordinate/charge gradients --------
    out = {}
    cref = syn.ball_clouds(rng, [24])[0].astype(np.float64)
    cfit = syn.ball_clouds(rng, [19])[0].astype(np.float64)
    sref, sfit = syn.sphere_clouds(rng, [60, 70])
    out.update(c_ref=cref, c_fit=cfit, s_ref=sref[0].astype(np.float64),
               s_fit=sfit[0].astype(np.float64), q_ref=sref[1].astype(np.float64),
               q_fit=sfit[1].astype(np.float64))
    x1 = torch.tensor(cref, requires_grad=True); x2 = torch.tensor(cfit, requires_grad=True)
    s = get_overlap(x1, x2, alpha=0.81)
    s.backward()
    out.update(vol_score=s.detach().numpy(), vol_grad_ref=x1.grad.numpy(),
               vol_grad_fit=x2.grad.numpy())
    for tag, lam in (("esp_surf", 0.3 * LAM_SCALING), ("esp_raw", 0.3)):
        p1 = torch.tensor(out["s_ref"], requires_grad=True)
        p2 = torch.tensor(out["s_fit"], requires_grad=True)
        c1 = torch.tensor(out["q_ref"], requires_grad=True)
        c2 = torch.tensor(out["q_fit"], requires_grad=True)
        s = get_overlap_esp(p1, p2, c1, c2, alpha=1.216, lam=lam)
        s.backward()
        out.update({f"{tag}_lam": np.float64(lam), f"{tag}_score": s.detach().numpy(),
                    f"{tag}_grad_ref": p1.grad.numpy(), f"{tag}_grad_fit": p2.grad.numpy(),
                    f"{tag}_gradq_ref": c1.grad.numpy(), f"{tag}_gradq_fit": c2.grad.numpy()})
    pr = syn.pharm_features(rng, [cref.astype(np.float32)], [9])[0]
    pf = syn.pharm_features(rng, [cfit.astype(np.float32)], [11])[0]
    out.update(pt_ref=pr[0], pa_ref=pr[1].astype(np.float64), pv_ref=pr[2].astype(np.float64),
               pt_fit=pf[0], pa_fit=pf[1].astype(np.float64), pv_fit=pf[2].astype(np.float64))
    for dl in (False, True):
        s = get_overlap_pharm(torch.tensor(pr[0]), torch.tensor(pf[0]), torch.tensor(out["pa_ref"]),
                              torch.tensor(out["pa_fit"]), torch.tensor(out["pv_ref"]),
                              torch.tensor(out["pv_fit"]), directionless=dl)
        out[f"pharm_score_dl{int(dl)}"] = s.detach().numpy()
        s = get_pharm_combo_score(torch.tensor(cref), torch.tensor(cfit), torch.tensor(pr[0]),
                                  torch.tensor(pf[0]), torch.tensor(out["pa_ref"]),
                                  torch.tensor(out["pa_fit"]), torch.tensor(out["pv_ref"]),
                                  torch.tensor(out["pv_fit"]), alpha=0.81, color_weight=0.5,
                                  directionless=dl)
        out[f"combo_score_dl{int(dl)}"] = s.detach().numpy()
    np.savez_compressed(os.path.join(HERE, "scores.npz"), **out)
    print("scores.npz")
    make_pharm_ext()
    make_esp_combo()
    make_trans_init()


def make_pharm_ext():
    """pharm_ext.npz: extended-point pharmacophore overlaps/gradients (autograd through
    batch_pharm_cross_overlap_with_transform, extended_points / only_extended), extended self overlaps
    (batch_pharm_self_overlap) and Tversky / extended-point alignments
    (coarse_fine_pharm_align_many) from the reference, on their own seeded inputs."""
    import torch
    from shepherd_score.accel.drivers.pharm import coarse_fine_pharm_align_many
    from shepherd_score.accel.drivers.pharm_overlap import (
        batch_pharm_cross_overlap_with_transform, batch_pharm_self_overlap)

    T = lambda a: torch.as_tensor(np.ascontiguousarray(a))
    rng = np.random.default_rng(2024)
    out = {}
    # single poses on unpadded molecules (8 features each): value, dO/dt, dO/dq
    refs, fits = syn.shape_pharm_pairs(6, seed=21, ph_lo=8, ph_hi=8)
    A = np.stack([m["pharm_ancs"] for m in refs]).astype(np.float64)
    B = np.stack([m["pharm_ancs"] for m in fits]).astype(np.float64)
    RV = np.stack([m["pharm_vecs"] for m in refs]).astype(np.float64)
    FV = np.stack([m["pharm_vecs"] for m in fits]).astype(np.float64)
    At = np.stack([m["pharm_types"] for m in refs]).astype(np.int64)
    Bt = np.stack([m["pharm_types"] for m in fits]).astype(np.int64)
    B[0], FV[0], Bt[0] = A[0] + 0.3, RV[0], At[0]          # a near-copy: many same-type pairs
    q = rand_quat(rng, 6).astype(np.float32).astype(np.float64)
    t = (0.5 * rng.standard_normal((6, 3))).astype(np.float32).astype(np.float64)
    # fp32-representable inputs, evaluated in fp64 (the oracle reads fp32 arrays)
    A, B, RV, FV = (x.astype(np.float32).astype(np.float64) for x in (A, B, RV, FV))
    out.update(sp_A=A, sp_B=B, sp_RV=RV, sp_FV=FV, sp_At=At, sp_Bt=Bt, sp_q=q, sp_t=t)
    for ext, only in ((1, False), (2, True)):
        # the typed path the batched fine loop differentiates on ragged buckets
        # (pharm.py:449-465): acceptor/donor get extended points, halogen keeps its cosine weight
        qv = T(q).clone().requires_grad_(True)
        tv = T(t).clone().requires_grad_(True)
        O = batch_pharm_cross_overlap_with_transform(T(A), T(B), T(RV), T(FV), T(At), T(Bt), qv,
                                                     tv, extended_points=True, only_extended=only)
        dQ, dT = torch.autograd.grad(O.sum(), (qv, tv))
        out[f"sp{ext}_O"] = O.detach().numpy()
        out[f"sp{ext}_dT"] = dT.numpy()
        out[f"sp{ext}_dQ"] = dQ.numpy()     # tangent to the unit sphere (q is normalised inside)

    # alignments: 5 ragged pairs, pair 0 a rotated copy
    prefs, pfits = syn.shape_pharm_pairs(5, seed=23)
    pfits[0] = dict(prefs[0])
    Rr = syn.random_rotation(rng)
    sh = rng.standard_normal(3)
    pfits[0]["pharm_ancs"] = (prefs[0]["pharm_ancs"] @ Rr.T + sh).astype(np.float32)
    pfits[0]["pharm_vecs"] = (prefs[0]["pharm_vecs"] @ Rr.T).astype(np.float32)
    PA, PN = pad([m["pharm_ancs"] for m in prefs]); PB, PM = pad([m["pharm_ancs"] for m in pfits])
    PRV, _ = pad([m["pharm_vecs"] for m in prefs]); PFV, _ = pad([m["pharm_vecs"] for m in pfits])
    PAt, _ = pad([m["pharm_types"] for m in prefs], fill=0, dtype=np.int64)
    PBt, _ = pad([m["pharm_types"] for m in pfits], fill=0, dtype=np.int64)
    out.update(al_A=PA, al_B=PB, al_RV=PRV, al_FV=PFV, al_At=PAt, al_Bt=PBt, al_N=PN, al_M=PM)
    for tag, sim, ext, only in (("tv", "tversky", False, False),
                                ("tvfit", "tversky_fit", False, False),
                                ("ext", "tanimoto", True, False),
                                ("onlyref", "tversky_ref", True, True)):
        VAA = batch_pharm_self_overlap(T(PA), T(PRV), T(PAt), extended_points=ext,
                                       only_extended=only, N_real=T(PN))
        VBB = batch_pharm_self_overlap(T(PB), T(PFV), T(PBt), extended_points=ext,
                                       only_extended=only, N_real=T(PM))
        sc, bq, bt = coarse_fine_pharm_align_many(
            T(PA), T(PB), T(PRV), T(PFV), T(PAt), T(PBt), VAA, VBB, similarity=sim,
            extended_points=ext, only_extended=only, num_seeds=16, steps_fine=40, lr=0.1,
            N_real=T(PN), M_real=T(PM), early_stop_patience=10 ** 9)
        out.update({f"{tag}_VAA": VAA.numpy(), f"{tag}_VBB": VBB.numpy(),
                    f"{tag}_score": sc.numpy(), f"{tag}_q": bq.numpy(), f"{tag}_t": bt.numpy()})
    np.savez_compressed(os.path.join(HERE, "pharm_ext.npz"), **out)
    print("pharm_ext.npz")



def make_esp_combo():
    """esp_combo.npz: the ShaEP ESP comparison (esp_comparison_batch, numba twin) on ragged
    rows, and vol_and_surf_esp alignments (coarse_fine_esp_combo_align_many, CPU eager loop:
    combo score tracked every 5th step and on the last) on their own seeded molecules."""
    import torch
    from shepherd_score.accel.kernels import cpu as rk
    from shepherd_score.accel.drivers.esp_combo import (coarse_fine_esp_combo_align_many,
                                                        _self_overlap_chunks)

    T = lambda a: torch.as_tensor(np.ascontiguousarray(a))
    rng = np.random.default_rng(77)
    out = {}
    refs, fits = syn.esp_combo_pairs(5, seed=31)
    # comparison rows: ref surface + ESP against the fit atoms moved onto the ref centre
    moved = []
    for r, f in zip(refs, fits):
        Rr = syn.random_rotation(rng)
        a = (f["atoms"] - f["atoms"].mean(0)) @ Rr.T + r["atoms"].mean(0) + 0.5 * rng.standard_normal(3)
        moved.append(a.astype(np.float32))
    P, PN = pad([r["surf"] for r in refs])
    PE, _ = pad([r["surf_esp"] for r in refs])
    A, AM = pad(moved)
    Q, _ = pad([f["charges"] for f in fits])
    R, _ = pad([f["radii"] for f in fits])
    S = rk.esp_comparison_batch(T(P), T(A), T(Q), T(PE), T(R), N_real=T(PN), M_real=T(AM),
                                probe_radius=1.0, lam=0.001)
    out.update(cmp_P=P, cmp_PE=PE, cmp_A=A, cmp_Q=Q, cmp_R=R, cmp_N=PN, cmp_M=AM,
               cmp_S=S.numpy())

    # alignments: pair 0 is a rotated, shifted copy of its reference
    refs, fits = syn.esp_combo_pairs(4, seed=32)
    Rr = syn.random_rotation(rng)
    sh = rng.standard_normal(3)
    f0 = dict(refs[0])
    for k in ("centers", "atoms", "surf"):
        f0[k] = (refs[0][k] @ Rr.T + sh).astype(np.float32)
    fits[0] = f0
    arr = {}
    for side, mols in (("1", refs), ("2", fits)):
        arr["C" + side], arr["CN" + side] = pad([m["centers"] for m in mols])
        arr["A" + side], arr["AN" + side] = pad([m["atoms"] for m in mols])
        arr["Q" + side], _ = pad([m["charges"] for m in mols])
        arr["R" + side], _ = pad([m["radii"] for m in mols])
        arr["S" + side], arr["SN" + side] = pad([m["surf"] for m in mols])
        arr["PE" + side], _ = pad([m["surf_esp"] for m in mols])
    VAA = _self_overlap_chunks(T(arr["C1"]), T(arr["CN1"]), 0.81)
    VBB = _self_overlap_chunks(T(arr["C2"]), T(arr["CN2"]), 0.81)
    sc, bq, bt = coarse_fine_esp_combo_align_many(
        T(arr["A1"]), T(arr["A2"]), T(arr["C1"]), T(arr["C2"]), T(arr["S1"]), T(arr["S2"]),
        T(arr["Q1"]), T(arr["Q2"]), T(arr["PE1"]), T(arr["PE2"]), T(arr["R1"]), T(arr["R2"]),
        VAA, VBB, alpha=0.81, lam=0.001, probe_radius=1.0, esp_weight=0.5, num_seeds=8,
        steps_fine=30, lr=0.1, N_real_centers=T(arr["CN1"]), M_real_centers=T(arr["CN2"]),
        N_real_atoms_w_H_1=T(arr["AN1"]), M_real_atoms_w_H_2=T(arr["AN2"]),
        N_real_surf_1=T(arr["SN1"]), M_real_surf_2=T(arr["SN2"]), early_stop_patience=10 ** 9)
    out.update({"al_" + k: v for k, v in arr.items()})
    out.update(al_score=sc.numpy(), al_q=bq.numpy(), al_t=bt.numpy())
    np.savez_compressed(os.path.join(HERE, "esp_combo.npz"), **out)
    print("esp_combo.npz")


def make_trans_init():
    """trans_init.npz: the legacy translation-seeded path (trans_init=True).  Per pair, the
    reference's start grid (legacy_seeds_with_translations_torch: identity, 4 principal-axis
    poses, 10 Fibonacci rotations per translation centre) and the coarse-grid + top-k + fine
    alignment of the surf_esp, pharm, vol_color and vol_and_surf_esp drivers (one pair per call,
    CPU path, early stop off), on their own seeded molecules; plus the 45-rotation table the
    legacy path uses for num_repeats_per_trans=45."""
    import torch
    from shepherd_score.accel.kernels import cpu as rk
    from shepherd_score.accel.drivers._common import legacy_seeds_with_translations_torch
    from shepherd_score.accel.drivers.esp import coarse_fine_esp_align_many
    from shepherd_score.accel.drivers.pharm import coarse_fine_pharm_align_many
    from shepherd_score.accel.drivers.pharm_overlap import batch_pharm_self_overlap
    from shepherd_score.accel.drivers.vol_color import coarse_fine_vol_color_align_many
    from shepherd_score.accel.drivers.esp_combo import (coarse_fine_esp_combo_align_many,
                                                        _self_overlap_chunks)
    from shepherd_score.alignment._torch import _get_45_fibo
    from shepherd_score.score.constants import LAM_SCALING

    T = lambda a: torch.as_tensor(np.ascontiguousarray(a))
    ES = 10 ** 9
    rng = np.random.default_rng(91)
    out = {"fibo45": _get_45_fibo().numpy()}
    kw = dict(num_repeats_per_trans=10, topk=30, steps_fine=30, lr=0.1, early_stop_patience=ES)

    def collect(tag, results):
        out[f"{tag}_score"] = np.array([r[0] for r in results], np.float32)
        out[f"{tag}_q"] = np.stack([r[1] for r in results]).astype(np.float32)
        out[f"{tag}_t"] = np.stack([r[2] for r in results]).astype(np.float32)

    # surf_esp: grid from the surfaces, translation centres = a few interior points
    refs, fits = syn.esp_surface_pairs(4, seed=41, lo=40, hi=90)
    fits[0] = (rotated_copy(rng, refs[0][0])[0], refs[0][1].copy())
    ctr = [(0.5 * p[rng.choice(len(p), n, replace=False)]).astype(np.float32)
           for (p, _), n in zip(refs, (5, 7, 6, 5))]
    lam_s = 0.3 * LAM_SCALING
    grids, res = [], []
    for (pa, ca), (pb, cb), c in zip(refs, fits, ctr):
        q, t = legacy_seeds_with_translations_torch(T(pa), T(pb), T(c), num_repeats_per_trans=10)
        grids.append((q.detach().numpy(), t.detach().numpy()))
        VAA = rk._batch_self_overlap_esp(T(pa[None]), T(ca[None]), T([len(pa)]), 0.81, lam_s)
        VBB = rk._batch_self_overlap_esp(T(pb[None]), T(cb[None]), T([len(pb)]), 0.81, lam_s)
        sc, bq, bt = coarse_fine_esp_align_many(
            T(pa[None]), T(pb[None]), T(ca[None]), T(cb[None]), VAA, VBB, alpha=0.81,
            lam=lam_s, trans_centers=T(c[None]), **kw)
        res.append((float(sc[0]), bq[0].detach().numpy(), bt[0].detach().numpy()))
    EA, EN = pad([p for p, _ in refs]); EB, EM = pad([p for p, _ in fits])
    ECA, _ = pad([c for _, c in refs]); ECB, _ = pad([c for _, c in fits])
    TC, TN = pad(ctr)
    GQ, GN = pad([g[0] for g in grids]); GT, _ = pad([g[1] for g in grids])
    out.update(esp_A=EA, esp_B=EB, esp_CA=ECA, esp_CB=ECB, esp_N=EN, esp_M=EM,
               esp_lam=np.float64(lam_s), esp_TC=TC, esp_TN=TN, esp_GQ=GQ, esp_GT=GT,
               esp_G=GN)
    collect("esp", res)
    q45, t45 = legacy_seeds_with_translations_torch(T(refs[1][0]), T(fits[1][0]), T(ctr[1][:2]),
                                                    num_repeats_per_trans=45)
    out.update(g45_q=q45.detach().numpy(), g45_t=t45.detach().numpy())

    def grid_of(a, b, c):
        q, t = legacy_seeds_with_translations_torch(T(a), T(b), T(c), num_repeats_per_trans=10)
        return q.detach().numpy(), t.detach().numpy()

    def store_grids(tag, grids):
        GQ, GN = pad([g[0] for g in grids]); GT, _ = pad([g[1] for g in grids])
        out.update({f"{tag}_GQ": GQ, f"{tag}_GT": GT, f"{tag}_G": GN})

    # pharm (Tanimoto, directional): translation centres = the reference anchors; the driver
    # builds the grid on per-cloud centred anchors with the centres shifted alike
    prefs, pfits = syn.shape_pharm_pairs(4, seed=42, ph_lo=4, ph_hi=9, atom_hi=30)
    res, grids = [], []
    for r, f in zip(prefs, pfits):
        ca = T(r["pharm_ancs"]).sum(0) / float(len(r["pharm_ancs"]))
        cb = T(f["pharm_ancs"]).sum(0) / float(len(f["pharm_ancs"]))
        grids.append(grid_of((T(r["pharm_ancs"]) - ca).numpy(), (T(f["pharm_ancs"]) - cb).numpy(),
                             (T(r["pharm_ancs"]) - ca).numpy()))
        # self overlaps as the public driver computes them (pharm.py:735-751): the coarse
        # grid ranks poses by the similarity built from them
        tr, tf = T(r["pharm_types"][None].astype(np.int64)), T(f["pharm_types"][None].astype(np.int64))
        VAA = batch_pharm_self_overlap(T(r["pharm_ancs"][None]), T(r["pharm_vecs"][None]), tr,
                                       extended_points=False, only_extended=False,
                                       N_real=T([len(r["pharm_ancs"])]))
        VBB = batch_pharm_self_overlap(T(f["pharm_ancs"][None]), T(f["pharm_vecs"][None]), tf,
                                       extended_points=False, only_extended=False,
                                       N_real=T([len(f["pharm_ancs"])]))
        sc, bq, bt = coarse_fine_pharm_align_many(
            T(r["pharm_ancs"][None]), T(f["pharm_ancs"][None]), T(r["pharm_vecs"][None]),
            T(f["pharm_vecs"][None]), tr, tf, VAA, VBB,
            trans_centers=T(r["pharm_ancs"][None]), **kw)
        res.append((float(sc[0]), bq[0].detach().numpy(), bt[0].detach().numpy()))
    PA, PN = pad([m["pharm_ancs"] for m in prefs]); PB, PM = pad([m["pharm_ancs"] for m in pfits])
    PRV, _ = pad([m["pharm_vecs"] for m in prefs]); PFV, _ = pad([m["pharm_vecs"] for m in pfits])
    PAt, _ = pad([m["pharm_types"] for m in prefs], fill=0, dtype=np.int64)
    PBt, _ = pad([m["pharm_types"] for m in pfits], fill=0, dtype=np.int64)
    out.update(pharm_A=PA, pharm_B=PB, pharm_RV=PRV, pharm_FV=PFV, pharm_At=PAt, pharm_Bt=PBt,
               pharm_N=PN, pharm_M=PM)
    collect("pharm", res)
    store_grids("pharm", grids)

    # vol_color: grid from the atom centres, translation centres = the reference atoms
    res, grids = [], []
    for r, f in zip(prefs, pfits):
        grids.append(grid_of(r["atom_pos"], f["atom_pos"], r["atom_pos"]))
        VAA = rk._batch_self_overlap(T(r["atom_pos"][None]), T([len(r["atom_pos"])]), 0.81)
        VBB = rk._batch_self_overlap(T(f["atom_pos"][None]), T([len(f["atom_pos"])]), 0.81)
        sc, bq, bt = coarse_fine_vol_color_align_many(
            T(r["atom_pos"][None]), T(f["atom_pos"][None]),
            T(r["pharm_types"][None].astype(np.int64)), T(f["pharm_types"][None].astype(np.int64)),
            T(r["pharm_ancs"][None]), T(f["pharm_ancs"][None]), VAA, VBB, alpha=0.81,
            color_weight=0.5, trans_centers=T(r["atom_pos"][None]), **kw)
        res.append((float(sc[0]), bq[0].detach().numpy(), bt[0].detach().numpy()))
    CA_, CN = pad([m["atom_pos"] for m in prefs]); CB_, CM = pad([m["atom_pos"] for m in pfits])
    PAt8, _ = pad([m["pharm_types"] for m in prefs], fill=8, dtype=np.int64)
    PBt8, _ = pad([m["pharm_types"] for m in pfits], fill=8, dtype=np.int64)
    out.update(color_A=CA_, color_B=CB_, color_N=CN, color_M=CM, color_At=PAt8, color_Bt=PBt8)
    collect("color", res)
    store_grids("color", grids)

    # vol_and_surf_esp: grid from the surfaces, translation centres = the reference centres
    refs, fits = syn.esp_combo_pairs(3, seed=43, surf_lo=50, surf_hi=80)
    res, grids = [], []
    for r, f in zip(refs, fits):
        grids.append(grid_of(r["surf"], f["surf"], r["centers"]))
        one = lambda m, k: T(m[k][None])
        cnt = lambda m, k: T([len(m[k])])
        VAA = _self_overlap_chunks(one(r, "centers"), cnt(r, "centers"), 0.81)
        VBB = _self_overlap_chunks(one(f, "centers"), cnt(f, "centers"), 0.81)
        sc, bq, bt = coarse_fine_esp_combo_align_many(
            one(r, "atoms"), one(f, "atoms"), one(r, "centers"), one(f, "centers"),
            one(r, "surf"), one(f, "surf"), one(r, "charges"), one(f, "charges"),
            one(r, "surf_esp"), one(f, "surf_esp"), one(r, "radii"), one(f, "radii"), VAA, VBB,
            alpha=0.81, lam=0.001, probe_radius=1.0, esp_weight=0.5,
            trans_centers=one(r, "centers"), **kw)
        res.append((float(sc[0]), bq[0].detach().numpy(), bt[0].detach().numpy()))
    arr = {}
    for side, mols in (("1", refs), ("2", fits)):
        arr["C" + side], arr["CN" + side] = pad([m["centers"] for m in mols])
        arr["A" + side], arr["AN" + side] = pad([m["atoms"] for m in mols])
        arr["Q" + side], _ = pad([m["charges"] for m in mols])
        arr["R" + side], _ = pad([m["radii"] for m in mols])
        arr["S" + side], arr["SN" + side] = pad([m["surf"] for m in mols])
        arr["PE" + side], _ = pad([m["surf_esp"] for m in mols])
    out.update({"combo_" + k: v for k, v in arr.items()})
    collect("combo", res)
    store_grids("combo", grids)
    np.savez_compressed(os.path.join(HERE, "trans_init.npz"), **out)
    print("trans_init.npz")


if __name__ == "__main__":
    main()
