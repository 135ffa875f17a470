"""Results do not depend on the CTA size or on which starts share a warp: the staged frame's
centroid is a fixed-order sum and the factored/plain exponent guard is voted by each pose's
own lanes, so start blocks of 2, 3, 4, 8 or 10 poses (16-lane poses: 1 to 5 warps, with an
idle half-warp in the odd blocks) give bit-identical start rows."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.layout import CloudSet
from test_gpu_align import assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [4, 5])
@pytest.mark.parametrize("mode", ["esp", "shape"])
def test_rows_independent_of_cta_size(cuda, mode, variant):
    refs, fits = syn.esp_surface_pairs(16, seed=41, lo=80, hi=160)
    ref = CloudSet.from_arrays([p for p, _ in refs], [c for _, c in refs], device=cuda)
    fit = CloudSet.from_arrays([p for p, _ in fits], [c for _, c in fits], device=cuda)
    idx = torch.arange(16, dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 50)
    # every third start begins 11 A off, so its first steps take the unfactored exponent
    # while its warp-mates stay factored
    st[:, ::3] += torch.tensor([11.0, 0.0, 0.0], device=cuda)
    kw = dict(ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, steps=30,
              lr=0.1, lam=0.3 * al.LAM_SCALING if mode == "esp" else None, lanes_per_pose=16,
              kernel_variant=variant)
    rows = [tuple(x.cpu().numpy() for x in al.align_packed(mode, chunks=c, **kw).rows)
            for c in (25, 17, 13, 7, 5)]
    for other in rows[1:]:
        for a, b in zip(rows[0], other):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("mode", ["shape", "esp", "shape_pharm", "pharm"])
def test_one_and_two_lanes_per_pose(cuda, mode):
    """Poses on 1 or 2 lanes (no lane reduction) agree with 4-lane poses: step-1 rows (the
    seeds' own scores) to fp32 rounding, then best scores within the alignment tolerance."""
    from fast_shepherd_score_b200.layout import PharmSet
    refs, fits = syn.shape_pharm_pairs(10, seed=42)
    g = lambda ms, k: [m[k] for m in ms]
    rng = np.random.default_rng(3)
    ch = lambda ms: [(0.2 * rng.standard_normal(len(m["atom_pos"]))).astype(np.float32)
                     for m in ms]
    esp = mode == "esp"
    ref = CloudSet.from_arrays(g(refs, "atom_pos"), ch(refs) if esp else None, device=cuda)
    fit = CloudSet.from_arrays(g(fits, "atom_pos"), ch(fits) if esp else None, device=cuda)
    ps = lambda ms: PharmSet.from_arrays(g(ms, "pharm_types"), g(ms, "pharm_ancs"),
                                         g(ms, "pharm_vecs"), device=cuda)
    idx = torch.arange(10, dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 20)
    kw = dict(pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, lr=0.1,
              lam=0.3 if esp else None)
    if mode != "pharm":
        kw.update(ref=ref, fit=fit)
    if mode in ("pharm", "shape_pharm"):
        kw.update(ref_ph=ps(refs), fit_ph=ps(fits))
    run = lambda lpp, steps: al.align_packed(mode, steps=steps, lanes_per_pose=lpp, **kw)
    base1 = run(4, 1).rows[0].cpu().numpy()
    base = run(4, 40)[0].cpu().numpy()
    for lpp in (1, 2):
        np.testing.assert_allclose(run(lpp, 1).rows[0].cpu().numpy(), base1, rtol=2e-5,
                                   atol=1e-6)
        sc = run(lpp, 40)[0].cpu().numpy()
        assert_parity(sc, base)


def test_one_and_two_lanes_per_pose_esp_combo(cuda):
    """vol_and_surf_esp with 1 or 2 lanes per pose: step-1 rows (shape Tanimoto + ESP
    comparison of the seed poses) agree with 16-lane poses to fp32 rounding."""
    refs, fits = syn.esp_combo_pairs(6, seed=44)
    g = lambda ms, k: [m[k] for m in ms]
    cs = lambda ms, k, v=None: CloudSet.from_arrays(g(ms, k), g(ms, v) if v else None,
                                                    device=cuda)
    rad = lambda ms: torch.as_tensor(np.concatenate(g(ms, "radii")).astype(np.float32),
                                     device=cuda)
    idx = torch.arange(6, dtype=torch.int32, device=cuda)
    ref, fit = cs(refs, "centers"), cs(fits, "centers")
    sq, st = K.seeds(ref, fit, idx, idx, 8)
    kw = dict(ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, steps=1,
              lr=0.1, lam=0.001, ref_atoms=cs(refs, "atoms", "charges"),
              fit_atoms=cs(fits, "atoms", "charges"), ref_radii=rad(refs), fit_radii=rad(fits),
              ref_surf=cs(refs, "surf", "surf_esp"), fit_surf=cs(fits, "surf", "surf_esp"))
    base = al.align_packed("esp_combo", lanes_per_pose=16, **kw).rows[0].cpu().numpy()
    for lpp in (1, 2):
        got = al.align_packed("esp_combo", lanes_per_pose=lpp, **kw).rows[0].cpu().numpy()
        np.testing.assert_allclose(got, base, rtol=5e-5, atol=1e-6)
