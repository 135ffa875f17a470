"""Seeded synthetic molecule clouds with the shapes and value distributions of the
benchmark workloads (no public dataset is used; every workload is generated here).

* ``ball_clouds``     -- atoms rejection-sampled uniformly in a 6 A ball, >= 1.2 A apart
* ``sphere_clouds``   -- surface points 5 A * u + N(0, 0.3^2), u uniform on S^2, charges N(0, 0.1^2)
* ``pharm_features``  -- 3-20 pharmacophores per molecule, 8 types uniform, anchors jittered
  N(0, 0.5^2) around random atoms, unit vectors on S^2 for the directional types
  (acceptor, donor, aromatic, halogen) and zero for the rest
* ``shape_pairs`` / ``esp_surface_pairs`` / ``shape_pharm_pairs`` -- the pair batches

All generators are numpy ``default_rng(seed)`` based and vectorised over molecules, so the
same seed gives the same data on every machine.
"""
from __future__ import annotations

import numpy as np

DIRECTIONAL_TYPES = (0, 1, 2, 4)   # Acceptor, Donor, Aromatic, Halogen
N_PHARM_TYPES = 8                   # real types 0..7; 8 is the Dummy padding type


def ball_clouds(rng, counts, radius=6.0, min_dist=1.2, max_tries=200):
    """Uniform points in a ball with a minimum pairwise spacing, one cloud per count.

    Vectorised over molecules: slot s is proposed for every molecule at once and
    re-proposed only where it violates the spacing against slots < s.
    Returns a list of float32 (n_i, 3) arrays.
    """
    counts = np.asarray(counts, np.int64)
    K = len(counts)
    nmax = int(counts.max()) if K else 0
    X = np.zeros((K, nmax, 3), np.float64)
    md2 = min_dist * min_dist

    def propose(n):
        v = rng.standard_normal((n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        r = radius * rng.random(n) ** (1.0 / 3.0)
        return v * r[:, None]

    for s in range(nmax):
        need = np.nonzero(counts > s)[0]
        for _ in range(max_tries):
            if need.size == 0:
                break
            cand = propose(need.size)
            if s == 0:
                X[need, 0] = cand
                need = need[:0]
                break
            d2 = ((X[need, :s] - cand[:, None, :]) ** 2).sum(-1).min(1)
            ok = d2 >= md2
            X[need[ok], s] = cand[ok]
            need = need[~ok]
        if need.size:  # crowded ball: accept the last proposal rather than loop forever
            X[need, s] = propose(need.size)
    return [X[i, :counts[i]].astype(np.float32) for i in range(K)]


def sphere_clouds(rng, counts, radius=5.0, jitter=0.3, charge_sd=0.1):
    """Surface-like clouds: points 5*u + N(0, 0.3^2) and per-point charges N(0, 0.1^2)."""
    out = []
    for n in np.asarray(counts, np.int64):
        u = rng.standard_normal((n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        p = radius * u + jitter * rng.standard_normal((n, 3))
        c = charge_sd * rng.standard_normal(n)
        out.append((p.astype(np.float32), c.astype(np.float32)))
    return out


def pharm_features(rng, atoms, counts, jitter=0.5):
    """Pharmacophores near the atoms of each molecule: (types int64, anchors, vectors)."""
    out = []
    for X, n in zip(atoms, np.asarray(counts, np.int64)):
        types = rng.integers(0, N_PHARM_TYPES, n)
        idx = rng.integers(0, len(X), n)
        anc = X[idx] + jitter * rng.standard_normal((n, 3))
        v = rng.standard_normal((n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        v[~np.isin(types, DIRECTIONAL_TYPES)] = 0.0
        out.append((types.astype(np.int64), anc.astype(np.float32), v.astype(np.float32)))
    return out


def shape_pairs(n_pairs, seed=0, lo=15, hi=50):
    """Atom-cloud pairs (ref, fit) with lo..hi atoms each (6 A ball, 1.2 A spacing)."""
    rng = np.random.default_rng(seed)
    nr = rng.integers(lo, hi + 1, n_pairs)
    nf = rng.integers(lo, hi + 1, n_pairs)
    refs = ball_clouds(rng, nr)
    fits = ball_clouds(rng, nf)
    return refs, fits


def esp_surface_pairs(n_pairs, seed=1, lo=200, hi=400):
    """Surface pairs with charges: lists of (points, charges) for ref and fit."""
    rng = np.random.default_rng(seed)
    nr = rng.integers(lo, hi + 1, n_pairs)
    nf = rng.integers(lo, hi + 1, n_pairs)
    return sphere_clouds(rng, nr), sphere_clouds(rng, nf)


def shape_pharm_molecules(n_mol, rng, atom_lo=15, atom_hi=60, ph_lo=3, ph_hi=20):
    """Molecules of atoms + pharmacophores: list of dicts (atom_pos, pharm_types/ancs/vecs)."""
    na = rng.integers(atom_lo, atom_hi + 1, n_mol)
    npf = rng.integers(ph_lo, ph_hi + 1, n_mol)
    atoms = ball_clouds(rng, na)
    feats = pharm_features(rng, atoms, npf)
    return [dict(atom_pos=a, pharm_types=f[0], pharm_ancs=f[1], pharm_vecs=f[2])
            for a, f in zip(atoms, feats)]


def shape_pharm_pairs(n_pairs, seed=2, **kw):
    """Pairs of shape+pharmacophore molecules (ref list, fit list)."""
    rng = np.random.default_rng(seed)
    return shape_pharm_molecules(n_pairs, rng, **kw), shape_pharm_molecules(n_pairs, rng, **kw)


def random_rotation(rng):
    """Uniform random rotation matrix (float64)."""
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def library_on_device(n_mol, seed=5, device="cuda", atom_lo=15, atom_hi=60, ph_lo=3, ph_hi=20,
                      radius=6.0, min_dist=1.2, max_tries=64):
    """A large shape+pharmacophore library generated directly on the device.

    Same distributions as :func:`shape_pharm_molecules` (atoms uniform in a 6 A ball with
    >= 1.2 A spacing, 3-20 pharmacophores of 8 uniform types near the atoms, unit vectors
    for the directional types), drawn with a seeded ``torch.Generator`` on ``device`` so a
    million molecules take seconds.  Returns (CloudSet atoms, PharmSet pharmacophores).
    """
    import torch
    from .layout import CloudSet, PharmSet, _offsets
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    na = torch.randint(atom_lo, atom_hi + 1, (n_mol,), generator=g, device=dev)
    nmax = int(atom_hi)
    X = torch.zeros(n_mol, nmax, 3, device=dev)

    def propose(k):
        v = torch.randn(k, 3, generator=g, device=dev)
        v = v / v.norm(dim=1, keepdim=True)
        r = radius * torch.rand(k, generator=g, device=dev) ** (1.0 / 3.0)
        return v * r[:, None]

    md2 = min_dist * min_dist
    for s in range(nmax):
        need = torch.nonzero(na > s).flatten()
        for _ in range(max_tries):
            if need.numel() == 0:
                break
            cand = propose(need.numel())
            if s == 0:
                X[need, 0] = cand
                need = need[:0]
                break
            d2 = ((X[need, :s] - cand[:, None, :]) ** 2).sum(-1).min(1).values
            ok = d2 >= md2
            X[need[ok], s] = cand[ok]
            need = need[~ok]
        if need.numel():
            X[need, s] = propose(need.numel())
    mask = torch.arange(nmax, device=dev)[None, :] < na[:, None]
    pts = torch.zeros(int(na.sum()), 4, device=dev)
    pts[:, :3] = X[mask]
    counts = na.cpu().numpy().astype(np.int64)
    atoms = CloudSet(pts, torch.from_numpy(_offsets(counts)).to(dev), counts, int(counts.max()))

    npf = torch.randint(ph_lo, ph_hi + 1, (n_mol,), generator=g, device=dev)
    tot = int(npf.sum())
    mol = torch.repeat_interleave(torch.arange(n_mol, device=dev), npf)
    pick = (torch.rand(tot, generator=g, device=dev) * na[mol]).long().clamp(max=nmax - 1)
    anc_xyz = X[mol, pick] + 0.5 * torch.randn(tot, 3, generator=g, device=dev)
    types = torch.randint(0, N_PHARM_TYPES, (tot,), generator=g, device=dev, dtype=torch.int32)
    v = torch.randn(tot, 3, generator=g, device=dev)
    v = v / v.norm(dim=1, keepdim=True)
    directional = torch.zeros_like(types, dtype=torch.bool)
    for t in DIRECTIONAL_TYPES:
        directional |= types == t
    v = torch.where(directional[:, None], v, torch.zeros_like(v))
    anc = torch.zeros(tot, 4, device=dev)
    anc[:, :3] = anc_xyz
    anc[:, 3] = types.view(torch.float32)
    vec = torch.zeros(tot, 4, device=dev)
    vec[:, :3] = v
    pc = npf.cpu().numpy().astype(np.int64)
    pharm = PharmSet(anc, vec, torch.from_numpy(_offsets(pc)).to(dev), pc, int(pc.max()))
    return atoms, pharm


COULOMB_SCALING = 1e4 / (4 * 55.263 * np.pi)   # eV*A/e^2 (score/constants.py:16)


def esp_combo_molecules(n_mol, rng, heavy_lo=10, heavy_hi=25, surf_lo=100, surf_hi=200,
                        h_per_heavy=0.8, charge_sd=0.2):
    """Molecules for the ShaEP combo mode: heavy-atom shape centres (uniform in a ball, >= 1.2 A
    apart), the same atoms plus hydrogens 1.1 A from random heavy atoms (the "atoms with H"),
    net-neutral partial charges N(0, 0.2^2), van der Waals radii (1.2 A for H, U(1.5, 1.9) for
    heavy atoms), surface points on a sphere 2 A outside the farthest atom, and the
    molecule's own Coulomb potential at those points (COULOMB_SCALING * sum_m q_m / d)."""
    nh = rng.integers(heavy_lo, heavy_hi + 1, n_mol)
    heavy = ball_clouds(rng, nh, radius=4.0)
    out = []
    for X in heavy:
        n_h = int(round(h_per_heavy * len(X)))
        anchor = rng.integers(0, len(X), n_h)
        u = rng.standard_normal((n_h, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        H = X[anchor] + 1.1 * u
        atoms = np.concatenate([X, H]).astype(np.float32)
        q = charge_sd * rng.standard_normal(len(atoms))
        q -= q.mean()
        radii = np.concatenate([rng.uniform(1.5, 1.9, len(X)), np.full(n_h, 1.2)])
        ns = int(rng.integers(surf_lo, surf_hi + 1))
        v = rng.standard_normal((ns, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        c = atoms.mean(0)
        rad = float(np.linalg.norm(atoms - c, axis=1).max()) + 2.0
        surf = (c + rad * v).astype(np.float32)
        d = np.linalg.norm(surf[:, None, :].astype(np.float64) - atoms[None].astype(np.float64),
                           axis=-1)
        esp = COULOMB_SCALING * (q[None, :] / np.maximum(d, 1e-6)).sum(1)
        out.append(dict(centers=X.astype(np.float32), atoms=atoms,
                        charges=q.astype(np.float32), radii=radii.astype(np.float32),
                        surf=surf, surf_esp=esp.astype(np.float32)))
    return out


def esp_combo_pairs(n_pairs, seed=6, **kw):
    """Pairs (ref list, fit list) of :func:`esp_combo_molecules`."""
    rng = np.random.default_rng(seed)
    return esp_combo_molecules(n_pairs, rng, **kw), esp_combo_molecules(n_pairs, rng, **kw)
