"""Seeded synthetic atom globules (the workloads the benchmarks and parity tests run on).

Atoms are placed by random sequential addition uniformly inside a sphere, rejecting any atom
closer than ``dmin`` to an already placed one; radii are drawn C 1.70 (p=0.62), N 1.55 (0.17),
O 1.52 (0.19), S 1.80 (0.02).

The nominal globule radius R = (3 N v / (4 pi))^(1/3) with v = 12 A^3 per atom asks for a packing
fraction of about 0.77 at dmin = 2.6 A, above the random-sequential-addition jamming limit
(about 0.38), so the addition stalls long before N atoms.  The resolution used throughout is
fixed and explicit: N, dmin and the radii are kept and the radius is grown by ``inflate`` = 1.37
(about 30 A^3 per atom, packing fraction about 0.30); ``achieved_density`` reports the outcome.
"""
from __future__ import annotations

import math

import numpy as np

RADII = np.array([1.70, 1.55, 1.52, 1.80])
PROBS = np.array([0.62, 0.17, 0.19, 0.02])
VOL_PER_ATOM = 12.0
INFLATE = 1.37
DMIN = 2.6


def globule_radius(n: int, inflate: float = INFLATE) -> float:
    return inflate * (3.0 * n * VOL_PER_ATOM / (4.0 * math.pi)) ** (1.0 / 3.0)


def rsa_globule(n: int, seed: int, inflate: float = INFLATE, dmin: float = DMIN,
                max_tries: int | None = None) -> np.ndarray:
    """(n, 4) float64 array x, y, z, r of a seeded random-sequential-addition globule.

    Candidates come from a seeded stream of uniform points in the bounding cube, kept when inside
    the sphere; a candidate is accepted when it is not closer than dmin to any previously accepted
    atom.  Each batch of candidates is checked against the atoms of earlier batches at once
    (k-d tree nearest neighbour) and then resolved sequentially among itself, which is the same
    acceptance rule as adding the candidates one at a time.
    """
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    R = globule_radius(n, inflate)
    pts = np.zeros((n, 3))
    placed = 0
    tries = 0
    max_tries = max_tries or 200 * n + 10000
    tree = None
    tree_n = 0
    while placed < n and tries < max_tries:
        batch = rng.uniform(-R, R, size=(4096, 3))
        batch = batch[(batch * batch).sum(1) <= R * R]
        if tree is None or placed - tree_n > max(2048, tree_n // 4):
            tree = cKDTree(pts[:placed]) if placed else None
            tree_n = placed
        ok = np.ones(len(batch), bool)
        if tree is not None:
            d, _ = tree.query(batch, k=1, distance_upper_bound=dmin)
            ok &= ~(d < dmin)
        # atoms accepted since the tree was built
        if placed > tree_n:
            recent = pts[tree_n:placed]
            cand = np.nonzero(ok)[0]
            if len(cand):
                rt = cKDTree(recent)
                d, _ = rt.query(batch[cand], k=1, distance_upper_bound=dmin)
                ok[cand[d < dmin]] = False
        cand = np.nonzero(ok)[0]
        if len(cand) == 0:
            tries += len(batch)
            continue
        # sequential resolution inside the batch, in stream order
        sub = batch[cand]
        diff = sub[:, None, :] - sub[None, :, :]
        close = (diff * diff).sum(-1) < dmin * dmin
        accepted = []
        last = len(batch)
        for a, ci in enumerate(cand):
            if placed + len(accepted) >= n:
                last = ci
                break
            if not any(close[a, b] for b in accepted):
                accepted.append(a)
        tries += last if placed + len(accepted) >= n else len(batch)
        if accepted:
            acc = sub[accepted]
            pts[placed:placed + len(acc)] = acc
            placed += len(acc)
    if placed < n:
        raise RuntimeError(f"random sequential addition placed only {placed} of {n} atoms")
    radii = RADII[rng.choice(4, size=n, p=PROBS)]
    return np.concatenate([pts, radii[:, None]], axis=1)


def achieved_density(atoms: np.ndarray, inflate: float = INFLATE) -> float:
    """Volume per atom (A^3) of the globule sphere."""
    R = globule_radius(len(atoms), inflate)
    return 4.0 / 3.0 * math.pi * R ** 3 / len(atoms)


def ensemble(n_base: int = 32, n_perturb: int = 16, n_min: int = 500, n_max: int = 8000, sigma: float = 0.3,
             seed: int = 5) -> list[np.ndarray]:
    """Conformer ensemble: n_base globules of uniform size in [n_min, n_max], each perturbed
    n_perturb times by i.i.d. Gaussian coordinate noise of standard deviation sigma."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=n_base)
    out = []
    for b, nb in enumerate(sizes):
        base = rsa_globule(int(nb), seed=1000 + b)
        for _ in range(n_perturb):
            a = base.copy()
            a[:, :3] += rng.normal(0.0, sigma, size=(len(a), 3))
            out.append(a)
    return out


# Workloads of the benchmark configurations.
CONFIGS = {
    "ses_327": dict(n=327, seed=1, probe=1.4, scale=2.0, perfil=70.0, cav_vol=10.0),
    "skin_10k": dict(n=10000, seed=2, scale=3.0, perfil=80.0),
    "ses_100k": dict(n=100000, seed=3, probe=1.4, scale=4.0, perfil=70.0),
    "diff_2k": dict(n=2000, seed=4, probe=1.4, scale=3.0, perfil=80.0),
}
