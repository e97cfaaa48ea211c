"""Seeded synthetic configurations (numpy / scipy only, no native code).

The reference measures on no public dataset; these generators build the
inputs its documented use implies: periodic Si diamond supercells and
periodic two-species random packings, plus the served request stream.
This module imports nothing from the package's native extension, so the
CPU reference arm of the benchmark can load it by file path and build the
same inputs as the GPU arm without loading this library.

Served stream.  Each request draws its own atom count log-uniformly from
[n_min, n_max] and its own configuration: a cube of side (n / density)^(1/3)
cut at a uniformly random offset out of one of a few large periodic random
packings (random sequential addition at the same density and minimum
distance), made periodic with its own side.  Atoms that the new periodic
boundary brings closer than d_min to another are dropped (a few near the
faces), so a request holds about n atoms.
"""
from __future__ import annotations

import numpy as np

# 8-atom conventional diamond basis (fractional)
DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                    [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])

SF24_G2_ETA = (0.001, 0.005, 0.01, 0.02, 0.04, 0.08, 0.16, 0.32)
SF24_G4_ETA = (0.001, 0.01, 0.03, 0.08)


def sf24_params():
    """The 24-d Behler set: 8 g2 (Rs = 0) + 16 g4 rows ordered (zeta, lambda, eta)."""
    g2 = [[e, 0.0] for e in SF24_G2_ETA]
    g4 = [[z, lam, e] for z in (1.0, 4.0) for lam in (-1.0, 1.0) for e in SF24_G4_ETA]
    params = [v for row in g2 for v in row] + [v for row in g4 for v in row]
    return ["g2", "g4"], [8, 2, 16, 3], params


def diamond_cell(n1, n2, n3, a=5.43, jitter=0.0, strain=0.0, seed=0):
    """Si diamond supercell of n1 x n2 x n3 conventional cells.  strain: each
    cell-matrix entry perturbed by U(-strain, strain) (H = (I + eps) H0)."""
    rng = np.random.default_rng(seed)
    h0 = np.diag([n1 * a, n2 * a, n3 * a]).astype(np.float64)
    eps = rng.uniform(-strain, strain, (3, 3)) if strain else np.zeros((3, 3))
    cell = h0 @ (np.eye(3) + eps).T  # rows are lattice vectors
    grid = np.array([[i, j, k] for i in range(n1) for j in range(n2) for k in range(n3)], dtype=np.float64)
    frac = (grid[:, None, :] + DIAMOND[None, :, :]).reshape(-1, 3) / np.array([n1, n2, n3])
    x = frac @ cell
    if jitter:
        x = x + rng.normal(0.0, jitter, x.shape)
    return np.ascontiguousarray(x), np.ascontiguousarray(cell)


def _drop_close_pairs(pairs, keep):
    """Greedy in index order: drop the later member of each close pair."""
    if pairs.size:
        order = np.argsort(pairs[:, 0], kind="stable")
        for a, b in pairs[order]:
            if keep[a] and keep[b]:
                keep[b] = False
    return keep


def random_packing(n, density=0.05, dmin=2.0, n_species=2, seed=0, max_tries=200):
    """n atoms uniformly in a periodic cube of side (n/density)^(1/3) with a
    minimum pair distance dmin (random sequential addition by rejection).
    Species alternate 0,1,... so the mix is 50/50 for two species."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    side = (n / density) ** (1.0 / 3.0)
    acc = np.zeros((0, 3))
    tries = 0
    while acc.shape[0] < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("random_packing: could not place all atoms")
        m = max(64, int(1.3 * (n - acc.shape[0])))
        cand = rng.uniform(0.0, side, (m, 3))
        if acc.shape[0]:
            tree = cKDTree(acc, boxsize=side)
            d, _ = tree.query(cand, k=1)
            cand = cand[d >= dmin]
        if cand.shape[0] == 0:
            continue
        ct = cKDTree(cand, boxsize=side)
        keep = _drop_close_pairs(ct.query_pairs(dmin, output_type="ndarray"), np.ones(cand.shape[0], dtype=bool))
        cand = cand[keep][: n - acc.shape[0]]
        acc = np.concatenate([acc, cand])
    species = (np.arange(n) % n_species).astype(np.int32)
    return np.ascontiguousarray(acc), np.eye(3) * side, species


class PackingSource:
    """Periodic random packings of any size cut out of a few large ones."""

    def __init__(self, n_base=4, base_atoms=32768, density=0.05, dmin=2.0, seed=0):
        self.density, self.dmin = float(density), float(dmin)
        self.bases = [random_packing(base_atoms, density, dmin, n_species=1, seed=seed * 1000 + 17 + i)[0]
                      for i in range(n_base)]
        self.side = (base_atoms / density) ** (1.0 / 3.0)

    def cut(self, n, rng, n_species=2):
        """About n atoms in a periodic cube of side (n / density)^(1/3):
        coordinates, cell (rows = lattice vectors), species (alternating)."""
        from scipy.spatial import cKDTree

        L = min((n / self.density) ** (1.0 / 3.0), self.side)
        for _ in range(100):
            base = self.bases[int(rng.integers(len(self.bases)))]
            x = np.mod(base - rng.uniform(0.0, self.side, 3), self.side)
            if L < self.side:
                x = x[np.all(x < L, axis=1)]
            if x.shape[0] < 2:
                continue
            near = np.nonzero(np.any((x < self.dmin) | (x > L - self.dmin), axis=1))[0]
            keep = np.ones(x.shape[0], dtype=bool)
            if near.size > 1:
                # only pairs that meet through the new periodic faces can be
                # closer than dmin (the base packing keeps every other pair apart)
                xs = np.clip(x[near], 0.0, np.nextafter(L, 0.0))
                pairs = cKDTree(xs, boxsize=L).query_pairs(self.dmin, output_type="ndarray")
                sub = _drop_close_pairs(pairs, np.ones(near.size, dtype=bool))
                keep[near[~sub]] = False
            x = x[keep]
            x[x >= L] -= L          # np.mod may round up to the side itself
            x = np.ascontiguousarray(x)
            if x.shape[0] >= 2:
                return x, np.eye(3) * L, (np.arange(x.shape[0]) % n_species).astype(np.int32)
        raise RuntimeError("PackingSource.cut: no configuration with two atoms")


def stream_draws(n_req, mix, n_min=16, n_max=32768, seed=0):
    """Per request: atom count (log-uniform in [n_min, n_max]) and lane
    (drawn with the probabilities of ``mix``)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_req)).round().astype(np.int64)
    names = list(mix)
    p = np.array([mix[k] for k in names], dtype=np.float64)
    lanes = [names[i] for i in rng.choice(len(names), size=n_req, p=p / p.sum())]
    return sizes, lanes


class GradientPool:
    """dL/d(desc) of the requests: N(0, 1) rows, one seeded block per lane;
    a request takes a contiguous run of rows at its own random offset, so
    memory stays bounded however long the stream."""

    def __init__(self, widths: dict, n_max=32768, seed=0):
        self.n_max = int(n_max)
        self.blocks = {k: np.random.default_rng(seed * 31 + i).normal(size=(2 * self.n_max, w))
                       for i, (k, w) in enumerate(sorted(widths.items()))}

    def take(self, lane, rows, rng):
        o = int(rng.integers(0, self.blocks[lane].shape[0] - rows + 1))
        return self.blocks[lane][o:o + rows]


def stream_requests(n_req, widths, mix, prepare, n_min=16, n_max=32768, density=0.05, dmin=2.0, cutoff=5.0,
                    seed=0, source=None, grads=None, first=0, last=None):
    """Requests first .. last-1 of an n_req-request stream as (i, lane, cfg,
    dE): request i's atom count and lane come from ``stream_draws``, its
    packing from ``source.cut`` with the generator seeded by (seed, i), its
    ghosts and neighbour lists from ``prepare(coords, cell, species,
    cutoff)`` (any builder of the reference's layout), its dL/d(desc) from
    ``grads``.  Request i depends only on (seed, i)."""
    sizes, lanes = stream_draws(n_req, mix, n_min, n_max, seed)
    source = source or PackingSource(density=density, dmin=dmin, seed=seed)
    grads = grads or GradientPool(widths, n_max, seed)
    for i in range(first, n_req if last is None else min(last, n_req)):
        rng = np.random.default_rng([seed, i])
        x, cell, sp = source.cut(int(sizes[i]), rng)
        cfg = prepare(x, cell, sp, cutoff)
        yield i, lanes[i], cfg, grads.take(lanes[i], cfg.n_atoms, rng)
