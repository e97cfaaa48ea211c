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

    def __init__(self, n_base=4, base_atoms=32768, density=0.05, dmin=2.0, seed=0, bases=None):
        from scipy.spatial import cKDTree

        self.density, self.dmin = float(density), float(dmin)
        self.bases = bases if bases is not None else [
            random_packing(base_atoms, density, dmin, n_species=1, seed=seed * 1000 + 17 + i)[0]
            for i in range(n_base)]
        self.side = (base_atoms / density) ** (1.0 / 3.0)
        # periodic trees of the bases: a small cube is gathered from the ball
        # around its centre instead of a scan of the whole base
        self.trees = [cKDTree(np.clip(b, 0.0, np.nextafter(self.side, 0.0)), boxsize=self.side)
                      for b in self.bases]

    def _candidates(self, b, o, L):
        """Indices of base b's atoms that may lie in the cube [o, o + L) (periodic)."""
        if L > 0.45 * self.side:
            return None
        c = np.mod(o + 0.5 * L, self.side)
        return np.asarray(self.trees[b].query_ball_point(c, 0.5 * np.sqrt(3.0) * L * (1.0 + 1e-9)), dtype=np.int64)

    def cut(self, n, rng, n_species=2):
        """About n atoms in a periodic cube of side (n / density)^(1/3):
        coordinates, cell (rows = lattice vectors), species (alternating)."""
        L = min((n / self.density) ** (1.0 / 3.0), self.side)
        for _ in range(100):
            b = int(rng.integers(len(self.bases)))
            o = rng.uniform(0.0, self.side, 3)
            cand = self._candidates(b, o, L)
            x = (self.bases[b] if cand is None else self.bases[b][np.sort(cand)]) - o
            x += (x < 0.0) * self.side
            x[x >= self.side] -= self.side
            if L < self.side:
                x = x[(x[:, 0] < L) & (x[:, 1] < L) & (x[:, 2] < L)]
            if x.shape[0] < 2:
                continue
            x = x[_face_conflicts_kept(x, L, self.dmin)]
            x = np.ascontiguousarray(x)
            if x.shape[0] >= 2:
                return x, np.eye(3) * L, (np.arange(x.shape[0]) % n_species).astype(np.int32)
        raise RuntimeError("PackingSource.cut: no configuration with two atoms")


def _face_conflicts_kept(x, L, dmin):
    """Mask of the atoms kept when the cube [0, L)^3 is made periodic: only
    atoms within dmin of a face can meet another one closer than dmin
    through the new periodic faces (every other pair is at least dmin apart
    already).  Those pairs are found among the near-face atoms and their
    images shifted by -L along the axes where they lie near the upper face;
    the later atom of each close pair is dropped."""
    from scipy.spatial import cKDTree

    keep = np.ones(x.shape[0], dtype=bool)
    hi = x > L - dmin
    near = np.nonzero((x < dmin).any(axis=1) | hi.any(axis=1))[0]
    if near.size < 2:
        return keep
    pts, owner = [x[near]], [near]
    hn = hi[near]
    for mask in range(1, 8):
        axes = [d for d in range(3) if mask >> d & 1]
        sel = np.all(hn[:, axes], axis=1)
        if sel.any():
            sh = x[near[sel]].copy()
            sh[:, axes] -= L
            pts.append(sh)
            owner.append(near[sel])
    pts = np.concatenate(pts)
    owner = np.concatenate(owner)
    pairs = cKDTree(pts).query_pairs(dmin, output_type="ndarray")
    if pairs.size == 0:
        return keep
    a, b = owner[pairs[:, 0]], owner[pairs[:, 1]]
    m = a != b
    if not m.any():
        return keep
    # the later atom of every close pair goes (a superset of a greedy pass:
    # every remaining pair is at least dmin apart)
    keep[np.maximum(a[m], b[m])] = False
    return keep


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


_WORKER_SOURCE = None


def _cut_worker_init(bases, base_atoms, density, dmin):
    global _WORKER_SOURCE
    _WORKER_SOURCE = PackingSource(base_atoms=base_atoms, density=density, dmin=dmin, bases=bases)


def _cut_chunk(args):
    seed, first, sizes = args
    out = []
    for k, n in enumerate(sizes):
        x, cell, _ = _WORKER_SOURCE.cut(int(n), np.random.default_rng([seed, first + k]))
        out.append((x, float(cell[0, 0])))
    return out


def stream_cuts(n_req, mix, n_min=16, n_max=32768, seed=0, source=None, first=0, last=None, processes=1):
    """The packings (coordinates, cube side) of requests first .. last-1,
    computed in ``processes`` spawned worker processes when > 1 (the cuts
    hold the interpreter lock; spawning is safe after CUDA is in use)."""
    sizes, _ = stream_draws(n_req, mix, n_min, n_max, seed)
    last = n_req if last is None else min(last, n_req)
    source = source or PackingSource(seed=seed)
    if processes <= 1 or last - first < 256:
        return [(lambda x: (x[0], float(x[1][0, 0])))(source.cut(int(sizes[i]), np.random.default_rng([seed, i])))
                for i in range(first, last)]
    import multiprocessing as mp

    chunk = max(64, (last - first) // (8 * processes))
    jobs = [(seed, c, sizes[c:min(c + chunk, last)]) for c in range(first, last, chunk)]
    base_atoms = int(round(source.density * source.side ** 3))
    with mp.get_context("spawn").Pool(processes, initializer=_cut_worker_init,
                                      initargs=(source.bases, base_atoms, source.density, source.dmin)) as pool:
        parts = pool.map(_cut_chunk, jobs)
    return [c for part in parts for c in part]


def stream_requests(n_req, widths, mix, prepare, n_min=16, n_max=32768, density=0.05, dmin=2.0, cutoff=5.0,
                    seed=0, source=None, grads=None, first=0, last=None, processes=1):
    """Requests first .. last-1 of an n_req-request stream as (i, lane, cfg,
    dE): request i's atom count and lane come from ``stream_draws``, its
    packing from ``source.cut`` with the generator seeded by (seed, i), its
    ghosts and neighbour lists from ``prepare(coords, cell, species,
    cutoff)`` (any builder of the reference's layout), its dL/d(desc) rows
    from ``grads`` at an offset drawn from (seed, i, 1).  Request i depends
    only on (seed, i)."""
    _, lanes = stream_draws(n_req, mix, n_min, n_max, seed)
    last = n_req if last is None else min(last, n_req)
    source = source or PackingSource(density=density, dmin=dmin, seed=seed)
    grads = grads or GradientPool(widths, n_max, seed)
    cuts = stream_cuts(n_req, mix, n_min, n_max, seed, source, first, last, processes)
    for i, (x, L) in zip(range(first, last), cuts):
        sp = (np.arange(x.shape[0]) % 2).astype(np.int32)
        cfg = prepare(x, np.eye(3) * L, sp, cutoff)
        yield i, lanes[i], cfg, grads.take(lanes[i], cfg.n_atoms, np.random.default_rng([seed, i, 1]))
