"""Generate the committed golden fixtures from the REFERENCE's own C++.

Run in a container that has the reference source tree (it builds
oracle/_ref/libldref.so from it with oracle/Makefile):

    python tests/golden/make_golden.py

Each fixture stores seeded inputs in the reference layout and the
reference's outputs on them:
  * desc      -- DescriptorKind::compute over every centre (reference C++)
  * fd_index, fd_dE, fd_grad -- the reference's own finite-difference
    self-gradient (num_gradient_single_atom, 8th-order stencil) of a few
    centres, which pins the analytic gradients.
Inputs are generated with numpy + the reference's neighbour builder, so the
fixtures do not depend on this library at all.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import Reference, ReferenceDescriptor  # noqa: E402

_DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])


def diamond(n, a=5.43, jitter=0.05, seed=0):
    rng = np.random.default_rng(seed)
    grid = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    x = ((grid[:, None, :] + _DIAMOND[None]) * a).reshape(-1, 3)
    return x + rng.normal(0, jitter, x.shape), np.eye(3) * a * n


def packing(n, density=0.05, dmin=2.0, seed=0):
    rng = np.random.default_rng(seed)
    side = (n / density) ** (1 / 3)
    pts = []
    while len(pts) < n:
        c = rng.uniform(0, side, 3)
        ok = True
        for p in pts:
            d = c - p
            d -= side * np.round(d / side)
            if d @ d < dmin * dmin:
                ok = False
                break
        if ok:
            pts.append(c)
    return np.array(pts), np.eye(3) * side


def layout(x, cell, species, rc):
    pc, ps, pi = Reference.create_paddings(rc, cell, [1, 1, 1], x, species)
    allx = np.concatenate([x, pc])
    alls = np.concatenate([species, ps]).astype(np.int32)
    need = np.zeros(len(allx), np.int32)
    need[: len(x)] = 1
    counts, nbl = Reference.neighbor_list(allx, rc, need, len(x))
    image = np.concatenate([np.arange(len(x)), pi]).astype(np.int32)
    return allx, alls, counts.astype(np.int32), nbl.astype(np.int32), image


def sf24():
    g2 = [[e, 0.0] for e in (0.001, 0.005, 0.01, 0.02, 0.04, 0.08, 0.16, 0.32)]
    g4 = [[z, l, e] for z in (1.0, 4.0) for l in (-1.0, 1.0) for e in (0.001, 0.01, 0.03, 0.08)]
    return ["g2", "g4"], [8, 2, 16, 3], np.array(sum(g2, []) + sum(g4, []))


def sf_mixed():
    # every symmetry-function type, non-integer zeta, shifted Rs
    g1 = []
    g2 = [[0.05, 1.5], [0.3, 2.5]]
    g3 = [[1.3], [2.7]]
    g4 = [[1.5, 1.0, 0.02], [2.0, -1.0, 0.05], [3.3, 1.0, 0.005]]
    g5 = [[1.0, -1.0, 0.01], [2.5, 1.0, 0.03]]
    types = ["g1", "g2", "g3", "g4", "g5"]
    sizes = [1, 1, 2, 2, 2, 1, 3, 3, 2, 3]
    params = np.array([0.0] + sum(g2, []) + sum(g3, []) + sum(g4, []) + sum(g5, []))
    del g1
    return types, sizes, params


def save(name, **kw):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **kw)
    print("wrote", name, {k: np.asarray(v).shape for k, v in kw.items()})


def smooth_centres(x, counts, nbl, rc, k, margin=0.16, pairs=True):
    """Centres whose every neighbour (and neighbour pair) distance stays
    `margin` away from the cutoff: the 8th-order stencil (step ~0.037, reach
    ~0.15) is then accurate, since the cutoff functions are only C1 at rc."""
    off = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for i in range(len(counts)):
        nb = nbl[off[i]:off[i + 1]]
        d = np.linalg.norm(x[nb] - x[i], axis=1)
        dd = np.linalg.norm(x[nb][:, None] - x[nb][None], axis=2)[np.triu_indices(len(nb), 1)]
        if np.all(np.abs(d - rc) > margin) and (not pairs or np.all(np.abs(dd - rc) > margin)):
            out.append(i)
        if len(out) == k:
            break
    return out


def fd_pin(ref, x, s, counts, nbl, width, centres, seed):
    rng = np.random.default_rng(seed)
    off = np.concatenate([[0], np.cumsum(counts)])
    dEs, grads = [], []
    for i in centres:
        dE = rng.normal(size=width)
        g = ref.num_gradient_single_atom(int(i), s, nbl[off[i]:off[i + 1]], x, dE)
        dEs.append(dE)
        grads.append(g)
    return np.asarray(centres, np.int32), np.asarray(dEs), np.asarray(grads)


def main():
    oracle.build(with_ref=True)
    rc = 5.0
    # the 64-atom diamond with the 24-d symmetry functions
    x, cell = diamond(2, jitter=0.05, seed=0)
    sp = np.zeros(len(x), np.int32)
    allx, alls, counts, nbl, image = layout(x, cell, sp, rc)
    types, sizes, params = sf24()
    ref = ReferenceDescriptor.symmetry_functions(1, np.full((1, 1), rc), types, sizes, params)
    desc = ref.compute(len(x), alls, nbl, counts, allx)
    fi, fdE, fg = fd_pin(ref, allx, alls, counts, nbl, ref.width,
                         smooth_centres(allx, counts, nbl, rc, 3), 1)
    save("sf24_diamond64", n_atoms=len(x), coords=allx, species=alls, counts=counts, nbl=nbl,
         image=image, cutoff=rc, desc=desc, fd_index=fi, fd_dE=fdE, fd_grad=fg)
    # all five symmetry-function types, two species with a species-pair cutoff matrix
    xr, cellr = packing(48, seed=3)
    sp2 = (np.arange(48) % 2).astype(np.int32)
    allx, alls, counts, nbl, image = layout(xr, cellr, sp2, 5.5)
    types, sizes, params = sf_mixed()
    cm = np.array([[5.5, 4.5], [4.5, 5.0]])
    ref = ReferenceDescriptor.symmetry_functions(2, cm, types, sizes, params)
    desc = ref.compute(48, alls, nbl, counts, allx)
    save("sf_mixed_packing48", n_atoms=48, coords=allx, species=alls, counts=counts, nbl=nbl,
         image=image, cutoff_matrix=cm, desc=desc)
    # bispectrum: 2J = 8 / 6 style 3 on a two-species packing; styles 0..2
    xr, cellr = packing(64, seed=5)
    sp2 = (np.arange(64) % 2).astype(np.int32)
    allx, alls, counts, nbl, image = layout(xr, cellr, sp2, rc)
    cm = np.full((2, 2), rc)
    for J, style, sw in ((8, 3, 1), (6, 3, 1), (4, 0, 1), (4, 1, 1), (4, 2, 1), (6, 3, 0)):
        ref = ReferenceDescriptor.bispectrum(0.99363, J, style, 0.0, sw, 0, 2, cm, [1.0, 0.5])
        desc = ref.compute(64, alls, nbl, counts, allx)
        kw = {}
        if style == 3 and sw == 1:
            fi, fdE, fg = fd_pin(ref, allx, alls, counts, nbl, ref.width,
                                     smooth_centres(allx, counts, nbl, rc, 3, pairs=False), 2)
            kw = dict(fd_index=fi, fd_dE=fdE, fd_grad=fg)
        save(f"bs_j{J}_style{style}_sw{sw}_packing64", n_atoms=64, coords=allx, species=alls,
             counts=counts, nbl=nbl, image=image, cutoff=rc, twojmax=J, style=style,
             switch_flag=sw, rfac0=0.99363, rmin0=0.0, weights=np.array([1.0, 0.5]), desc=desc, **kw)
    # bzero_flag: the reference subtracts bzero[j] = j w_self^3 from every
    # B of output layer j (src/Bispectrum.cpp:64-67, 423)
    ref = ReferenceDescriptor.bispectrum(0.99363, 6, 3, 0.0, 1, 1, 2, cm, [1.0, 0.5])
    desc = ref.compute(64, alls, nbl, counts, allx)
    save("bs_j6_bzero_packing64", n_atoms=64, coords=allx, species=alls, counts=counts, nbl=nbl,
         image=image, cutoff=rc, twojmax=6, style=3, switch_flag=1, bzero_flag=1, rfac0=0.99363, rmin0=0.0,
         weights=np.array([1.0, 0.5]), desc=desc)
    # non-uniform species-pair cutoffs: the reference reads the bispectrum
    # cutoff as element [jSpecies] of the flattened matrix
    cmq = np.array([[5.0, 4.0], [4.5, 3.5]])
    ref = ReferenceDescriptor.bispectrum(0.99363, 6, 3, 0.0, 1, 0, 2, cmq, [1.0, 0.5])
    desc = ref.compute(64, alls, nbl, counts, allx)
    save("bs_j6_cutmatrix_packing64", n_atoms=64, coords=allx, species=alls, counts=counts, nbl=nbl,
         image=image, cutoff_matrix=cmq, twojmax=6, style=3, switch_flag=1, rfac0=0.99363, rmin0=0.0,
         weights=np.array([1.0, 0.5]), desc=desc)
    # bispectrum with rmin0 > 0 on the diamond cell
    x, cell = diamond(2, jitter=0.1, seed=7)
    sp = np.zeros(len(x), np.int32)
    allx, alls, counts, nbl, image = layout(x, cell, sp, rc)
    ref = ReferenceDescriptor.bispectrum(0.97, 6, 3, 0.5, 1, 0, 1, np.full((1, 1), rc), [1.0])
    desc = ref.compute(len(x), alls, nbl, counts, allx)
    save("bs_j6_rmin_diamond64", n_atoms=len(x), coords=allx, species=alls, counts=counts, nbl=nbl,
         image=image, cutoff=rc, twojmax=6, style=3, switch_flag=1, rfac0=0.97, rmin0=0.5,
         weights=np.array([1.0]), desc=desc)


if __name__ == "__main__":
    main()
