"""Seeded synthetic inputs: periodic cells, ghost padding and neighbour lists.

The reference measures nothing on a public dataset; these generators build the
cells its documented use implies (periodic Si diamond supercells, random
two-species packings) and turn them into the reference's input layout with the
library's own padding / neighbour-list builder (``create_paddings`` and
``NeighList``, the KLIFF-derived algorithm of
python_bindings/neighbor/neighbor_list.cpp).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _libdescriptor as _ext

# the pure-numpy generators live in synth.py (importable without the extension)
from .synth import (DIAMOND, SF24_G2_ETA, SF24_G4_ETA, diamond_cell,  # noqa: E402,F401
                    random_packing, sf24_params)


@dataclass
class Config:
    """One configuration in the reference's input layout."""

    n_atoms: int
    coords: np.ndarray          # (n_total, 3): contributing atoms then ghosts
    species: np.ndarray         # (n_total,) int32
    image: np.ndarray           # (n_total,) master atom of each row
    counts: np.ndarray          # (n_atoms,) int32
    nbl: np.ndarray             # (sum counts,) int32
    cell: np.ndarray = field(default=None)

    @property
    def n_total(self) -> int:
        return int(self.coords.shape[0])


def prepare(coords, cell, species, cutoff, pbc=(1, 1, 1)) -> Config:
    """Ghost padding + full neighbour list within `cutoff` of every
    contributing atom (reference NeighborList semantics)."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    species = np.ascontiguousarray(species, dtype=np.int32)
    n = coords.shape[0]
    pc, ps, pi = _ext.create_paddings(float(cutoff), np.ascontiguousarray(cell, dtype=np.float64),
                                      np.asarray(pbc, dtype=np.int32), coords, species)
    allx = np.ascontiguousarray(np.concatenate([coords, pc]))
    alls = np.ascontiguousarray(np.concatenate([species, ps]).astype(np.int32))
    image = np.concatenate([np.arange(n, dtype=np.int32), pi.astype(np.int32)])
    need = np.zeros(allx.shape[0], dtype=np.int32)
    need[:n] = 1
    nl = _ext.NeighList()
    nl.build(allx, float(cutoff), np.asarray([cutoff], dtype=np.float64), need)
    counts = np.zeros(n, dtype=np.int32)
    lists = []
    cut = np.asarray([cutoff], dtype=np.float64)
    for i in range(n):
        c, nb = nl.get_neigh(cut, 0, i)
        counts[i] = c
        lists.append(nb)
    nbl = np.ascontiguousarray(np.concatenate(lists).astype(np.int32)) if lists else np.zeros(0, np.int32)
    return Config(n, allx, alls, image, counts, nbl, np.asarray(cell))


@dataclass
class Batch:
    """Concatenated configurations in the compute_batch layout
    (src/Descriptors.cpp:138-163): centre of row (c, j) is j + config_ptr[c]."""

    n_atoms: np.ndarray
    config_ptr: np.ndarray
    coords: np.ndarray
    species: np.ndarray
    image: np.ndarray           # global master row of every coordinate row
    counts: np.ndarray
    nbl: np.ndarray
    row_centre: np.ndarray
    contrib_rows: np.ndarray    # global coordinate row of every centre

    @property
    def n_rows(self) -> int:
        return int(self.n_atoms.sum())


def concat(configs) -> Batch:
    n_atoms, ptr, xs, ss, ims, cnts, nbls, centres = [], [], [], [], [], [], [], []
    base = 0
    for c in configs:
        n_atoms.append(c.n_atoms)
        ptr.append(base)
        xs.append(c.coords)
        ss.append(c.species)
        ims.append(c.image + base)
        cnts.append(c.counts)
        nbls.append(c.nbl + base)
        centres.append(np.arange(c.n_atoms, dtype=np.int32) + base)
        base += c.n_total
    rc = np.concatenate(centres).astype(np.int32)
    return Batch(np.asarray(n_atoms, np.int32), np.asarray(ptr, np.int32),
                 np.ascontiguousarray(np.concatenate(xs)), np.concatenate(ss).astype(np.int32),
                 np.concatenate(ims).astype(np.int32), np.concatenate(cnts).astype(np.int32),
                 np.concatenate(nbls).astype(np.int32), rc, rc)


def fold(grad, n_atoms, image):
    """Ghost rows added onto their masters (the reference's assemble_forces,
    python_package/libdescriptor/neighbor.py:227-263)."""
    out = np.array(grad[:n_atoms], dtype=np.float64, copy=True)
    np.add.at(out, image[n_atoms:], grad[n_atoms:])
    return out


@dataclass
class DeviceConfig:
    """One configuration prepared on the device (``prepare_dev``): torch
    tensors in the reference's layout plus the CSR row offsets."""

    n_atoms: int
    coords: object      # (n_total, 3) f64: contributing atoms, then ghosts
    species: object     # (n_total,) i32
    image: object       # (n_total,) i32
    counts: object      # (n_atoms,) i32
    off: object         # (n_atoms + 1,) i64
    nbl: object         # (nnz,) i32
    max_neigh: int

    @property
    def n_total(self) -> int:
        return int(self.coords.shape[0])

    def to_host(self, cell=None) -> Config:
        """The same configuration as host arrays (the ``prepare`` layout)."""
        return Config(self.n_atoms, self.coords.cpu().numpy(), self.species.cpu().numpy(),
                      self.image.cpu().numpy(), self.counts.cpu().numpy(), self.nbl.cpu().numpy(),
                      None if cell is None else np.asarray(cell))


def prepare_dev(coords, cell, species, cutoff, pbc=(1, 1, 1), device="cuda", stream=None) -> DeviceConfig:
    """``prepare`` on the device: ghost padding and the full neighbour list of
    the contributing atoms with the library's device builder
    (``ld_create_paddings_dev`` / ``ld_build_neighbor_list_dev``); the ghosts
    and lists are identical to the host builder's."""
    import torch

    dev = torch.device(device)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    x = torch.as_tensor(np.ascontiguousarray(coords, dtype=np.float64), device=dev)
    sp = torch.as_tensor(np.ascontiguousarray(species, dtype=np.int32), device=dev)
    n = int(x.shape[0])
    cellf = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    pbci = np.ascontiguousarray(pbc, dtype=np.int32)
    m = _ext._create_paddings_dev(float(cutoff), cellf, pbci, x.data_ptr(), sp.data_ptr(), n, 0, 0, 0, 0,
                                  s.cuda_stream)
    allx = torch.empty((n + m, 3), dtype=torch.float64, device=dev)
    alls = torch.empty(n + m, dtype=torch.int32, device=dev)
    image = torch.empty(n + m, dtype=torch.int32, device=dev)
    allx[:n] = x
    alls[:n] = sp
    image[:n] = torch.arange(n, dtype=torch.int32, device=dev)
    if m:
        _ext._create_paddings_dev(float(cutoff), cellf, pbci, x.data_ptr(), sp.data_ptr(), n, m,
                                  allx[n:].data_ptr(), alls[n:].data_ptr(), image[n:].data_ptr(), s.cuda_stream)
    need = torch.zeros(n + m, dtype=torch.int32, device=dev)
    need[:n] = 1
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    nnz, _ = _ext._build_neighbor_list_dev(allx.data_ptr(), n + m, float(cutoff), need.data_ptr(), n,
                                           counts.data_ptr(), off.data_ptr(), 0, 0, s.cuda_stream)
    nbl = torch.empty(max(int(nnz), 1), dtype=torch.int32, device=dev)
    nnz, mx = _ext._build_neighbor_list_dev(allx.data_ptr(), n + m, float(cutoff), need.data_ptr(), n,
                                            counts.data_ptr(), off.data_ptr(), int(nnz), nbl.data_ptr(),
                                            s.cuda_stream)
    return DeviceConfig(n, allx, alls, image, counts, off, nbl[:int(nnz)], max(int(mx), 1))
