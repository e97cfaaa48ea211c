"""torch.autograd.Function over the descriptor kernels.

``descriptors(kind, coords, rows)`` returns the (n_rows, width) FP64
descriptors of device tensor ``coords`` (n_total, 3) and records a backward
that runs the fused descriptor + VJP kernel: the reverse pass recomputes the
forward on chip and contracts with the upstream gradient dL/d(desc), so the
per-neighbour Jacobian is never stored (the reference differentiates
``Descriptor::compute`` with Enzyme instead, src/Descriptors.cpp:165-215).
The gradient w.r.t. ``coords`` has the shape of ``coords``: ghost rows get
their own gradient, as the reference's ``gradient`` returns it; fold them
onto masters with ``fold_image`` (or by building the ghosts from the masters
with torch ops, so that autograd folds them).

Double backward is not provided.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _ext


@dataclass
class Rows:
    """Device-resident neighbour rows (the reference's per-call
    ``species``, ``neighbor_list``, ``number_of_neighs`` arguments)."""

    n_rows: int
    species: torch.Tensor       # (n_total,) i32
    nbl: torch.Tensor           # (nnz,) i32
    off: torch.Tensor           # (n_rows + 1,) i64
    max_neigh: int
    row_centre: torch.Tensor | None = None   # (n_rows,) i32; None: centre == row

    @classmethod
    def build(cls, kind, species, neighbor_list, number_of_neighs, device="cuda", row_centre=None) -> "Rows":
        dev = torch.device(device)

        def t(a, dt):
            if isinstance(a, torch.Tensor):
                return a.to(device=dev, dtype=dt).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)

        counts = t(number_of_neighs, torch.int32)
        n_rows = int(counts.shape[0])
        nbl = t(neighbor_list, torch.int32)
        if nbl.numel() == 0:
            nbl = torch.zeros(1, dtype=torch.int32, device=dev)
        off = torch.empty(n_rows + 1, dtype=torch.int64, device=dev)
        s = torch.cuda.current_stream(dev).cuda_stream
        mx = int(_ext._neighbor_offsets_dev(kind, n_rows, counts.data_ptr(), off.data_ptr(), True, s))
        rc = t(row_centre, torch.int32) if row_centre is not None else None
        return cls(n_rows, t(species, torch.int32), nbl, off, max(mx, 1), rc)


def _check_coords(coords: torch.Tensor) -> None:
    if not coords.is_cuda or coords.dtype != torch.float64 or coords.dim() != 2 or coords.shape[1] != 3:
        raise ValueError("coords must be a CUDA float64 tensor of shape (n_total, 3)")


class DescriptorFunction(torch.autograd.Function):
    """desc = D(coords); backward: dL/dcoords = VJP(coords, dL/ddesc)."""

    @staticmethod
    def forward(ctx, coords, kind, rows: Rows):
        _check_coords(coords)
        coords_c = coords.detach().contiguous()
        W = int(kind.width)
        desc = torch.empty((rows.n_rows, W), dtype=torch.float64, device=coords.device)
        s = torch.cuda.current_stream(coords.device).cuda_stream
        rc = rows.row_centre.data_ptr() if rows.row_centre is not None else 0
        _ext._compute_dev(kind, rows.n_rows, rc, rows.species.data_ptr(), rows.nbl.data_ptr(), rows.off.data_ptr(),
                          rows.max_neigh, coords_c.data_ptr(), desc.data_ptr(), s)
        ctx.kind = kind
        ctx.rows = rows
        ctx.save_for_backward(coords_c)
        return desc

    @staticmethod
    def backward(ctx, grad_desc):
        (coords_c,) = ctx.saved_tensors
        rows: Rows = ctx.rows
        g = grad_desc.to(torch.float64).contiguous()
        dc = torch.zeros_like(coords_c)
        s = torch.cuda.current_stream(coords_c.device).cuda_stream
        rc = rows.row_centre.data_ptr() if rows.row_centre is not None else 0
        _ext._gradient_dev(ctx.kind, rows.n_rows, rc, rows.species.data_ptr(), rows.nbl.data_ptr(),
                           rows.off.data_ptr(), rows.max_neigh, coords_c.data_ptr(), g.data_ptr(), dc.data_ptr(),
                           0, 0, s)
        return dc, None, None


def descriptors(kind, coords: torch.Tensor, rows: Rows) -> torch.Tensor:
    """Differentiable descriptors of ``coords`` (see module docstring)."""
    return DescriptorFunction.apply(coords, kind, rows)


def sync_status(kind) -> None:
    """Raise the first device-side error (capacity / bad index) of ``kind``'s
    kernels on the current stream."""
    _ext._sync_status(kind, torch.cuda.current_stream().cuda_stream)


def fold_image(grad: torch.Tensor, n_atoms: int, image) -> torch.Tensor:
    """Ghost rows added onto their masters (the reference's assemble_forces,
    python_package/libdescriptor/neighbor.py:227-263)."""
    img = torch.as_tensor(np.asarray(image), device=grad.device, dtype=torch.int64)
    out = grad[:n_atoms].clone()
    out.index_add_(0, img[n_atoms:], grad[n_atoms:])
    return out
