"""libdescriptor_b200 -- B200-native (sm_100a) drop-in for libdescriptor's
per-atom descriptor hot path.

The module mirrors the reference's Python package ``libdescriptor``
(python_bindings/python_bindings.cpp:50-556,
python_package/libdescriptor/__init__.py): ``AvailableDescriptors``,
``DescriptorKind.init_descriptor`` (symmetry functions, bispectrum, parameter
files), ``compute`` / ``compute_batch`` / ``compute_single_atom``,
``gradient`` / ``gradient_batch`` / ``gradient_single_atom``, ``jacobian``,
``num_gradient_single_atom``, ``NeighList`` / ``create`` and
``create_paddings``.  Every compute call runs the hand-written CUDA kernels
of ``_lib/libldb200.so`` in FP64; there is no CPU fallback -- without a CUDA
device the calls raise.

Extras beyond the reference API: ``gradient_params`` (dL/d(parameters):
the symmetry functions' eta, Rs, kappa, zeta, lambda or the bispectrum's
rfac0, which the reference computes with Enzyme and discards), ``torch_ops``
(torch.autograd.Function over
device tensors), ``batch`` (one launch over many configurations, CUDA
graphs, autotuning) and ``serving`` (continuous-batching request loop).
"""
from __future__ import annotations

import enum
import os

_HERE = os.path.dirname(os.path.abspath(__file__))

try:
    from . import _libdescriptor as _ext
except ImportError as exc:  # fail loudly: no silent fallback
    raise ImportError(
        "libdescriptor_b200: native extension not built "
        "(run `python libdescriptor_b200/build.py`): " + str(exc)) from exc


class AvailableDescriptors(enum.IntEnum):
    """Descriptor kinds, numbered as the reference's AvailableDescriptor
    (include/Descriptors.hpp:21-26)."""

    SymmetryFunctions = 0
    Bispectrum = 1
    SOAP = 2
    Xi = 3


DescriptorKind = _ext.DescriptorKind
compute = _ext.compute
compute_batch = _ext.compute_batch
compute_single_atom = _ext.compute_single_atom
gradient = _ext.gradient
gradient_batch = _ext.gradient_batch
gradient_single_atom = _ext.gradient_single_atom
compute_and_gradient = _ext.compute_and_gradient
gradient_params = _ext.gradient_params
jacobian = _ext.jacobian
num_gradient_single_atom = _ext.num_gradient_single_atom
NeighList = _ext.NeighList
create = _ext.create
create_paddings = _ext.create_paddings

LIB_PATH = os.path.join(_HERE, "_lib", "libldb200.so")


def launch_count() -> int:
    """Number of this library's kernel launches issued by this process."""
    return int(_ext._launch_count())


def measure_fp64_peak(iters: int = 4096) -> float:
    """Achieved FP64 FMA rate of the current device in TFLOP/s."""
    return float(_ext._measure_fp64_peak(int(iters)))


__all__ = [
    "AvailableDescriptors", "DescriptorKind", "compute", "compute_batch",
    "compute_single_atom", "gradient", "gradient_batch", "gradient_single_atom",
    "compute_and_gradient", "gradient_params",
    "jacobian", "num_gradient_single_atom", "NeighList", "create",
    "create_paddings", "launch_count", "measure_fp64_peak", "LIB_PATH",
]
