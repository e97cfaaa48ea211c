"""Test helpers: build the oracle and the GPU descriptor for a golden fixture,
and the tolerance rule used by every parity test.

Tolerance (the parity bar: descriptors 1e-10 relative, gradients 1e-8):
an element passes when

    |x - ref| <= rtol * max(|ref|, 1e-3 * scale_c)

where scale_c is the largest |ref| of that output column (descriptor
component, or the gradient over all rows).  The floor keeps values that are
exact cancellations of O(scale) terms -- whose absolute error is set by the
size of the terms, not by the tiny result -- from failing on round-off.
"""
from __future__ import annotations

import numpy as np

from conftest import sf24, sf_mixed

DESC_RTOL = 1e-10
GRAD_RTOL = 1e-8


def rel_err(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.size == 0:
        return 0.0
    r2 = ref.reshape(ref.shape[0], -1) if ref.ndim > 1 else ref.reshape(-1, 1)
    x2 = x.reshape(r2.shape)
    scale = np.max(np.abs(r2), axis=0, keepdims=True)
    den = np.maximum(np.abs(r2), 1e-3 * scale)
    den = np.where(den == 0, 1.0, den)
    return float(np.max(np.abs(x2 - r2) / den))


def assert_close(x, ref, rtol, what=""):
    e = rel_err(x, ref)
    assert np.all(np.isfinite(np.asarray(x))), f"{what}: non-finite values"
    assert e <= rtol, f"{what}: relative error {e:.3e} > {rtol:.1e}"
    return e


def kind_of(name: str) -> str:
    return "sf" if name.startswith("sf") else "bs"


def sf_params_of(name):
    return sf_mixed() if "mixed" in name else sf24()


def cutoff_matrix(g, n_species):
    if "cutoff_matrix" in g:
        return np.asarray(g["cutoff_matrix"], dtype=np.float64)
    return np.full((n_species, n_species), float(g["cutoff"]))


def n_species_of(g):
    return int(np.max(g["species"])) + 1


def bzero_of(g) -> int:
    """The golden's bzero_flag (fixtures made before it was recorded: 0)."""
    return int(g["bzero_flag"]) if "bzero_flag" in g else 0


def oracle_for(name, g):
    from oracle import OracleDescriptor

    ns = n_species_of(g)
    if kind_of(name) == "sf":
        t, s, p = sf_params_of(name)
        return OracleDescriptor.symmetry_functions(ns, cutoff_matrix(g, ns), t, s, p)
    return OracleDescriptor.bispectrum(float(g["rfac0"]), int(g["twojmax"]), int(g["style"]),
                                       float(g["rmin0"]), int(g["switch_flag"]), bzero_of(g), ns,
                                       cutoff_matrix(g, ns), g["weights"])


def gpu_for(name, g):
    """GPU descriptor through the C ABI (ctypes handle wrapper)."""
    from abi import Abi

    ns = n_species_of(g)
    if kind_of(name) == "sf":
        t, s, p = sf_params_of(name)
        return Abi.create_sf(ns, cutoff_matrix(g, ns), t, s, p)
    return Abi.create_bs(float(g["rfac0"]), int(g["twojmax"]), int(g["style"]), float(g["rmin0"]),
                         int(g["switch_flag"]), bzero_of(g), ns, cutoff_matrix(g, ns), g["weights"])
