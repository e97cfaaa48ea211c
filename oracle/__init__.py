"""CPU oracle for the descriptor hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
``--impl reference`` legs import this package, as the checker.  The product
(``libdescriptor_b200``) never imports it and has no CPU fallback.

Two libraries are wrapped with ctypes:

* ``libldoracle.so`` -- the plain-C restatement in ``ld_oracle.c`` (forward of
  symmetry functions and bispectrum following the reference step by step, an
  independent analytic VJP, and the reference's 8th-order finite-difference
  stencil).
* ``_ref/libldref.so`` -- the reference's own C++ (``src/SymmetryFunctions.cpp``,
  ``src/Bispectrum.cpp``, ``src/helper.cpp``,
  ``python_bindings/neighbor/neighbor_list.cpp``) compiled from its source tree
  by ``oracle/Makefile``; present wherever it was built (it travels with the
  repository snapshot as a built file).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libldoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libldref.so")
# the reference source tree (its path on the build machine; override with
# LDB200_REFERENCE_SRC)
REFERENCE_SRC = os.environ.get("LDB200_REFERENCE_SRC", "/root/reference")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(with_ref: bool | None = None) -> None:
    """Compile the oracle (and the reference library when its sources exist)."""
    targets = ["all"]
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REFERENCE_SRC, "src"))
    if with_ref:
        targets.append("ref")
    subprocess.check_call(["make", "-s", "-C", HERE, "REF=" + REFERENCE_SRC] + targets)


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class _Lib:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(cls.PATH):
                raise FileNotFoundError(cls.PATH)
            cls._lib = C.CDLL(cls.PATH)
            cls._declare(cls._lib)
        return cls._lib


class Oracle(_Lib):
    """ctypes wrapper of ld_oracle.c."""

    PATH = ORACLE_SO

    @staticmethod
    def _declare(L):
        L.ldo_sf_new.restype = C.c_void_p
        L.ldo_sf_new.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _ip, _dp]
        L.ldo_sf_free.argtypes = [C.c_void_p]
        L.ldo_sf_width.argtypes = [C.c_void_p]
        L.ldo_bs_new.restype = C.c_void_p
        L.ldo_bs_new.argtypes = [C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                 C.c_int, C.c_int, _dp, _dp]
        L.ldo_bs_free.argtypes = [C.c_void_p]
        L.ldo_bs_width.argtypes = [C.c_void_p]
        L.ldo_run.argtypes = [C.c_int, C.c_void_p, C.c_int, _ip, _ip, _ip, _ip, _ip, _dp,
                              C.c_int, _dp, C.c_void_p, C.c_void_p, C.c_int]
        L.ldo_fd_vjp.argtypes = [C.c_int, C.c_void_p, C.c_int, _ip, _ip, _ip, _dp, C.c_int,
                                 _dp, C.c_int, _ip, _dp, C.c_double, C.c_int]


class OracleDescriptor:
    """One descriptor kind held by the oracle (kind 0 = SF, 1 = BS)."""

    def __init__(self, kind: int, handle: int, width: int, free_fn):
        self.kind, self.handle, self.width, self._free = kind, handle, width, free_fn

    def __del__(self):
        try:
            if self.handle:
                self._free(self.handle)
        except Exception:
            pass

    @classmethod
    def symmetry_functions(cls, n_species, cutoff_matrix, types, sizes, params):
        L = Oracle.lib()
        codes = _i32([int(t.lower().lstrip("g")) for t in types])
        sizes = _i32(sizes).reshape(-1, 2)
        h = L.ldo_sf_new(int(n_species), _f64(cutoff_matrix).ravel(), len(codes), codes,
                         _i32(sizes[:, 0]), _i32(sizes[:, 1]), _f64(params).ravel())
        return cls(0, h, L.ldo_sf_width(h), L.ldo_sf_free)

    @classmethod
    def bispectrum(cls, rfac0, twojmax, diagonalstyle, rmin0, switch_flag, bzero_flag,
                   n_species, cutoff_matrix, weights):
        L = Oracle.lib()
        h = L.ldo_bs_new(float(rfac0), int(twojmax), int(diagonalstyle), float(rmin0),
                         int(switch_flag), int(bzero_flag), int(n_species),
                         _f64(cutoff_matrix).ravel(), _f64(weights).ravel())
        if not h:
            raise ValueError("invalid bispectrum parameters")
        return cls(1, h, L.ldo_bs_width(h), L.ldo_bs_free)

    def run(self, n_atoms, species, nbl, counts, coords, dE=None, n_configs=0,
            config_ptr=None, n_threads=None):
        """desc (rows x width) and, when dE is given, the unfolded coordinate
        gradient (n_total x 3)."""
        L = Oracle.lib()
        coords = _f64(coords).reshape(-1, 3)
        n_total = coords.shape[0]
        n_atoms = _i32(np.atleast_1d(n_atoms))
        config_ptr = _i32(config_ptr if config_ptr is not None else [0])
        rows = int(n_atoms.sum()) if n_configs else int(n_atoms[0])
        desc = np.zeros((rows, self.width), dtype=np.float64)
        n_threads = n_threads or os.cpu_count() or 1
        dcoords = None
        if dE is not None:
            dE = _f64(dE).reshape(rows, self.width)
            dcoords = np.zeros((n_total, 3), dtype=np.float64)
        L.ldo_run(self.kind, self.handle, int(n_configs), n_atoms, config_ptr,
                  _i32(species), _i32(nbl), _i32(counts), coords.ravel(), n_total, desc,
                  dE.ctypes.data if dE is not None else None,
                  dcoords.ctypes.data if dcoords is not None else None, int(n_threads))
        return (desc, dcoords) if dE is not None else desc

    def fd_vjp(self, n_atoms, species, nbl, counts, coords, dE, flat_idx, step=1e-5,
               n_threads=None):
        """Finite-difference VJP; step > 0: central difference with that
        step, step <= 0: the reference's 8th-order stencil."""
        L = Oracle.lib()
        coords = _f64(coords).reshape(-1, 3)
        idx = _i32(flat_idx)
        out = np.zeros(idx.shape[0], dtype=np.float64)
        L.ldo_fd_vjp(self.kind, self.handle, int(n_atoms), _i32(species), _i32(nbl),
                     _i32(counts), coords.ravel(), coords.shape[0],
                     _f64(dE).ravel(), idx.shape[0], idx, out, float(step),
                     int(n_threads or os.cpu_count() or 1))
        return out


class Reference(_Lib):
    """ctypes wrapper of the reference's own C++ (oracle/_ref/libldref.so)."""

    PATH = REF_SO

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    @staticmethod
    def _declare(L):
        L.ref_sf_new.restype = C.c_void_p
        L.ref_sf_new.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp]
        L.ref_bs_new.restype = C.c_void_p
        L.ref_bs_new.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                 C.c_int, C.c_int, _dp, _dp]
        L.ref_from_file.restype = C.c_void_p
        L.ref_from_file.argtypes = [C.c_char_p, C.c_int]
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_width.argtypes = [C.c_void_p]
        L.ref_compute.argtypes = [C.c_void_p, C.c_int, _ip, _ip, _ip, _ip, _ip, _dp, _dp,
                                  C.c_int]
        L.ref_num_gradient_single_atom.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip,
                                                   C.c_int, _dp, _dp, _dp]
        L.ref_create_paddings.argtypes = [C.c_double, _dp, _ip, _dp, _ip, C.c_int,
                                          C.POINTER(C.c_int),
                                          C.POINTER(C.POINTER(C.c_double)),
                                          C.POINTER(C.POINTER(C.c_int)),
                                          C.POINTER(C.POINTER(C.c_int))]
        L.ref_nbl_build.argtypes = [_dp, C.c_int, C.c_double, _ip, C.c_int,
                                    C.POINTER(C.POINTER(C.c_int)),
                                    C.POINTER(C.POINTER(C.c_int)),
                                    C.POINTER(C.c_longlong)]
        L.ref_free_buf.argtypes = [C.c_void_p]

    @staticmethod
    def create_paddings(cutoff, cell, pbc, coords, species):
        L = Reference.lib()
        n = C.c_int(0)
        pc = C.POINTER(C.c_double)()
        ps = C.POINTER(C.c_int)()
        pi = C.POINTER(C.c_int)()
        coords = _f64(coords).reshape(-1, 3)
        err = L.ref_create_paddings(float(cutoff), _f64(cell).ravel(), _i32(pbc),
                                    coords.ravel(), _i32(species), coords.shape[0],
                                    C.byref(n), C.byref(pc), C.byref(ps), C.byref(pi))
        if err:
            raise RuntimeError("reference nbl_create_paddings failed")
        m = n.value
        out = (np.ctypeslib.as_array(pc, shape=(max(m, 1) * 3,))[: m * 3].reshape(m, 3).copy(),
               np.ctypeslib.as_array(ps, shape=(max(m, 1),))[:m].copy(),
               np.ctypeslib.as_array(pi, shape=(max(m, 1),))[:m].copy())
        for p in (pc, ps, pi):
            L.ref_free_buf(C.cast(p, C.c_void_p))
        return out

    @staticmethod
    def neighbor_list(coords, cutoff, need_neigh, n_query):
        L = Reference.lib()
        cnt = C.POINTER(C.c_int)()
        nbl = C.POINTER(C.c_int)()
        nnz = C.c_longlong(0)
        coords = _f64(coords).reshape(-1, 3)
        err = L.ref_nbl_build(coords.ravel(), coords.shape[0], float(cutoff),
                              _i32(need_neigh), int(n_query), C.byref(cnt), C.byref(nbl),
                              C.byref(nnz))
        if err:
            raise RuntimeError("reference nbl_build failed")
        counts = np.ctypeslib.as_array(cnt, shape=(max(n_query, 1),))[:n_query].copy()
        k = nnz.value
        flat = np.ctypeslib.as_array(nbl, shape=(max(k, 1),))[:k].copy()
        L.ref_free_buf(C.cast(cnt, C.c_void_p))
        L.ref_free_buf(C.cast(nbl, C.c_void_p))
        return counts, flat


class ReferenceDescriptor:
    def __init__(self, handle, width):
        self.handle, self.width = handle, width

    def __del__(self):
        try:
            if self.handle:
                Reference.lib().ref_free(self.handle)
        except Exception:
            pass

    @classmethod
    def symmetry_functions(cls, n_species, cutoff_matrix, types, sizes, params):
        L = Reference.lib()
        codes = _i32([int(t.lower().lstrip("g")) for t in types])
        h = L.ref_sf_new(int(n_species), _f64(cutoff_matrix).ravel(), len(codes), codes,
                         _i32(sizes).ravel(), _f64(params).ravel())
        return cls(h, L.ref_width(h))

    @classmethod
    def from_file(cls, path, kind):
        """The reference's parameter-file constructors (kind 0: symmetry
        functions, 1: bispectrum)."""
        L = Reference.lib()
        h = L.ref_from_file(os.fsencode(path), int(kind))
        if not h:
            raise ValueError(f"the reference could not read {path}")
        return cls(h, L.ref_width(h))

    @classmethod
    def bispectrum(cls, rfac0, twojmax, diagonalstyle, rmin0, switch_flag, bzero_flag,
                   n_species, cutoff_matrix, weights, use_shared_arrays=0):
        L = Reference.lib()
        h = L.ref_bs_new(float(rfac0), int(twojmax), int(diagonalstyle),
                         int(use_shared_arrays), float(rmin0), int(switch_flag),
                         int(bzero_flag), int(n_species), _f64(cutoff_matrix).ravel(),
                         _f64(weights).ravel())
        return cls(h, L.ref_width(h))

    def compute(self, n_atoms, species, nbl, counts, coords, n_configs=0, config_ptr=None,
                n_threads=1):
        L = Reference.lib()
        n_atoms = _i32(np.atleast_1d(n_atoms))
        config_ptr = _i32(config_ptr if config_ptr is not None else [0])
        rows = int(n_atoms.sum()) if n_configs else int(n_atoms[0])
        desc = np.zeros((rows, self.width), dtype=np.float64)
        L.ref_compute(self.handle, int(n_configs), n_atoms, config_ptr, _i32(species),
                      _i32(nbl), _i32(counts), _f64(coords).ravel(), desc, int(n_threads))
        return desc

    def num_gradient_single_atom(self, index, species, neighbors, coords, dE):
        L = Reference.lib()
        coords = _f64(coords).reshape(-1, 3)
        out = np.zeros(3, dtype=np.float64)
        nb = _i32(neighbors)
        L.ref_num_gradient_single_atom(self.handle, int(index), coords.shape[0],
                                       _i32(species), nb, nb.shape[0], coords.ravel(),
                                       _f64(dE).ravel(), out)
        return out
