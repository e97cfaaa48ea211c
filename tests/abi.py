"""ctypes binding of include/libdescriptor_b200.h for the tests.

The GPU parity tests call the library through this C ABI (the drop-in
boundary), exactly as a foreign caller would.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "libdescriptor_b200", "_lib", "libldb200.so")
HEADER = os.path.join(ROOT, "include", "libdescriptor_b200.h")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def header_functions():
    """Names of every function the public header declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ld_[a-z0-9_]+)\s*\(", txt)))


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class AbiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Abi:
    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(LIB)
            L.ld_error_message.restype = C.c_char_p
            L.ld_launch_count.restype = C.c_longlong
            L.ld_alloc_count.restype = C.c_longlong
            L.ld_fail_next_allocation.argtypes = [C.c_int]
            L.ld_debug_fill_scratch.argtypes = [C.c_int]
            L.ld_debug_bulk_wait_timeout.argtypes = [C.c_longlong]
            L.ld_create_symmetry_functions.argtypes = [C.POINTER(C.c_void_p), C.c_int, _dp, C.c_int,
                                                       _ip, _ip, _dp]
            L.ld_create_bispectrum.argtypes = [C.POINTER(C.c_void_p), C.c_double, C.c_int, C.c_int,
                                               C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp]
            L.ld_create_from_file.argtypes = [C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
            L.ld_describe_parameter_file.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_size_t,
                                                     C.POINTER(C.c_size_t)]
            L.ld_destroy.argtypes = [C.c_void_p]
            L.ld_width.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
            L.ld_kind.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
            L.ld_compute.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _ip, _dp, _dp]
            L.ld_gradient.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _ip, _dp, _dp, _dp,
                                      C.c_void_p]
            L.ld_compute_batch.argtypes = [C.c_void_p, C.c_int, _ip, _ip, C.c_int, _ip, _ip, _ip, _dp,
                                           _dp]
            L.ld_gradient_batch.argtypes = [C.c_void_p, C.c_int, _ip, _ip, C.c_int, _ip, _ip, _ip, _dp,
                                            _dp, _dp, C.c_void_p]
            L.ld_compute_single_atom.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, C.c_int, _dp,
                                                 _dp]
            L.ld_gradient_single_atom.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, C.c_int, _dp,
                                                  _dp, _dp, C.c_void_p]
            L.ld_jacobian.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _ip, _dp, _dp]
            L.ld_create_paddings.argtypes = [C.c_double, _dp, _ip, _dp, _ip, C.c_int,
                                             C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p]
            L.ld_build_neighbor_list.argtypes = [_dp, C.c_int, C.c_double, _ip, C.c_int, _ip, C.c_void_p,
                                                 C.POINTER(C.c_longlong)]
            L.ld_compute_dev.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
            L.ld_gradient_dev.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
            L.ld_sync_status.argtypes = [C.c_void_p, C.c_void_p]
            L.ld_neighbor_offsets_dev.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.POINTER(C.c_int), C.c_void_p]
            L.ld_compute_rows_dev.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_size_t, C.c_void_p]
            L.ld_gradient_rows_dev.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                               C.c_void_p]
            L.ld_rows_work_bytes.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_size_t)]
            L.ld_stage_bytes.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_int, C.POINTER(C.c_size_t)]
            L.ld_stage_request.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_int, C.c_int,
                                           C.c_longlong, _dp, _ip, _ip, _ip, _ip, _dp, C.c_void_p, C.c_size_t]
            L.ld_stage_request.argtypes += [C.c_void_p] * 9
            L.ld_stage_pack.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_int, C.c_int,
                                        C.c_longlong, _dp, _ip, _ip, _ip, _ip, _dp, C.c_void_p, C.c_size_t]
            L.ld_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.ld_get_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
            cls._lib = L
        return cls._lib

    @classmethod
    def check(cls, rc):
        if rc != 0:
            raise AbiError(rc, cls.lib().ld_error_message().decode())

    @classmethod
    def create_sf(cls, ns, cutoff_matrix, types, sizes, params):
        h = C.c_void_p()
        codes = _i([int(t.lstrip("g")) for t in types])
        cls.check(cls.lib().ld_create_symmetry_functions(C.byref(h), int(ns), _f(cutoff_matrix).ravel(),
                                                         len(codes), codes, _i(sizes), _f(params)))
        return Handle(h)

    @classmethod
    def create_bs(cls, rfac0, twojmax, style, rmin0, switch_flag, bzero_flag, ns, cutoff_matrix,
                  weights):
        h = C.c_void_p()
        cls.check(cls.lib().ld_create_bispectrum(C.byref(h), float(rfac0), int(twojmax), int(style), 0,
                                                 float(rmin0), int(switch_flag), int(bzero_flag),
                                                 int(ns), _f(cutoff_matrix).ravel(), _f(weights)))
        return Handle(h)

    @classmethod
    def create_from_file(cls, path, kind):
        h = C.c_void_p()
        cls.check(cls.lib().ld_create_from_file(C.byref(h), path.encode(), int(kind)))
        return Handle(h)


def describe_parameter_file(path, kind):
    """ld_describe_parameter_file as a dict of numpy arrays / scalars."""
    L = Abi.lib()
    n = C.c_size_t(0)
    Abi.check(L.ld_describe_parameter_file(path.encode(), int(kind), None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value)
    Abi.check(L.ld_describe_parameter_file(path.encode(), int(kind), buf, n.value, C.byref(n)))
    out = {}
    for line in buf.value.decode().splitlines():
        key, _, val = line.partition(" = ")
        toks = val.split()
        if key == "species":
            out[key] = toks
        elif key in ("kind", "n_species", "twojmax", "diagonalstyle", "switch_flag", "bzero_flag"):
            out[key] = int(toks[0])
        elif key in ("type_codes", "sizes"):
            out[key] = np.array([int(t) for t in toks], dtype=np.int32)
        elif key in ("rfac0", "rmin0"):
            out[key] = float(toks[0])
        else:
            out[key] = np.array([float(t) for t in toks])
    return out


class Handle:
    def __init__(self, h):
        self.h = h
        w = C.c_int()
        Abi.check(Abi.lib().ld_width(h, C.byref(w)))
        self.width = w.value

    def __del__(self):
        try:
            Abi.lib().ld_destroy(self.h)
        except Exception:
            pass

    def compute(self, n_atoms, species, nbl, counts, coords):
        coords = _f(coords).reshape(-1, 3)
        out = np.zeros((n_atoms, self.width))
        Abi.check(Abi.lib().ld_compute(self.h, int(n_atoms), coords.shape[0], _i(species), _i(nbl),
                                       _i(counts), coords.ravel(), out))
        return out

    def gradient(self, n_atoms, species, nbl, counts, coords, dE, want_desc=False):
        coords = _f(coords).reshape(-1, 3)
        dc = np.zeros(coords.shape)
        desc = np.zeros((n_atoms, self.width)) if want_desc else None
        Abi.check(Abi.lib().ld_gradient(self.h, int(n_atoms), coords.shape[0], _i(species), _i(nbl),
                                        _i(counts), coords.ravel(), _f(dE).ravel(), dc.ravel(),
                                        desc.ctypes.data if want_desc else None))
        return (dc, desc) if want_desc else dc

    def compute_batch(self, n_atoms, config_ptr, species, nbl, counts, coords):
        coords = _f(coords).reshape(-1, 3)
        n_atoms = _i(n_atoms)
        out = np.zeros((int(n_atoms.sum()), self.width))
        Abi.check(Abi.lib().ld_compute_batch(self.h, len(n_atoms), n_atoms, _i(config_ptr),
                                             coords.shape[0], _i(species), _i(nbl), _i(counts),
                                             coords.ravel(), out))
        return out

    def gradient_batch(self, n_atoms, config_ptr, species, nbl, counts, coords, dE):
        coords = _f(coords).reshape(-1, 3)
        n_atoms = _i(n_atoms)
        dc = np.zeros(coords.shape)
        Abi.check(Abi.lib().ld_gradient_batch(self.h, len(n_atoms), n_atoms, _i(config_ptr),
                                              coords.shape[0], _i(species), _i(nbl), _i(counts),
                                              coords.ravel(), _f(dE).ravel(), dc.ravel(), None))
        return dc

    def compute_single_atom(self, index, species, neighbors, coords):
        coords = _f(coords).reshape(-1, 3)
        out = np.zeros(self.width)
        nb = _i(neighbors)
        Abi.check(Abi.lib().ld_compute_single_atom(self.h, int(index), coords.shape[0], _i(species), nb,
                                                   nb.shape[0], coords.ravel(), out))
        return out

    def gradient_single_atom(self, index, species, neighbors, coords, dE):
        coords = _f(coords).reshape(-1, 3)
        dc = np.zeros(coords.shape)
        nb = _i(neighbors)
        Abi.check(Abi.lib().ld_gradient_single_atom(self.h, int(index), coords.shape[0], _i(species), nb,
                                                    nb.shape[0], coords.ravel(), _f(dE).ravel(),
                                                    dc.ravel(), None))
        return dc

    def jacobian(self, n_atoms, species, nbl, counts, coords):
        coords = _f(coords).reshape(-1, 3)
        J = np.zeros((self.width * n_atoms, coords.size))
        Abi.check(Abi.lib().ld_jacobian(self.h, int(n_atoms), coords.shape[0], _i(species), _i(nbl),
                                        _i(counts), coords.ravel(), J))
        return J

    def set_tuning(self, key, value):
        Abi.check(Abi.lib().ld_set_tuning(self.h, int(key), int(value)))

    def get_tuning(self, key):
        v = C.c_int()
        Abi.check(Abi.lib().ld_get_tuning(self.h, int(key), C.byref(v)))
        return v.value

    def rows_work_bytes(self, n_rows, vjp):
        b = C.c_size_t()
        Abi.check(Abi.lib().ld_rows_work_bytes(self.h, int(n_rows), int(vjp), C.byref(b)))
        return b.value
