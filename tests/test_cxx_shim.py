"""The C++ driver API (include/cxx/Descriptors.hpp + libldb200_cxx.so).

tests/cxx/call_site.cpp is a caller written against the reference's header
(include/Descriptors.hpp:19-271): DescriptorKind::initDescriptor overloads
and the free functions compute, compute_batch, compute_single_atom,
gradient, gradient_batch, gradient_single_atom, num_gradient_single_atom
and jacobian.  It compiles against this library's header and links with the
shim unchanged (CPU test); on the GPU its results match the reference's
goldens and the oracle, with the reference's buffer rules (symmetry
functions added into desc, the bispectrum overwritten, gradients added into
caller-zeroed buffers).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, sf24

LIBDIR = os.path.join(ROOT, "libdescriptor_b200", "_lib")
SRC = os.path.join(ROOT, "tests", "cxx", "call_site.cpp")


def _build(tmp):
    exe = os.path.join(str(tmp), "call_site")
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include", "cxx"), SRC,
                    "-L" + LIBDIR, "-lldb200_cxx", "-Wl,-rpath," + LIBDIR, "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def _case(tmp, name, g, spec, index, dE):
    d = os.path.join(str(tmp), name)
    os.makedirs(d, exist_ok=True)
    n, nt = int(g["n_atoms"]), int(g["coords"].shape[0])
    with open(os.path.join(d, "meta.txt"), "w") as f:
        f.write(f"{spec[0]} {n} {nt} {int(g['nbl'].size)} {index}\n")
        f.write(" ".join(str(v) for v in spec[1:]) + "\n")
    for key, dt in (("species", np.int32), ("nbl", np.int32), ("counts", np.int32)):
        np.ascontiguousarray(g[key], dtype=dt).tofile(os.path.join(d, key + ".i32"))
    np.ascontiguousarray(g["coords"], dtype=np.float64).tofile(os.path.join(d, "coords.f64"))
    np.ascontiguousarray(dE, dtype=np.float64).tofile(os.path.join(d, "dE.f64"))
    return d


def _sf_spec(ns):
    t, sz, p = sf24()
    names = [f"S{k}" for k in range(ns)]
    return ["sf", ns] + names + [5.0, len(t)] + list(t) + list(sz) + [len(p)] + list(p)


def _bs_spec(g, ns):
    names = [f"S{k}" for k in range(ns)]
    return (["bs", float(g["rfac0"]), int(g["twojmax"]), int(g["style"]), float(g["rmin0"]), int(g["switch_flag"]),
             0, float(g["cutoff"]), ns] + names + [float(w) for w in g["weights"]])


def test_call_site_compiles_and_links_against_the_shim(tmp_path):
    """The reference-shaped call site builds with no edits; without a device
    its first call throws (no CPU fallback)."""
    exe = _build(tmp_path)
    g = load_golden("sf24_diamond64")
    d = _case(tmp_path, "sf", g, _sf_spec(1), 0, np.zeros((64, 24)))
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present (the GPU test runs the program)")
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sf24_diamond64", "bs_j8_style3_sw1_packing64", "bs_j6_style3_sw1_packing64"])
def test_call_site_results_match_reference(tmp_path, name):
    from helpers import oracle_for

    exe = _build(tmp_path)
    g = load_golden(name)
    ns = int(np.max(g["species"])) + 1
    is_sf = name.startswith("sf")
    spec = _sf_spec(ns) if is_sf else _bs_spec(g, ns)
    n, nt = int(g["n_atoms"]), int(g["coords"].shape[0])
    W = g["desc"].shape[1]
    index = int(g["fd_index"][0])
    dE = np.random.default_rng(8).normal(size=(n, W))
    dE[index] = g["fd_dE"][0]
    d = _case(tmp_path, "case", g, spec, index, dE)
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def out(key, shape):
        return np.fromfile(os.path.join(d, key + ".f64")).reshape(shape)

    desc = out("desc", (n, W))
    assert_close(desc, g["desc"], DESC_RTOL, f"{name}: Descriptor::compute vs the reference")
    twice = out("desc_twice", (n, W))
    assert_close(twice, (2.0 if is_sf else 1.0) * g["desc"], DESC_RTOL, f"{name}: accumulate / overwrite rule")
    assert_close(out("desc_batch", (n, W)), g["desc"], DESC_RTOL, f"{name}: compute_batch")
    ora = oracle_for(name, g)
    d_ora, g_ora = ora.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE)
    assert_close(out("grad", (nt, 3)), g_ora, GRAD_RTOL, f"{name}: Descriptor::gradient vs the oracle")
    assert_close(out("desc_grad", (n, W)), g["desc"], DESC_RTOL, f"{name}: gradient's descriptors")
    assert_close(out("grad_batch", (nt, 3)), g_ora, GRAD_RTOL, f"{name}: gradient_batch")
    assert_close(out("desc_single", (1, W)), g["desc"][index:index + 1], DESC_RTOL, f"{name}: compute_single_atom")
    one = np.zeros_like(dE)
    one[index] = dE[index]
    _, g_one = ora.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=one)
    assert_close(out("grad_single", (nt, 3)), g_one, GRAD_RTOL, f"{name}: gradient_single_atom")
    # the reference's own finite-difference self-gradient of that centre
    num = out("num_grad_single", (3,))
    assert np.max(np.abs(num - g["fd_grad"][0])) <= 1e-8 * max(1.0, np.abs(g["fd_grad"][0]).max())
    J = out("jacobian", (n * W, 3 * nt))
    assert_close((dE.ravel() @ J).reshape(nt, 3), g_ora, GRAD_RTOL, f"{name}: jacobian^T dE")


@pytest.mark.gpu
def test_call_site_with_a_parameter_file(tmp_path):
    exe = _build(tmp_path)
    g = load_golden("sf24_diamond64")
    t, sz, p = sf24()
    path = os.path.join(str(tmp_path), "sf24.txt")
    with open(path, "w") as f:
        f.write("cos\n1\nSi Si 5.0\n1\n")                 # one type: no shared-vector effect
        f.write(f"g2 {sz[0]} {sz[1]}\n")
        for k in range(sz[0]):
            f.write(f"{p[2 * k]} {p[2 * k + 1]}\n")
        f.write("false\n8\n")
    n = int(g["n_atoms"])
    d = _case(tmp_path, "file", g, ["file", 0, path], 0, np.ones((n, 8)))
    r = subprocess.run([exe, d], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    desc = np.fromfile(os.path.join(d, "desc.f64")).reshape(n, 8)
    assert_close(desc, g["desc"][:, :8], DESC_RTOL, "g2 block from a parameter file")
