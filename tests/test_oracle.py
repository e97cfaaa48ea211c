"""CPU: the oracle (checker) against the reference's own outputs.

* golden fixtures (reference C++ outputs committed in tests/golden/);
* the reference's own finite-difference self-gradient (fd_* in fixtures);
* live reference library (oracle/_ref, when it was built here) on fresh
  seeds, batch layout included;
* the oracle's analytic VJP against its own 8th-order finite differences.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from helpers import kind_of, oracle_for, rel_err


@pytest.mark.parametrize("name", golden_names())
def test_oracle_forward_matches_reference_golden(oracle_mod, name):
    g = load_golden(name)
    o = oracle_for(name, g)
    desc = o.run(int(g["n_atoms"]), g["species"], g["nbl"], g["counts"], g["coords"], n_threads=2)
    assert desc.shape == g["desc"].shape
    # same algorithm, same operation order, same compiler: agreement to the last bits
    assert rel_err(desc, g["desc"]) <= 1e-14, name


@pytest.mark.parametrize("name", [n for n in golden_names() if "fd_index" in load_golden(n)])
def test_oracle_vjp_matches_reference_fd(oracle_mod, name):
    g = load_golden(name)
    o = oracle_for(name, g)
    n = int(g["n_atoms"])
    for k, i in enumerate(g["fd_index"]):
        dE = np.zeros((n, o.width))
        dE[i] = g["fd_dE"][k]
        _, dc = o.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE, n_threads=1)
        # the reference's stencil differentiates desc_i w.r.t. r_i only
        np.testing.assert_allclose(dc[i], g["fd_grad"][k], rtol=2e-7, atol=1e-9 * np.abs(g["fd_grad"][k]).max())


@pytest.mark.parametrize("name", ["sf24_diamond64", "sf_mixed_packing48", "bs_j6_style3_sw1_packing64",
                                  "bs_j4_style0_sw1_packing64", "bs_j6_rmin_diamond64",
                                  "bs_j6_cutmatrix_packing64"])
def test_oracle_vjp_matches_finite_differences(oracle_mod, name):
    g = load_golden(name)
    o = oracle_for(name, g)
    n = int(g["n_atoms"])
    rng = np.random.default_rng(11)
    dE = rng.normal(size=(n, o.width))
    _, dc = o.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE, n_threads=4)
    idx = rng.choice(g["coords"].size, 10, replace=False)
    # central differences with h = 1e-5 A (the cutoff functions are only C1
    # at rc, so a wide high-order stencil is inexact near the cutoff)
    fd = o.fd_vjp(n, g["species"], g["nbl"], g["counts"], g["coords"], dE, idx, step=1e-5, n_threads=4)
    scale = np.abs(dc).max()
    np.testing.assert_allclose(dc.ravel()[idx], fd, rtol=0, atol=1e-6 * scale)


def _fresh_inputs(seed, n=40, ns=2, rc=5.0):
    from oracle import Reference

    rng = np.random.default_rng(seed)
    side = (n / 0.05) ** (1 / 3)
    x = rng.uniform(0, side, (n, 3))
    # push apart pairs that are too close so the neighbour builder accepts them
    sp = (np.arange(n) % ns).astype(np.int32)
    pc, ps, pi = Reference.create_paddings(rc, np.eye(3) * side, [1, 1, 1], x, sp)
    allx = np.concatenate([x, pc])
    alls = np.concatenate([sp, ps]).astype(np.int32)
    need = np.zeros(len(allx), np.int32)
    need[:n] = 1
    counts, nbl = Reference.neighbor_list(allx, rc, need, n)
    return n, allx, alls, counts, nbl


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_live_reference(oracle_mod, seed):
    from oracle import OracleDescriptor, Reference, ReferenceDescriptor

    if not Reference.available():
        pytest.skip("reference library not built here")
    n, x, s, counts, nbl = _fresh_inputs(seed)
    cm = np.full((2, 2), 5.0)
    from conftest import sf24

    t, sz, p = sf24()
    for ref, ora in [
        (ReferenceDescriptor.symmetry_functions(2, cm, t, sz, p),
         OracleDescriptor.symmetry_functions(2, cm, t, sz, p)),
        (ReferenceDescriptor.bispectrum(0.99363, 8, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5]),
         OracleDescriptor.bispectrum(0.99363, 8, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5])),
        (ReferenceDescriptor.bispectrum(0.9, 5, 3, 0.2, 1, 0, 2, cm, [0.7, 1.3]),
         OracleDescriptor.bispectrum(0.9, 5, 3, 0.2, 1, 0, 2, cm, [0.7, 1.3])),
    ]:
        a = ref.compute(n, s, nbl, counts, x, n_threads=2)
        b = ora.run(n, s, nbl, counts, x, n_threads=2)
        assert rel_err(b, a) <= 1e-14


def test_oracle_batch_layout_matches_reference(oracle_mod):
    from oracle import OracleDescriptor, Reference, ReferenceDescriptor

    if not Reference.available():
        pytest.skip("reference library not built here")
    parts = [_fresh_inputs(s, n=20 + 7 * s) for s in (3, 4, 5)]
    xs, ss, cs, ns_, n_atoms, ptr = [], [], [], [], [], []
    base = 0
    for n, x, s, c, nb in parts:
        n_atoms.append(n)
        ptr.append(base)
        xs.append(x)
        ss.append(s)
        cs.append(c)
        ns_.append(nb + base)
        base += len(x)
    x = np.concatenate(xs)
    s = np.concatenate(ss).astype(np.int32)
    c = np.concatenate(cs).astype(np.int32)
    nb = np.concatenate(ns_).astype(np.int32)
    cm = np.full((2, 2), 5.0)
    ref = ReferenceDescriptor.bispectrum(0.99363, 6, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5])
    ora = OracleDescriptor.bispectrum(0.99363, 6, 3, 0.0, 1, 0, 2, cm, [1.0, 0.5])
    a = ref.compute(n_atoms, s, nb, c, x, n_configs=3, config_ptr=ptr)
    b = ora.run(n_atoms, s, nb, c, x, n_configs=3, config_ptr=ptr)
    assert rel_err(b, a) <= 1e-14
    # per-configuration results equal the batch rows
    r0 = 0
    for (n, xx, sp, cc, nbb) in parts:
        one = ora.run(n, sp, nbb, cc, xx)
        np.testing.assert_array_equal(one, b[r0:r0 + n])
        r0 += n


def test_oracle_invariances(oracle_mod):
    """Rotation / translation invariance of the forward, zero net gradient."""
    g = load_golden("bs_j6_style3_sw1_packing64")
    o = oracle_for("bs_j6_style3_sw1_packing64", g)
    n = int(g["n_atoms"])
    x = g["coords"]
    d0 = o.run(n, g["species"], g["nbl"], g["counts"], x)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    d1 = o.run(n, g["species"], g["nbl"], g["counts"], x @ R.T + 3.3)
    assert rel_err(d1, d0) <= 1e-9
    dE = np.random.default_rng(0).normal(size=d0.shape)
    _, dc = o.run(n, g["species"], g["nbl"], g["counts"], x, dE=dE)
    assert np.abs(dc.sum(axis=0)).max() <= 1e-10 * np.abs(dc).max() * len(dc)
