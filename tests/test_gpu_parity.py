"""GPU parity: the CUDA kernels, called through the C ABI, against the
reference's outputs (golden fixtures) and the oracle.

Bars (see helpers.py for the exact element rule): descriptors 1e-10
relative, gradients 1e-8 relative.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from helpers import DESC_RTOL, GRAD_RTOL, assert_close, gpu_for, kind_of, oracle_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names())
def test_forward_matches_reference(name):
    g = load_golden(name)
    h = gpu_for(name, g)
    desc = h.compute(int(g["n_atoms"]), g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(desc, g["desc"], DESC_RTOL, name)


@pytest.mark.parametrize("name", golden_names())
def test_gradient_matches_oracle(oracle_mod, name):
    g = load_golden(name)
    h = gpu_for(name, g)
    o = oracle_for(name, g)
    n = int(g["n_atoms"])
    dE = np.random.default_rng(3).normal(size=(n, h.width))
    dc, desc = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE, want_desc=True)
    _, dco = o.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE)
    assert_close(dc, dco, GRAD_RTOL, name + " grad")
    assert_close(desc, g["desc"], DESC_RTOL, name + " desc of the fused pass")


@pytest.mark.parametrize("name", [n for n in golden_names() if n.startswith("sf")])
def test_table_driven_sf_kernel_matches(oracle_mod, name):
    """The table-driven symmetry-function kernel (any parameter set; chosen
    when a set does not factor into a (lambda, zeta) x eta grid), forced on
    the symmetry-function goldens: forward vs the reference, fused VJP vs the
    oracle."""
    g = load_golden(name)
    h = gpu_for(name, g)
    h.set_tuning(4, 1)
    o = oracle_for(name, g)
    n = int(g["n_atoms"])
    desc = h.compute(n, g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(desc, g["desc"], DESC_RTOL, name + " table-driven desc")
    dE = np.random.default_rng(4).normal(size=(n, h.width))
    dc, desc2 = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE, want_desc=True)
    _, dco = o.run(n, g["species"], g["nbl"], g["counts"], g["coords"], dE=dE)
    assert_close(dc, dco, GRAD_RTOL, name + " table-driven grad")
    assert_close(desc2, g["desc"], DESC_RTOL, name + " table-driven desc of the fused pass")


@pytest.mark.parametrize("name", [n for n in golden_names() if load_golden(n).get("fd_index") is not None
                                  and len(load_golden(n)["fd_index"])])
def test_gradient_matches_reference_fd(name):
    """The reference's own 8th-order finite-difference self-gradient."""
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    for k, i in enumerate(g["fd_index"]):
        dE = np.zeros((n, h.width))
        dE[i] = g["fd_dE"][k]
        dc = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], dE)
        np.testing.assert_allclose(dc[i], g["fd_grad"][k], rtol=2e-7,
                                   atol=1e-9 * np.abs(g["fd_grad"][k]).max())


def _three_configs():
    from libdescriptor_b200 import workloads as W

    cfgs = []
    for s, (n1, n2, n3) in enumerate([(1, 1, 2), (2, 1, 1), (1, 2, 2)]):
        x, cell = W.diamond_cell(n1, n2, n3, jitter=0.1, strain=0.03, seed=10 + s)
        sp = (np.arange(len(x)) % 2).astype(np.int32)
        cfgs.append(W.prepare(x, cell, sp, 5.0))
    return cfgs


@pytest.mark.parametrize("kind", ["sf", "bs"])
def test_batch_equals_per_configuration(kind):
    from libdescriptor_b200 import workloads as W
    from abi import Abi

    cfgs = _three_configs()
    b = W.concat(cfgs)
    if kind == "sf":
        t, sz, p = W.sf24_params()
        h = Abi.create_sf(2, np.full((2, 2), 5.0), t, sz, p)
    else:
        h = Abi.create_bs(0.99363, 6, 3, 0.0, 1, 0, 2, np.full((2, 2), 5.0), [1.0, 0.5])
    desc = h.compute_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords)
    dE = np.random.default_rng(5).normal(size=desc.shape)
    dc = h.gradient_batch(b.n_atoms, b.config_ptr, b.species, b.nbl, b.counts, b.coords, dE)
    r0, x0 = 0, 0
    for c in cfgs:
        one = h.compute(c.n_atoms, c.species, c.nbl, c.counts, c.coords)
        assert_close(desc[r0:r0 + c.n_atoms], one, 1e-13, "batch desc")
        g1 = h.gradient(c.n_atoms, c.species, c.nbl, c.counts, c.coords, dE[r0:r0 + c.n_atoms])
        assert_close(dc[x0:x0 + c.n_total], g1, 1e-11, "batch grad")
        r0 += c.n_atoms
        x0 += c.n_total


@pytest.mark.parametrize("name", ["sf24_diamond64", "bs_j8_style3_sw1_packing64"])
def test_single_atom_and_jacobian(oracle_mod, name):
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    off = np.concatenate([[0], np.cumsum(g["counts"])])
    for i in (0, 5, n - 1):
        nb = g["nbl"][off[i]:off[i + 1]]
        d = h.compute_single_atom(i, g["species"], nb, g["coords"])
        assert_close(d[None], g["desc"][i][None], DESC_RTOL, "single atom")
        dE = np.random.default_rng(i).normal(size=h.width)
        dc = h.gradient_single_atom(i, g["species"], nb, g["coords"], dE)
        full = np.zeros((n, h.width))
        full[i] = dE
        want = h.gradient(n, g["species"], g["nbl"], g["counts"], g["coords"], full)
        assert_close(dc, want, 1e-12, "single-atom gradient")
    # Jacobian rows are VJPs with one-hot upstream vectors
    m = 6
    J = h.jacobian(m, g["species"], g["nbl"], g["counts"][:m], g["coords"])
    assert J.shape == (m * h.width, g["coords"].size)
    rng = np.random.default_rng(9)
    dE = rng.normal(size=(m, h.width))
    want = h.gradient(m, g["species"], g["nbl"], g["counts"][:m], g["coords"], dE)
    assert_close((dE.ravel() @ J).reshape(-1, 3), want, 1e-11, "jacobian")


def test_edge_cases():
    """Empty configurations, centres without neighbours, out-of-range indices."""
    from abi import Abi, AbiError

    for h in (Abi.create_sf(1, np.full((1, 1), 5.0), ["g2", "g4"], [1, 2, 1, 3], [0.1, 0.0, 1.0, 1.0, 0.01]),
              Abi.create_bs(0.99363, 4, 3, 0.0, 1, 0, 1, np.full((1, 1), 5.0), [1.0])):
        x = np.array([[0.0, 0.0, 0.0], [20.0, 0.0, 0.0]])
        sp = np.zeros(2, np.int32)
        out = h.compute(0, sp, np.zeros(0, np.int32), np.zeros(0, np.int32), x)
        assert out.shape == (0, h.width)
        d = h.compute(2, sp, np.zeros(0, np.int32), np.zeros(2, np.int32), x)
        assert np.all(np.isfinite(d))
        dc = h.gradient(2, sp, np.zeros(0, np.int32), np.zeros(2, np.int32), x, np.ones((2, h.width)))
        assert np.all(dc == 0)
        with pytest.raises(AbiError):
            h.compute(1, sp, np.array([5], np.int32), np.array([1], np.int32), x)


def test_device_api_capacity_error_is_raised():
    import torch

    import libdescriptor_b200 as lds

    g = load_golden("sf24_diamond64")
    from libdescriptor_b200.workloads import sf24_params

    t, sz, p = sf24_params()
    ds = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["Si"], "cos", 5.0,
                                            t, sz, p)
    dev = torch.device("cuda")
    sp = torch.as_tensor(g["species"], device=dev)
    nbl = torch.as_tensor(g["nbl"], device=dev)
    cnt = torch.as_tensor(g["counts"], device=dev)
    x = torch.as_tensor(g["coords"], device=dev)
    off = torch.empty(len(g["counts"]) + 1, dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    mx = lds._ext._neighbor_offsets_dev(ds, len(g["counts"]), cnt.data_ptr(), off.data_ptr(), True, s)
    assert mx == int(g["counts"].max())
    desc = torch.empty((len(g["counts"]), ds.width), dtype=torch.float64, device=dev)
    lds._ext._compute_dev(ds, len(g["counts"]), 0, sp.data_ptr(), nbl.data_ptr(), off.data_ptr(), mx - 3,
                          x.data_ptr(), desc.data_ptr(), s)
    with pytest.raises(RuntimeError, match="max_neigh"):
        lds._ext._sync_status(ds, s)
    assert torch.isnan(desc).any()
    lds._ext._compute_dev(ds, len(g["counts"]), 0, sp.data_ptr(), nbl.data_ptr(), off.data_ptr(), mx,
                          x.data_ptr(), desc.data_ptr(), s)
    lds._ext._sync_status(ds, s)
    assert_close(desc.cpu().numpy(), g["desc"], DESC_RTOL, "device api")


@pytest.mark.parametrize("name", ["sf24_diamond64", "bs_j6_style3_sw1_packing64"])
def test_invariances(name):
    g = load_golden(name)
    h = gpu_for(name, g)
    n = int(g["n_atoms"])
    x = g["coords"]
    d0 = h.compute(n, g["species"], g["nbl"], g["counts"], x)
    th = 0.9
    R = np.array([[1, 0, 0], [0, np.cos(th), -np.sin(th)], [0, np.sin(th), np.cos(th)]])
    d1 = h.compute(n, g["species"], g["nbl"], g["counts"], x @ R.T - 1.7)
    assert_close(d1, d0, 1e-9, "rotation/translation")
    # permuting each neighbour list leaves the descriptors unchanged
    off = np.concatenate([[0], np.cumsum(g["counts"])])
    nbl = g["nbl"].copy()
    rng = np.random.default_rng(2)
    for i in range(n):
        rng.shuffle(nbl[off[i]:off[i + 1]])
    d2 = h.compute(n, g["species"], nbl, g["counts"], x)
    assert_close(d2, d0, 1e-12, "neighbour permutation")
    dE = np.random.default_rng(0).normal(size=d0.shape)
    dc = h.gradient(n, g["species"], g["nbl"], g["counts"], x, dE)
    assert np.abs(dc.sum(axis=0)).max() <= 1e-10 * np.abs(dc).max() * len(dc)


def test_reference_python_api_through_the_module():
    """The reference-shaped pybind module (compute / gradient / NeighList)."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200.workloads import sf24_params

    g = load_golden("sf24_diamond64")
    t, sz, p = sf24_params()
    ds = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, ["Si"], "cos", 5.0,
                                            t, sz, p)
    assert ds.width == 24
    n = int(g["n_atoms"])
    desc = lds.compute(ds, n, g["species"], g["nbl"], g["counts"], g["coords"])
    assert_close(desc, g["desc"], DESC_RTOL, "module compute")
    dE = np.ones((n, 24))
    grad = lds.gradient(ds, n, g["species"], g["nbl"], g["counts"], g["coords"], desc, dE)
    assert grad.shape == g["coords"].shape
    bs = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 8, 3, 0, 0.0, 1, 0,
                                            5.0, ["Si", "Ge"], [1.0, 0.5])
    assert bs.width == 55
    gb = load_golden("bs_j8_style3_sw1_packing64")
    d = lds.compute(bs, 64, gb["species"], gb["nbl"], gb["counts"], gb["coords"])
    assert_close(d, gb["desc"], DESC_RTOL, "module bispectrum")
    off = np.concatenate([[0], np.cumsum(gb["counts"])])
    one = ds.compute(3, g["species"], g["nbl"][np.concatenate([[0], np.cumsum(g["counts"])])[3]:
                                              np.concatenate([[0], np.cumsum(g["counts"])])[4]], g["coords"])
    assert_close(one[None], g["desc"][3][None], DESC_RTOL, "DescriptorKind.compute")
    ng = lds.num_gradient_single_atom(bs, 0, gb["species"], gb["nbl"][off[0]:off[1]], gb["coords"],
                                      np.ones(55))
    assert ng.shape == (3,)
    with pytest.raises(ValueError):
        lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SOAP, 4, 3, 4.0, ["Si"], "polynomial", 0.1)
