"""GPU: the device neighbour builder gives the host builder's ghosts (same
order and coordinates, bit for bit) and lists (same order), and its output
feeds the descriptor kernels directly."""
import numpy as np
import pytest

from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _cases():
    from libdescriptor_b200 import workloads as W

    out = []
    for n, s in ((1, 3), (2, 4), (3, 5)):
        x, cell = W.diamond_cell(n, 1 + n % 2, 2, jitter=0.1, strain=0.03, seed=s)
        out.append((f"diamond{n}", x, cell, np.zeros(len(x), np.int32), (1, 1, 1)))
    for n, s in ((16, 1), (300, 2), (3000, 3)):
        x, cell, sp = W.random_packing(n, density=0.05, dmin=2.0, n_species=2, seed=s)
        out.append((f"packing{n}", x, cell, sp, (1, 1, 1)))
    x, cell, sp = W.random_packing(500, density=0.05, dmin=2.0, n_species=2, seed=9)
    out.append(("packing500_pbc101", x, cell, sp, (1, 0, 1)))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_builder_matches_host(case):
    from libdescriptor_b200 import workloads as W

    name, x, cell, sp, pbc = case
    h = W.prepare(x, cell, sp, 5.0, pbc=pbc)
    d = W.prepare_dev(x, cell, sp, 5.0, pbc=pbc)
    assert d.n_total == h.n_total
    np.testing.assert_array_equal(d.coords.cpu().numpy(), h.coords)
    np.testing.assert_array_equal(d.species.cpu().numpy(), h.species)
    np.testing.assert_array_equal(d.image.cpu().numpy(), h.image)
    np.testing.assert_array_equal(d.counts.cpu().numpy(), h.counts)
    np.testing.assert_array_equal(d.nbl.cpu().numpy(), h.nbl)
    off = np.concatenate([[0], np.cumsum(h.counts)])
    np.testing.assert_array_equal(d.off.cpu().numpy(), off)
    assert d.max_neigh == max(int(h.counts.max()), 1)


def test_device_pipeline_descriptors_and_forces():
    """coords + cell -> device ghosts and lists -> fused desc + VJP with the
    ghost fold inside the kernel, against the host-prepared call."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W

    x, cell, sp = W.random_packing(800, density=0.05, dmin=2.0, n_species=2, seed=4)
    k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 6, 3, 0, 0.0, 1, 0, 5.0,
                                           ["A", "B"], [1.0, 0.5])
    h = W.prepare(x, cell, sp, 5.0)
    dE = np.random.default_rng(1).normal(size=(h.n_atoms, k.width))
    desc_ref, g = lds.compute_and_gradient(k, h.n_atoms, h.species, h.nbl, h.counts, h.coords, dE)
    forces_ref = W.fold(g, h.n_atoms, h.image)
    d = W.prepare_dev(x, cell, sp, 5.0)
    dEd = torch.as_tensor(dE, device="cuda")
    desc = torch.empty((d.n_atoms, k.width), dtype=torch.float64, device="cuda")
    dc = torch.zeros((d.n_atoms, 3), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lds._ext._gradient_dev(k, d.n_atoms, 0, d.species.data_ptr(), d.nbl.data_ptr(), d.off.data_ptr(), d.max_neigh,
                           d.coords.data_ptr(), dEd.data_ptr(), dc.data_ptr(), desc.data_ptr(), d.image.data_ptr(), s)
    lds._ext._sync_status(k, s)
    assert_close(desc.cpu().numpy(), desc_ref, DESC_RTOL, "device-prepared desc")
    assert_close(dc.cpu().numpy(), forces_ref, GRAD_RTOL, "device-prepared folded forces")


def test_device_builder_errors():
    from libdescriptor_b200 import workloads as W

    x, cell, sp = W.random_packing(50, density=0.05, dmin=2.0, n_species=2, seed=6)
    with pytest.raises(ValueError):
        W.prepare_dev(x, np.zeros((3, 3)), sp, 5.0)          # singular cell
    x2 = x.copy()
    x2[1] = x2[0]                                             # two atoms on one site
    with pytest.raises(ValueError):
        W.prepare_dev(x2, cell, sp, 5.0)
