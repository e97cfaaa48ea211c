"""CPU: the C-ABI library and the host-side logic (no kernel launches).

* the shared library loads and exports every function the public header
  declares; the Python module exposes the reference's API names;
* the neighbour builder (ghost padding + cell list) reproduces the
  reference's own builder exactly, on orthogonal, strained, small
  (multi-image) and partly periodic cells, and agrees with brute force;
* error behaviour: collisions, singular cells, no device.
"""
import ctypes as C
import os

import numpy as np
import pytest

from abi import LIB, Abi, AbiError, header_functions


def test_library_exports_every_header_symbol():
    assert os.path.exists(LIB), "build the library first (python -m libdescriptor_b200.build)"
    lib = C.CDLL(LIB)
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"undefined: {missing}"


def test_python_module_mirrors_reference_api():
    import libdescriptor_b200 as lds

    for name in ["AvailableDescriptors", "DescriptorKind", "compute", "compute_batch",
                 "compute_single_atom", "gradient", "gradient_batch", "gradient_single_atom",
                 "jacobian", "num_gradient_single_atom", "NeighList", "create", "create_paddings"]:
        assert hasattr(lds, name), name
    assert int(lds.AvailableDescriptors.SymmetryFunctions) == 0
    assert int(lds.AvailableDescriptors.Bispectrum) == 1
    assert int(lds.AvailableDescriptors.SOAP) == 2
    assert int(lds.AvailableDescriptors.Xi) == 3


def _cells():
    from libdescriptor_b200.workloads import diamond_cell, random_packing

    out = []
    x, cell = diamond_cell(2, 2, 2, jitter=0.05, seed=0)
    out.append((x, cell, np.zeros(len(x), np.int32), (1, 1, 1)))
    x, cell = diamond_cell(1, 2, 3, jitter=0.1, strain=0.03, seed=4)   # 5.43 A < 2 rc: many images
    out.append((x, cell, (np.arange(len(x)) % 2).astype(np.int32), (1, 1, 1)))
    x, cell = diamond_cell(2, 1, 1, jitter=0.1, seed=5)
    out.append((x, cell, np.zeros(len(x), np.int32), (1, 0, 1)))        # one direction open
    x, cell, sp = random_packing(150, seed=2)
    out.append((x, cell, sp, (1, 1, 1)))
    return out


@pytest.mark.parametrize("case", range(4))
def test_neighbor_builder_matches_reference(oracle_mod, case):
    from libdescriptor_b200 import workloads as W
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference library not built here")
    x, cell, sp, pbc = _cells()[case]
    rc = 5.0
    cfg = W.prepare(x, cell, sp, rc, pbc=pbc)
    pc, ps, pi = Reference.create_paddings(rc, cell, list(pbc), x, sp)
    allx = np.concatenate([x, pc])
    np.testing.assert_array_equal(cfg.coords, allx)          # bit-identical ghosts
    np.testing.assert_array_equal(cfg.species[len(x):], ps)
    np.testing.assert_array_equal(cfg.image[len(x):], pi)
    need = np.zeros(len(allx), np.int32)
    need[: len(x)] = 1
    counts, nbl = Reference.neighbor_list(allx, rc, need, len(x))
    np.testing.assert_array_equal(cfg.counts, counts)
    np.testing.assert_array_equal(cfg.nbl, nbl)              # same order


@pytest.mark.parametrize("case", range(4))
def test_neighbor_builder_matches_brute_force(case):
    from libdescriptor_b200 import workloads as W

    x, cell, sp, pbc = _cells()[case]
    rc = 5.0
    cfg = W.prepare(x, cell, sp, rc, pbc=pbc)
    off = np.concatenate([[0], np.cumsum(cfg.counts)])
    allx = cfg.coords
    for i in range(cfg.n_atoms):
        d2 = np.sum((allx - allx[i]) ** 2, axis=1)
        want = set(np.nonzero((d2 < rc * rc) & (np.arange(len(allx)) != i))[0].tolist())
        got = cfg.nbl[off[i]:off[i + 1]].tolist()
        assert len(got) == len(set(got))
        assert set(got) == want
    # every periodic image within rc of the home cell is present: the
    # folded neighbour count equals the minimum-image-free count
    assert cfg.image.max() < cfg.n_atoms


def test_neighbor_builder_errors():
    import libdescriptor_b200 as lds

    with pytest.raises(ValueError, match="determinant"):
        lds.create_paddings(5.0, np.zeros((3, 3)), np.ones(3, np.int32), np.zeros((2, 3)),
                            np.zeros(2, np.int32))
    nl = lds.create()
    x = np.array([[0.0, 0, 0], [0.0, 0, 1e-7], [3.0, 0, 0]])
    with pytest.raises(RuntimeError):
        nl.build(x, 5.0, np.array([5.0]), np.ones(3, np.int32))


def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(AbiError) as e:
        Abi.create_sf(1, np.full((1, 1), 5.0), ["g2"], [1, 2], [0.1, 0.0])
    assert e.value.code == 7  # LD_ERR_NO_DEVICE
    import libdescriptor_b200 as lds

    with pytest.raises(RuntimeError, match="no CUDA device"):
        lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, 8, 3, 0, 0.0,
                                           1, 0, 5.0, ["Si"], [1.0])


def test_allocation_fault_injection_is_host_side():
    """ld_fail_next_allocation arms a host-side failure of the library's k-th
    next device allocation (the GPU tests drive the failure itself); arming
    and disarming touch no device."""
    L = Abi.lib()
    n0 = L.ld_alloc_count()
    assert L.ld_fail_next_allocation(-1) == 2          # LD_ERR_INVALID_ARG
    assert L.ld_fail_next_allocation(3) == 0
    assert L.ld_fail_next_allocation(0) == 0           # disarmed
    assert L.ld_alloc_count() == n0


def test_scratch_fill_hook_checks_its_byte():
    """ld_debug_fill_scratch takes a byte or -1 (off); arming it touches no
    device (the GPU test runs the kernels with every allocation filled)."""
    L = Abi.lib()
    assert L.ld_debug_fill_scratch(-2) == 2           # LD_ERR_INVALID_ARG
    assert L.ld_debug_fill_scratch(256) == 2
    assert L.ld_debug_fill_scratch(0xFF) == 0
    assert L.ld_debug_fill_scratch(-1) == 0


def test_bulk_wait_self_test_checks_its_limit():
    """ld_debug_bulk_wait_timeout takes 1 .. 1e9 ns and needs a device (the
    GPU test makes the wait run out)."""
    import torch

    L = Abi.lib()
    assert L.ld_debug_bulk_wait_timeout(0) == 2
    assert L.ld_debug_bulk_wait_timeout(2 * 10**9) == 2
    if not torch.cuda.is_available():
        assert L.ld_debug_bulk_wait_timeout(1000) == 7          # LD_ERR_NO_DEVICE
