"""GPU: every twojmax the bispectrum kernels are compiled for (0..10, odd
values included) against the oracle, descriptors and the coordinate
gradient, at the parity bars.

The golden fixtures pin the reference at 2J = 4, 6, 8; this sweep reaches the
other template instances: the rows-in-lanes Z kernel for every column count,
its global-weight form (2J = 9, where the weights and betaj do not fit next to
the U block) and the per-centre fallback (2J = 10, whose U block does not fit
one SM).
"""
import numpy as np
import pytest

from helpers import DESC_RTOL, GRAD_RTOL, assert_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("twojmax", list(range(0, 11)))
def test_every_twojmax_matches_oracle(oracle_mod, twojmax):
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W
    from oracle import OracleDescriptor

    x, cell, sp = W.random_packing(40, density=0.05, dmin=2.0, n_species=2, seed=21)
    cfg = W.prepare(x, cell, sp, 5.0)
    k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, 0.99363, twojmax, 3, 0, 0.0, 1, 0,
                                           5.0, ["A", "B"], [1.0, 0.5])
    o = OracleDescriptor.bispectrum(0.99363, twojmax, 3, 0.0, 1, 0, 2, np.full((2, 2), 5.0), [1.0, 0.5])
    assert int(k.width) == o.width
    n = cfg.n_atoms
    dE = np.random.default_rng(twojmax).normal(size=(n, o.width))
    desc, grad = lds.compute_and_gradient(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    desc_o, grad_o = o.run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE)
    assert_close(desc, desc_o, DESC_RTOL, f"2J={twojmax} desc")
    assert_close(grad, grad_o, GRAD_RTOL, f"2J={twojmax} grad")
    # the forward-only call agrees with the fused pass
    d2 = lds.compute(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
    assert_close(d2, desc_o, DESC_RTOL, f"2J={twojmax} forward-only desc")
