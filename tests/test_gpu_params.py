"""GPU: gradients of a loss with respect to the descriptor's own parameters
(symmetry functions: eta, Rs, kappa, zeta, lambda; bispectrum: rfac0) -- the
part of the reference's Enzyme gradient that it computes into a shadow
DescriptorKind and discards.

Checked against central finite differences of the oracle's forward
(the reference's forward restated in C) in every parameter:
L(theta) = sum dE * desc(theta), dL/dtheta_k ~ (L(theta + h_k) - L(theta -
h_k)) / (2 h_k), h_k = 1e-6 * max(|theta_k|, 1e-2).  Bar: 1e-6 relative to
the largest partial (the finite differences carry about 1e-8 of it).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_RTOL = 1e-6


def _case(kind):
    from libdescriptor_b200 import workloads as W

    if kind == "sf24":
        x, cell = W.diamond_cell(2, 2, 2, jitter=0.05, seed=5)
        sp = np.zeros(len(x), np.int32)
        t, sz, p = W.sf24_params()
        return W.prepare(x, cell, sp, 5.0), ["Si"], t, sz, p
    # every type, non-integer zeta, fractional lambda, non-zero Rs, two species
    x, cell, sp = W.random_packing(48, density=0.05, dmin=2.0, n_species=2, seed=8)
    types = ["g1", "g2", "g3", "g4", "g5"]
    sizes = [1, 0, 3, 2, 2, 1, 4, 3, 3, 3]
    params = ([0.02, 0.5, 0.05, 1.0, 0.3, 2.0] + [0.7, 1.3] +
              [1.0, 1.0, 0.01, 1.7, -1.0, 0.03, 4.0, 0.5, 0.005, 2.6, -0.4, 0.02] +
              [1.0, -1.0, 0.01, 2.3, 1.0, 0.004, 3.0, 0.6, 0.02])
    return W.prepare(x, cell, sp, 5.0), ["A", "B"], types, sizes, params


@pytest.mark.parametrize("kind", ["sf24", "all_types"])
def test_parameter_gradient_matches_oracle_fd(oracle_mod, kind):
    import libdescriptor_b200 as lds
    from oracle import OracleDescriptor

    cfg, species, types, sizes, params = _case(kind)
    params = np.asarray(params, dtype=np.float64)
    k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.SymmetryFunctions, species, "cos", 5.0,
                                           types, sizes, params.tolist())
    W = int(k.width)
    n = cfg.n_atoms
    dE = np.random.default_rng(9).normal(size=(n, W))
    got = lds.gradient_params(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    assert got.shape == params.shape

    ns = len(species)
    cm = np.full((ns, ns), 5.0)

    def loss(theta):
        o = OracleDescriptor.symmetry_functions(ns, cm, types, np.asarray(sizes).reshape(-1, 2), theta)
        desc = o.run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
        return float(np.sum(dE * desc))

    fd = np.zeros_like(params)
    for i in range(params.size):
        h = 1e-6 * max(abs(params[i]), 1e-2)
        tp, tm = params.copy(), params.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (loss(tp) - loss(tm)) / (2 * h)
    scale = np.max(np.abs(fd))
    assert scale > 0
    err = np.max(np.abs(got - fd)) / scale
    assert err <= FD_RTOL, (err, got, fd)
    # a second call on the same handle agrees to rounding (the per-lane sums
    # meet in FP64 atomics, whose order varies)
    again = lds.gradient_params(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    np.testing.assert_allclose(again, got, rtol=1e-12, atol=1e-12 * scale)


@pytest.mark.parametrize("twojmax", [6, 8])
def test_rfac0_gradient_matches_oracle_fd(oracle_mod, twojmax):
    """Bispectrum: the one parameter, rfac0 (it enters through theta0 of the
    Cayley-Klein map); two species with different weights, switching on."""
    import libdescriptor_b200 as lds
    from libdescriptor_b200 import workloads as W
    from oracle import OracleDescriptor

    x, cell, sp = W.random_packing(48, density=0.05, dmin=2.0, n_species=2, seed=12)
    cfg = W.prepare(x, cell, sp, 5.0)
    rfac0, wts = 0.99363, [1.0, 0.5]
    k = lds.DescriptorKind.init_descriptor(lds.AvailableDescriptors.Bispectrum, rfac0, twojmax, 3, 0, 0.0, 1, 0,
                                           5.0, ["A", "B"], wts)
    n = cfg.n_atoms
    dE = np.random.default_rng(13).normal(size=(n, int(k.width)))
    got = lds.gradient_params(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE)
    assert got.shape == (1,)
    cm = np.full((2, 2), 5.0)

    def loss(rf):
        o = OracleDescriptor.bispectrum(rf, twojmax, 3, 0.0, 1, 0, 2, cm, wts)
        return float(np.sum(dE * o.run(n, cfg.species, cfg.nbl, cfg.counts, cfg.coords)))

    h = 1e-6 * rfac0
    fd = (loss(rfac0 + h) - loss(rfac0 - h)) / (2 * h)
    assert abs(got[0] - fd) <= FD_RTOL * abs(fd), (got[0], fd)
    # the coordinate gradient of the same pass is unaffected
    desc0 = np.zeros((n, int(k.width)))
    ref = lds.gradient(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, desc0, dE)
    again = lds.gradient(k, n, cfg.species, cfg.nbl, cfg.counts, cfg.coords, desc0, dE)
    np.testing.assert_allclose(again, ref, rtol=1e-12, atol=1e-12 * np.max(np.abs(ref)))
