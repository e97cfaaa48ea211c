"""Parameter-file init (DescriptorKind::initDescriptor(file, kind)).

Files in the reference's format are read by the library
(ld_describe_parameter_file on the host, ld_create_from_file on the GPU) and
by the reference's own readers (SymmetryFunctions(std::string&),
src/SymmetryFunctions.cpp:262-407; Bispectrum(std::string&),
src/Bispectrum.cpp:848-1007, compiled into oracle/_ref).  Reproduced
reading rules:

* blank lines and lines starting with '#' are skipped; numbers are the
  whitespace tokens that parse as numbers (include/file_io_utils.hpp);
* the species block has n_species pair lines; species are ordered as a
  sorted set and a pair the file does not list gets cutoff 0;
* symmetry functions: the parameter vector is shared across types and never
  cleared, and every type reads its block from the START of that vector
  (so a second type re-reads the first type's numbers);
* bispectrum: the file gives jmax, and twojmax = 2 jmax.

Not reproduced: the bispectrum reader's capacity of 25 neighbours per centre
(src/Bispectrum.cpp:979-980), past which the reference writes out of bounds.
Centres with more neighbours are checked against the reference's direct
init with the same parameters, whose capacity is 250.
"""
import ctypes as C
import os

import numpy as np
import pytest

from abi import Abi, AbiError, describe_parameter_file
from helpers import DESC_RTOL, GRAD_RTOL, assert_close

SF_FILE = """# symmetry functions, two species
cos
2
Si Si 5.0
# the C-C pair is not listed: its cutoff is 0
Si C 4.5

2
g2 8 2
0.001 0.0
0.005 0.0
0.01 0.0
0.02 0.0
0.04 0.0
0.08 0.0
0.16 0.0
0.32 0.0
g4 16 3
1 -1 0.001
1 -1 0.01
1 -1 0.03
1 -1 0.08
1 1 0.001
1 1 0.01
1 1 0.03
1 1 0.08
4 -1 0.001
4 -1 0.01
4 -1 0.03
4 -1 0.08
4 1 0.001
4 1 0.01
4 1 0.03
4 1 0.08
false
24
"""

BS_FILE = """# bispectrum
cos
2
A A {rc}
A B {rc}
# jmax (twojmax = 2 jmax)
{jmax}
0.99363
3
0.0
1
0
1.0 0.5
"""


def _write(tmp_path, name, text):
    p = os.path.join(str(tmp_path), name)
    with open(p, "w") as f:
        f.write(text)
    return p


def _sf_expected():
    g2 = [v for e in (0.001, 0.005, 0.01, 0.02, 0.04, 0.08, 0.16, 0.32) for v in (e, 0.0)]
    g4 = [v for z in (1, 4) for lam in (-1, 1) for e in (0.001, 0.01, 0.03, 0.08) for v in (z, lam, e)]
    shared = g2 + g4
    return g2 + shared[:48]


def test_sf_file_is_read_with_the_reference_rules(tmp_path):
    d = describe_parameter_file(_write(tmp_path, "sf.txt", SF_FILE), 0)
    assert d["kind"] == 0 and d["n_species"] == 2
    assert d["species"] == ["C", "Si"]                       # sorted set
    np.testing.assert_array_equal(d["cutoff_matrix"], [0.0, 4.5, 4.5, 5.0])
    np.testing.assert_array_equal(d["type_codes"], [2, 4])
    np.testing.assert_array_equal(d["sizes"], [8, 2, 16, 3])
    np.testing.assert_array_equal(d["params"], _sf_expected())  # g4 re-reads from the start


def test_bs_file_is_read_with_the_reference_rules(tmp_path):
    d = describe_parameter_file(_write(tmp_path, "bs.txt", BS_FILE.format(rc=4.0, jmax=3)), 1)
    assert d["kind"] == 1 and d["species"] == ["A", "B"]
    assert d["twojmax"] == 6 and d["diagonalstyle"] == 3 and d["switch_flag"] == 1 and d["bzero_flag"] == 0
    assert d["rfac0"] == 0.99363 and d["rmin0"] == 0.0
    np.testing.assert_array_equal(d["weights"], [1.0, 0.5])
    np.testing.assert_array_equal(d["cutoff_matrix"], [4.0, 4.0, 4.0, 0.0])


def test_malformed_files_are_parse_errors(tmp_path):
    bad = _write(tmp_path, "bad.txt", "cos\n1\nSi Si 5.0\n1\ng2 2 2\n0.1 0.0\n")   # one row short
    with pytest.raises(AbiError) as e:
        describe_parameter_file(bad, 0)
    assert e.value.code == 8                                  # LD_ERR_PARSE
    with pytest.raises(AbiError) as e:
        describe_parameter_file(os.path.join(str(tmp_path), "missing.txt"), 0)
    assert e.value.code == 8 and "Could not open" in str(e.value)
    with pytest.raises(AbiError) as e:
        describe_parameter_file(_write(tmp_path, "sf.txt", SF_FILE), 2)
    assert e.value.code == 1                                  # SOAP: not supported
    # a too small text buffer: LD_ERR_CAPACITY and a truncated copy
    L = Abi.lib()
    buf = C.create_string_buffer(16)
    n = C.c_size_t(0)
    rc = L.ld_describe_parameter_file(_write(tmp_path, "sf2.txt", SF_FILE).encode(), 0, buf, 16, C.byref(n))
    assert rc == 3 and n.value > 16 and len(buf.value) == 15


def _packing(n, rc, seed):
    from libdescriptor_b200 import workloads as W

    x, cell, sp = W.random_packing(n, density=0.05, dmin=2.0, n_species=2, seed=seed)
    return W.prepare(x, cell, sp, rc)


def _oracle_of(d):
    from oracle import OracleDescriptor

    ns = d["n_species"]
    cm = np.asarray(d["cutoff_matrix"]).reshape(ns, ns)
    if d["kind"] == 0:
        names = [f"g{c}" for c in d["type_codes"]]
        return OracleDescriptor.symmetry_functions(ns, cm, names, d["sizes"], d["params"])
    return OracleDescriptor.bispectrum(d["rfac0"], d["twojmax"], d["diagonalstyle"], d["rmin0"], d["switch_flag"],
                                       d["bzero_flag"], ns, cm, d["weights"])


def test_parsed_parameters_give_the_reference_file_descriptors(tmp_path, oracle_mod):
    """On the CPU: the oracle with the parameters the library read equals the
    reference's file-constructed descriptors (symmetry functions, and the
    bispectrum on centres within the reference reader's 25 neighbours)."""
    from oracle import Reference, ReferenceDescriptor

    if not Reference.available():
        pytest.skip("reference library not built here")
    sf = _write(tmp_path, "sf.txt", SF_FILE)
    cfg = _packing(64, 5.0, 3)
    ref = ReferenceDescriptor.from_file(sf, 0)
    d = describe_parameter_file(sf, 0)
    ora = _oracle_of(d)
    assert ref.width == ora.width == 24
    want = ref.compute(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
    assert_close(ora.run(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords), want, DESC_RTOL, "sf file")
    bs = _write(tmp_path, "bs.txt", BS_FILE.format(rc=4.0, jmax=3))
    cfg = _packing(64, 4.0, 4)
    assert cfg.counts.max() <= 25        # inside the reference reader's capacity
    ref = ReferenceDescriptor.from_file(bs, 1)
    d = describe_parameter_file(bs, 1)
    ora = _oracle_of(d)
    assert ref.width == ora.width == 30
    want = ref.compute(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
    assert_close(ora.run(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords), want, DESC_RTOL, "bs file")


@pytest.mark.gpu
def test_gpu_descriptors_from_files_match_the_reference(tmp_path):
    """On the GPU: ld_create_from_file handles against the reference's
    file-constructed descriptors, the gradient against the oracle's adjoint;
    a bispectrum file on centres with more than 25 neighbours against the
    reference's direct init with the same parameters."""
    from oracle import Reference, ReferenceDescriptor

    cases = [(_write(tmp_path, "sf.txt", SF_FILE), 0, 5.0, 3, True),
             (_write(tmp_path, "bs6.txt", BS_FILE.format(rc=4.0, jmax=3)), 1, 4.0, 4, True),
             (_write(tmp_path, "bs8.txt", BS_FILE.format(rc=5.0, jmax=4)), 1, 5.0, 5, False)]
    for path, kind, rc, seed, file_ref in cases:
        cfg = _packing(256, rc, seed)
        h = Abi.create_from_file(path, kind)
        d = describe_parameter_file(path, kind)
        dE = np.random.default_rng(seed).normal(size=(cfg.n_atoms, h.width))
        grad, desc = h.gradient(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE, want_desc=True)
        d_ora, g_ora = _oracle_of(d).run(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords, dE=dE)
        assert_close(desc, d_ora, DESC_RTOL, f"{os.path.basename(path)} desc vs oracle")
        assert_close(grad, g_ora, GRAD_RTOL, f"{os.path.basename(path)} gradient vs oracle")
        if not Reference.available():
            continue
        if file_ref:
            assert kind == 0 or cfg.counts.max() <= 25
            ref = ReferenceDescriptor.from_file(path, kind)
        else:
            assert cfg.counts.max() > 25
            ns = d["n_species"]
            ref = ReferenceDescriptor.bispectrum(d["rfac0"], d["twojmax"], d["diagonalstyle"], d["rmin0"],
                                                 d["switch_flag"], d["bzero_flag"], ns,
                                                 np.asarray(d["cutoff_matrix"]).reshape(ns, ns), d["weights"])
        want = ref.compute(cfg.n_atoms, cfg.species, cfg.nbl, cfg.counts, cfg.coords)
        assert_close(desc, want, DESC_RTOL, f"{os.path.basename(path)} desc vs the reference")
