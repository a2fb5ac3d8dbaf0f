"""The synthetic orbitals that stand in for the benchmark systems: a seed
regenerates the same bits within a machine (the raw draws come from numpy's
seeded generator; the orthonormalisation runs through the host's BLAS and
LAPACK, so the last bits may differ between machines, which is why every
parity test compares the GPU with the oracle on the orbitals regenerated
where it runs, never with a fixture made from another machine's bits), the
sets are orthonormal, and every shape keeps the sizes the bench quotes."""
import numpy as np

from libisdf_b200 import synth


def test_orbitals_regenerate_bit_for_bit_on_one_machine():
    a = synth.shape_orbitals(synth.SI8, 0)
    b = synth.shape_orbitals(synth.SI8, 0)
    assert synth.sha256(a) == synth.sha256(b)
    assert synth.sha256(a) != synth.sha256(synth.shape_orbitals(synth.SI8, 1))


def test_orbitals_are_orthonormal():
    psi = synth.shape_orbitals(synth.SI8, 3)
    assert psi.shape == (synth.SI8.ng, synth.SI8.nstate)
    gram = psi.T @ psi
    assert np.abs(gram - np.eye(psi.shape[1])).max() < 1e-12


def test_shapes_quote_the_benchmark_sizes():
    assert (synth.SI8.ng, synth.SI8.nstate, synth.SI8.mu) == (64000, 32, 320)
    assert (synth.SI64.ng, synth.SI64.nstate, synth.SI64.mu) == (512000, 256, 2048)
    assert (synth.SI216.ng, synth.SI216.nstate, synth.SI216.mu) == (1259712, 864, 4320)
    for s in (synth.SI8, synth.SI64, synth.SI216):
        assert s.nv1 == s.nc1 == s.nv2 == s.nc2 == s.nocc == s.nstate // 2
        assert s.kmeans_iters == 100
