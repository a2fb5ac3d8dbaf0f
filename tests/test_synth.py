"""The synthetic orbitals that stand in for the benchmark systems: the
Si8-like set regenerates bit for bit (the hash its golden fixture recorded),
the sets are orthonormal, and every shape keeps the sizes the bench quotes."""
import numpy as np

from conftest import load_golden

from libisdf_b200 import synth


def test_si8_orbitals_regenerate_bit_for_bit():
    g = load_golden("si8_synth_seed0")
    psi = synth.shape_orbitals(synth.SI8, 0)
    assert synth.sha256(psi) == str(g["psi_sha256"])


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
