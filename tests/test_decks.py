"""Synthetic deck generators (CPU only)."""
import numpy as np

from mcmtop_b200.deck import taylor_bar, taylor_ensemble


def test_taylor_bar_lattice_counts():
    # cell-centred cylinder lattice: 208 particles per layer x 81 layers at dx = 0.4 mm
    assert taylor_bar(dx=0.4e-3).np == 16848


def test_ensemble_generator_ranges():
    decks = taylor_ensemble(nbodies=32, seed=5)
    n = np.array([d.np for d in decks])
    assert len(decks) == 32 and len({d.name for d in decks}) == 32
    assert n.min() >= 3000 and n.max() <= 70000
    for d in decks:
        m = d.materials[0]
        assert 200e6 * 1e-11 <= m.strinput[1] <= 600e6 * 1e-11
        vz = -d.v[0, 2] / 1e-4
        assert 120.0 <= vz <= 250.0
        r = np.hypot(d.x[:, 0], d.x[:, 1]).max() / 100.0
        assert r <= 4.1e-3


def test_ensemble_is_seeded():
    a = taylor_ensemble(nbodies=4, seed=9)
    b = taylor_ensemble(nbodies=4, seed=9)
    for da, db in zip(a, b):
        assert np.array_equal(da.x, db.x) and np.array_equal(da.v, db.v)
