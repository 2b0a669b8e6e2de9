"""Seeded synthetic media (CPU only)."""
import numpy as np

from lbx import geometry


def test_sphere_pack_porosity_and_determinism():
    a = geometry.sphere_pack(48, 40, 32, radius=4, porosity=0.4, seed=7)
    b = geometry.sphere_pack(48, 40, 32, radius=4, porosity=0.4, seed=7)
    assert a.dtype == np.uint8 and a.size == 48 * 40 * 32
    assert np.array_equal(a, b)
    por = geometry.porosity(a)
    assert 0.36 < por <= 0.4
    assert set(np.unique(a)) <= {0, 1}


def test_disc_pack_keeps_inlet_outlet_fluid():
    m = geometry.disc_pack(64, 48, radius=4, porosity=0.7, seed=3)
    g = m.reshape(48, 64)
    assert not g[:, 0].any() and not g[:, -1].any()
    assert geometry.porosity(m) <= 0.75


def test_transpose_roundtrip():
    m = (np.arange(12 * 5) % 3 == 0).astype(np.uint8)
    t = geometry.transpose_2d(m, 12, 5)
    assert np.array_equal(geometry.transpose_2d(t, 5, 12), m)
