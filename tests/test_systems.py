"""CPU checks of the seeded synthetic workloads."""
import numpy as np

from gpu_recip_b200 import systems as S


def test_water_geometry_and_charges():
    box = (20.0, 21.0, 22.0)
    x = S.water_box(500, box, seed=3)
    assert x.dtype == np.float32 and x.shape == (1500, 4)
    assert abs(float(x[:, 3].astype(np.float64).sum())) < 1e-4
    o, h1, h2 = x[0::3, :3].astype(np.float64), x[1::3, :3].astype(np.float64), x[2::3, :3].astype(np.float64)
    L = np.array(box)

    def mic(d):
        return d - L * np.round(d / L)
    d1, d2 = mic(h1 - o), mic(h2 - o)
    assert np.allclose(np.linalg.norm(d1, axis=1), S.R_OH, atol=1e-4)
    ang = np.degrees(np.arccos((d1 * d2).sum(1) / np.linalg.norm(d1, axis=1) / np.linalg.norm(d2, axis=1)))
    assert np.allclose(ang, S.ANGLE_HOH, atol=0.05)
    assert (x[:, :3] >= 0).all() and (x[:, :3] < np.array(box, np.float32)).all()


def test_seeded_and_reproducible():
    a = S.water_box(100, (10, 10, 10), seed=7)
    b = S.water_box(100, (10, 10, 10), seed=7)
    c = S.water_box(100, (10, 10, 10), seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_configs_match_workload_table():
    s = S.config_production()
    assert s.natom == 24000 and s.nfft == (64, 64, 64) and s.alg_bytes() == 9575680
    s1 = S.config_small()
    assert s1.natom == 3000 and s1.alg_bytes() == 1213344


def test_batch_distribution():
    b = S.batch_systems(64, seed=4)
    assert len(b) == 64
    for s in b:
        assert 648 <= s.natom <= 24000
        for n in s.nfft:
            assert 24 <= n <= 64 and n in S.smooth235(24, 64)
