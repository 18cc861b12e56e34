"""CPU tests of the oracle: pinned to the reference's golden vectors (forces, energy, virial of
its 23,558-atom recip test and its FFT known-answer vectors), to numpy's FFT, to finite
differences of its own energy, and to the analytic Ewald sum of two point charges."""
import math

import numpy as np
import pytest

from gpu_recip_b200 import systems as S


@pytest.mark.parametrize("order", [4, 6])
def test_reference_fixture(oracle, ref_fixture, order):
    f = ref_fixture
    box = f["box"]
    r = 1.0 / box
    res = oracle.evaluate(f["xyzq"].astype(np.float64), r, tuple(f["nfft"]), order, float(f["kappa"]))
    # tolerances of the reference test driver (gpu_recip.cu:146-174, :286-291; :373-384, :515)
    assert abs(res["energy"] - f[f"energy{order}"]) < f[f"tol_energy{order}"]
    assert np.abs(res["virial"] - f[f"virial{order}"]).max() < f[f"tol_virial{order}"]
    assert np.abs(res["force"] - f[f"force{order}"]).max() < f[f"tol_force{order}"]


def test_fft_known_answers(oracle, fft_kat):
    for tag in ("64", "64x2"):
        x = fft_kat["in" + tag]
        for row in range(x.shape[0]):
            got = oracle.fft1d(x[row].astype(np.complex128), -1)
            # reference compare tolerance: 1e-5 max abs (test_fbfft.cu:65-85)
            assert np.abs(got - fft_kat["out" + tag][row]).max() < 1e-5
    for tag in ("4x4", "64x64"):
        x = fft_kat["in" + tag]
        ny, nx = x.shape
        grid = np.broadcast_to(x, (4, ny, nx)).copy()           # 4 identical z planes
        half = oracle.fft3d_r2c(grid)
        got = half[0] / 4.0                                       # kz = 0 plane / nz
        assert np.abs(got - fft_kat["out" + tag][:, : nx // 2 + 1]).max() < 1e-4


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 8, 9, 12, 15, 24, 25, 27, 30, 32, 45, 60, 64, 100, 216, 7, 14])
def test_fft1d_vs_numpy(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    assert np.allclose(oracle.fft1d(x, -1), np.fft.fft(x), atol=1e-10 * n)
    assert np.allclose(oracle.fft1d(x, +1), np.fft.ifft(x) * n, atol=1e-10 * n)
    assert np.allclose(oracle.dft1d(x, -1), np.fft.fft(x), atol=1e-9 * n)


@pytest.mark.parametrize("shape", [(8, 6, 10), (5, 9, 12), (24, 25, 27)])
def test_fft3d_vs_numpy(oracle, shape):
    nz, ny, nx = shape
    rng = np.random.default_rng(7)
    g = rng.normal(size=shape)
    h = oracle.fft3d_r2c(g)
    assert np.allclose(h, np.fft.rfftn(g), atol=1e-9)
    back = oracle.fft3d_c2r(h, nx)
    assert np.allclose(back, g * g.size, atol=1e-8)


@pytest.mark.parametrize("order", [4, 6, 8])
def test_bspline_partition_of_unity(oracle, order):
    for u in (0.0, 0.13, 0.5, 0.999):
        th, dth = oracle.bspline(order, u)
        assert abs(th.sum() - 1.0) < 1e-14
        assert abs(dth.sum()) < 1e-14
        # derivative check against finite differences of the weights
        h = 1e-6
        tp, _ = oracle.bspline(order, min(u + h, 1.0))
        tm, _ = oracle.bspline(order, max(u - h, 0.0))
        fd = (tp - tm) / (min(u + h, 1.0) - max(u - h, 0.0))
        assert np.allclose(fd, dth, atol=1e-6)


def test_moduli_symmetric_positive(oracle):
    for order in (4, 6, 8):
        for n in (24, 25, 32, 64, 216):
            b = oracle.bspline_moduli(order, n)
            assert np.all(b > 0)
            assert np.allclose(b[1:], b[1:][::-1], rtol=1e-12)
            assert abs(b[0] - 1.0) < 1e-12


def test_forces_are_energy_gradient(oracle):
    """The gather output is +dE/dx (the reference's convention): check by central differences."""
    sys_ = S.water_box(30, (12.0, 13.0, 11.0), seed=5).astype(np.float64)
    nfft, order, kappa = (16, 16, 15), 4, 0.4
    r = 1.0 / np.array([12.0, 13.0, 11.0])
    res = oracle.evaluate(sys_, r, nfft, order, kappa)
    h = 1e-5
    for i in (0, 7, 29, 55):
        for d in range(3):
            xp = sys_.copy(); xp[i, d] += h
            xm = sys_.copy(); xm[i, d] -= h
            ep = oracle.evaluate(xp, r, nfft, order, kappa)["energy"]
            em = oracle.evaluate(xm, r, nfft, order, kappa)["energy"]
            assert abs((ep - em) / (2 * h) - res["force"][i, d]) < 1e-6 * max(1.0, abs(res["force"][i, d]))


def test_virial_matches_box_derivative(oracle):
    """Reciprocal virial W_aa = -L_a dE/dL_a at fixed fractional coordinates (diagonal)."""
    x = S.water_box(20, (10.0, 11.0, 12.0), seed=9).astype(np.float64)
    box = np.array([10.0, 11.0, 12.0])
    nfft, order, kappa = (20, 20, 20), 6, 0.35
    res = oracle.evaluate(x, 1.0 / box, nfft, order, kappa)
    frac = x[:, :3] / box
    for a in range(3):
        eps = 1e-6
        vals = []
        for s in (+1, -1):
            b = box.copy(); b[a] *= (1 + s * eps)
            xx = x.copy(); xx[:, :3] = frac * b
            vals.append(oracle.evaluate(xx, 1.0 / b, nfft, order, kappa)["energy"])
        dEdlnL = (vals[0] - vals[1]) / (2 * eps)
        assert abs(-dEdlnL - res["virial"][a, a]) < 2e-5 * max(1.0, abs(res["virial"][a, a]))
    assert np.allclose(res["virial"], res["virial"].T)


def _ewald_recip_pair(L, kappa, q1, q2, r12, kmax=40):
    """Exact reciprocal Ewald energy of two charges (plus their images) in a cube."""
    e = 0.0
    ks = np.arange(-kmax, kmax + 1)
    kx, ky, kz = np.meshgrid(ks, ks, ks, indexing="ij")
    m2 = (kx ** 2 + ky ** 2 + kz ** 2) / L ** 2
    mask = m2 > 0
    sf = q1 + q2 * np.exp(2j * np.pi * (kx * r12[0] + ky * r12[1] + kz * r12[2]) / L)
    term = np.exp(-np.pi ** 2 * m2[mask] / kappa ** 2) / m2[mask] * np.abs(sf[mask]) ** 2
    e = term.sum() / (2 * np.pi * L ** 3) * 332.0716
    return e


def test_two_charge_ewald(oracle):
    """The gpu_pair probe (gpu_pair.cu:80-139): +-1 charges at distance r in an L box."""
    L, kappa = 20.0, 0.32
    for r in (1.0, 3.5, 7.0):
        x = np.array([[-r / 2 + L / 2, L / 2, L / 2, -1.0], [r / 2 + L / 2, L / 2, L / 2, 1.0]])
        res = oracle.evaluate(x, np.full(3, 1.0 / L), (40, 40, 40), 8, kappa)
        exact = _ewald_recip_pair(L, kappa, -1.0, 1.0, np.array([r, 0.0, 0.0]))
        assert abs(res["energy"] - exact) < 1e-5 * abs(exact) + 1e-6
        # equal and opposite forces, along x
        f = res["force"]
        assert np.allclose(f[0], -f[1], atol=1e-6)
        assert abs(f[0, 1]) < 1e-6 and abs(f[0, 2]) < 1e-6
        assert abs(res["energy_self"] + 2 * kappa * 332.0716 / math.sqrt(math.pi)) < 1e-9


def test_fixed_grid_matches_f64(oracle):
    s = S.config_small()
    g64 = oracle.spread_f64(s.xyzq, s.recip3, s.nfft, s.order)
    gfx = oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, s.order)
    gf = gfx.astype(np.float64) / 2.0 ** 40
    assert np.abs(gf - g64).max() < 1e-5
    assert abs(gfx.sum() / 2.0 ** 40 - s.xyzq[:, 3].astype(np.float64).sum()) < 1e-6
    # conversion is one rounding of the exact quotient
    assert np.array_equal(oracle.fixed_to_float(gfx), (gfx.astype(np.float64) / 2.0 ** 40).astype(np.float32))


def test_fixed_grid_thread_count_independent(oracle):
    s = S.config_small(seed=11)
    a = oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, 6, nthreads=1)
    b = oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, 6, nthreads=5)
    assert np.array_equal(a, b)


def test_oracle_translation_invariance(oracle):
    """Shifting all atoms by a whole grid cell leaves energy and forces unchanged."""
    s = S.config_small(seed=3)
    x = s.xyzq.astype(np.float64)
    L = s.box[0]
    a = oracle.evaluate(x, s.recip3, s.nfft, s.order, s.kappa)
    y = x.copy(); y[:, 0] = np.mod(y[:, 0] + L / s.nfft[0] * 3, L)
    b = oracle.evaluate(y, s.recip3, s.nfft, s.order, s.kappa)
    assert abs(a["energy"] - b["energy"]) < 1e-9 * abs(a["energy"])
    assert np.allclose(a["force"], b["force"], atol=1e-9)
