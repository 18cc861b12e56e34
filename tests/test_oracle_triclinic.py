"""The oracle's triclinic mode (an extension: the reference accepts only orthorhombic boxes, so no
reference fixture pins it).  It is pinned instead against the exact Ewald reciprocal sum, computed
here directly from structure factors, and against the orthorhombic oracle on diagonal matrices."""
import ctypes

import numpy as np
import pytest

CC = 332.0716


def ewald_recip(xyzq, vectors, kappa, mmax=22):
    """Exact reciprocal Ewald sum: E = ccelec/(2 pi V) sum_{k != 0} exp(-pi^2 k^2/kappa^2)/k^2 |S(k)|^2
    with k = R m (R the inverse of the box-vector matrix), its virial in the form of
    CudaPMERecip.cu:871-886, and the gradient dE/dr_i."""
    B = np.asarray(vectors, dtype=np.float64)
    R = np.linalg.inv(B)
    V = abs(np.linalg.det(B))
    r, q = xyzq[:, :3], xyzq[:, 3]
    m = np.stack(np.meshgrid(*[np.arange(-mmax, mmax + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)
    m = m[np.any(m != 0, axis=1)]
    k = m @ R.T
    k2 = (k * k).sum(1)
    f = np.exp(-np.pi ** 2 * k2 / kappa ** 2) / k2
    ph = 2 * np.pi * (r @ k.T)
    S = (q[:, None] * np.exp(1j * ph)).sum(0)
    S2 = np.abs(S) ** 2
    E = CC / (2 * np.pi * V) * (f * S2).sum()
    vt = 2 * (np.pi ** 2 / kappa ** 2 + 1 / k2)
    W = np.array([[-0.5 * CC / (np.pi * V) * (f * S2 * (vt * k[:, i] * k[:, j] - (i == j))).sum()
                   for j in range(3)] for i in range(3)])
    im = np.imag(np.conj(S)[None, :] * np.exp(1j * ph))
    F = -(2 * CC / V) * q[:, None] * ((f[None, :] * im) @ k)
    return E, W, F


def _charges(vectors, n=40, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3)) @ np.asarray(vectors, dtype=np.float64)
    q = rng.normal(0.0, 0.5, n)
    q -= q.mean()
    return np.c_[x, q]


CELLS = {
    "orthorhombic": np.diag([21.0, 19.0, 20.0]),
    "triclinic": np.array([[21.0, 0.0, 0.0], [4.0, 19.0, 0.0], [-3.0, 5.0, 20.0]]),
    "tilted_cube": np.array([[20.0, 0.0, 0.0], [20.0, 20.0, 0.0], [0.0, -20.0, 20.0]]),  # a cube's lattice
}


@pytest.mark.parametrize("cell", list(CELLS))
def test_oracle_converges_to_exact_ewald(oracle, cell):
    B = CELLS[cell]
    xyzq = _charges(B)
    E, W, F = ewald_recip(xyzq, B, 0.34)
    res = oracle.evaluate(xyzq, np.linalg.inv(B).reshape(-1), (48, 48, 48), 8, 0.34)
    assert abs(res["energy"] - E) / abs(E) < 1e-8
    assert np.abs(res["virial"] - W).max() / np.abs(W).max() < 1e-7
    assert np.sqrt(((res["force"] - F) ** 2).sum() / (F ** 2).sum()) < 1e-7


def test_tilted_basis_of_a_cube_gives_the_cube_energy(oracle):
    """The same lattice in two bases (a, b, c) and (a, a + b, c - b): same exact energy, so the two
    PME energies agree to the PME error."""
    cube = np.diag([20.0, 20.0, 20.0])
    xyzq = _charges(cube, seed=3)
    e_cube = oracle.evaluate(xyzq, np.linalg.inv(cube).reshape(-1), (48, 48, 48), 8, 0.34)["energy"]
    tilt = CELLS["tilted_cube"]
    e_tilt = oracle.evaluate(xyzq, np.linalg.inv(tilt).reshape(-1), (48, 48, 48), 8, 0.34)["energy"]
    assert abs(e_tilt - e_cube) / abs(e_cube) < 1e-8


def _lib(oracle):
    return oracle.lib()


def test_triclinic_functions_on_a_diagonal_matrix_equal_the_orthorhombic_ones(oracle):
    """With zero off-diagonals the triclinic FP32 mirror gives the orthorhombic fixed-point grid bit
    for bit (the float-float coordinate adds exact zeros) and the FP64 evaluation agrees to rounding."""
    from gpu_recip_b200 import systems as S
    s = S.config_small(seed=4)
    L = _lib(oracle)
    r9 = np.array(s.recip9)
    nx, ny, nz = s.nfft
    P = ctypes.c_void_p
    g_t = np.zeros((nz, ny, nx), np.int64)
    x32 = np.ascontiguousarray(s.xyzq, np.float32)
    assert L.orc_spread_fixed_tric(P(x32.ctypes.data), s.natom, P(r9.ctypes.data), nx, ny, nz, s.order,
                                   P(g_t.ctypes.data), 0) == 0
    assert np.array_equal(g_t, oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, s.order))
    x64 = np.ascontiguousarray(s.xyzq, np.float64)
    f = np.zeros((s.natom, 3)); e = np.zeros(1); es = np.zeros(1); v = np.zeros(9)
    assert L.orc_eval_tric(P(x64.ctypes.data), s.natom, P(r9.ctypes.data), nx, ny, nz, s.order,
                           ctypes.c_double(s.kappa), P(f.ctypes.data), P(e.ctypes.data), P(es.ctypes.data),
                           P(v.ctypes.data), 0) == 0
    ref = oracle.evaluate(x64, s.recip3, s.nfft, s.order, s.kappa)
    assert abs(e[0] - ref["energy"]) <= 1e-12 * abs(ref["energy"])
    assert np.abs(v.reshape(3, 3) - ref["virial"]).max() <= 1e-11 * np.abs(ref["virial"]).max()
    assert np.abs(f - ref["force"]).max() <= 1e-10 * np.abs(ref["force"]).max()


def test_triclinic_water_systems_are_wrapped_and_neutral():
    from gpu_recip_b200 import systems as S
    for s in (S.config_triclinic_small(), S.config_triclinic()):
        frac = s.xyzq[:, :3].astype(np.float64) @ np.array(s.recip9).reshape(3, 3)
        assert frac.min() >= -1e-6 and frac.max() < 1.0 + 1e-6
        assert abs(float(s.xyzq[:, 3].astype(np.float64).sum())) < 1e-3
