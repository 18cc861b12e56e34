"""GPU parity of the sm_100a path against the CPU oracle and the reference's golden vectors.

Bars: the int64 charge grid is bit-exact against the oracle's FP32 mirror; forces within a
relative RMS of 1e-5 and energy within a relative 1e-6 of the FP64 oracle; the reference's own
energy/virial/force tolerances on its 23,558-atom fixture.
"""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5       # relative RMS of forces vs FP64 oracle
FORCE_ABS_FLOOR = 1e-5     # kcal/mol/A: RMS floor for systems whose exact forces are ~0 (one atom)
ENERGY_REL_TOL = 1e-6      # relative energy error vs FP64 oracle
VIRIAL_REL_TOL = 1e-5      # max |dW| / max |W|


def _sys(name):
    if name == "water1k_32":
        return S.config_small()
    if name == "water8k_64_p4":
        return S.config_production(4)
    if name == "water8k_64_p6":
        return S.config_production(6)
    if name == "water1k_p8":
        s = S.config_small(seed=21)
        return S.PmeSystem("p8", s.xyzq, s.box, (36, 32, 40), 8, 0.34)
    if name == "odd_grid":
        box = (25.3, 27.1, 44.0)
        return S.PmeSystem("odd", S.water_box(900, box, 31), box, (25, 27, 45), 4, 0.32)
    if name == "noncubic_p6":
        box = (30.0, 24.0, 40.0)
        return S.PmeSystem("nc", S.water_box(700, box, 32), box, (30, 24, 40), 6, 0.3)
    if name == "one_atom":
        return S.PmeSystem("one", np.array([[1.3, 2.7, 4.1, 0.5]], np.float32), (10.0, 10.0, 10.0),
                           (16, 16, 16), 4, 0.4)
    if name == "long_z":      # nz > 256: the fused path runs separate y / z passes, not plane tiles
        box = (15.0, 16.0, 300.0)
        return S.PmeSystem("lz", S.water_box(1500, box, 34), box, (16, 18, 320), 4, 0.35)
    if name == "bigq":        # two charges of +-700: the fused tile leaves its 2-sum accumulation form
        s = _sys("odd_grid")
        x = s.xyzq.copy()
        x[0, 3], x[1, 3] = 700.0, -700.0
        return S.PmeSystem("bigq", x, s.box, s.nfft, s.order, s.kappa)
    if name == "dense_p8":    # > 65,536 candidate atoms per row block: the carry accumulation form
        box = (20.0, 20.0, 20.0)
        return S.PmeSystem("dense", S.water_box(45000, box, 35), box, (16, 16, 16), 8, 0.4)
    if name == "ragged33":
        box = (15.0, 15.0, 15.0)
        x = S.water_box(11, box, 33)
        return S.PmeSystem("r33", x, box, (16, 18, 20), 6, 0.35)
    raise KeyError(name)


CASES = ["water1k_32", "water8k_64_p4", "water8k_64_p6", "water1k_p8", "odd_grid", "noncubic_p6",
         "one_atom", "ragged33", "long_z", "bigq"]


def _pme(cuda, s):
    from gpu_recip_b200 import CudaPMERecip
    return CudaPMERecip(*s.nfft, s.order)


def _run(cuda, s, staged=False, kind="soa", pme=None):
    from gpu_recip_b200 import force_stride, recip_from_box
    torch = cuda
    pme = pme or _pme(cuda, s)
    x = torch.from_numpy(np.ascontiguousarray(s.xyzq)).cuda()
    n = s.natom
    recip = recip_from_box(s.box)
    ev = pme.energy_virial
    ev.clear()
    if kind == "soa":
        stride = force_stride(n)
        f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
    else:
        stride = 1
        f = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    if staged:
        pme.spread_charge(x, n, recip)
        pme.r2c_fft()
        pme.scalar_sum(recip, s.kappa, True, True)
        pme.c2r_fft()
        pme.gather_force(x, n, recip, stride, f)
        pme.calc_self_energy(x, n, s.kappa)
    else:
        pme.eval_ortho([1.0 / b for b in s.box], x, n, s.kappa, True, True, f, stride)
    torch.cuda.synchronize()
    ev.copyToHost()
    if kind == "soa":
        F = f.view(3, stride)[:, :n].T.cpu().numpy().astype(np.float64)
    else:
        F = f.cpu().numpy().astype(np.float64)
    return dict(force=F, energy=ev.getEnergy("recip"), energy_self=ev.getEnergy("self"),
                virial=ev.getVirial(), pme=pme, x=x)


def _rel_rms(a, b):
    """Relative RMS force error, with an absolute floor for near-zero reference forces."""
    err = np.sqrt(((a - b) ** 2).sum())
    ref = np.sqrt((b ** 2).sum())
    return float(err / max(ref, FORCE_ABS_FLOOR * np.sqrt(b.shape[0]) / FORCE_RMS_TOL))


@pytest.mark.parametrize("name", CASES + ["empty"])
def test_spread_grid_bit_exact(cuda, oracle, name):
    if name == "empty":
        s = S.PmeSystem("empty", np.zeros((0, 4), np.float32), (10.0, 10.0, 10.0), (16, 16, 16), 4, 0.3)
    else:
        s = _sys(name)
    from gpu_recip_b200 import recip_from_box
    pme = _pme(cuda, s)
    x = cuda.from_numpy(np.ascontiguousarray(s.xyzq)).cuda() if s.natom else cuda.zeros((1, 4), device="cuda")
    pme.spread_charge(x, s.natom, recip_from_box(s.box))
    got = pme.charge_grid_fixed()
    want = oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, s.order)
    assert got.shape == want.shape
    assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} grid points differ"
    # float view of the grid is the one-rounding conversion of the fixed-point values
    assert np.array_equal(pme.charge_grid(), oracle.fixed_to_float(want))


@pytest.mark.parametrize("name", CASES)
def test_eval_matches_fp64_oracle(cuda, oracle, name):
    s = _sys(name)
    got = _run(cuda, s)
    ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
    e_rel = abs(got["energy"] - ref["energy"]) / abs(ref["energy"])
    f_rms = _rel_rms(got["force"], ref["force"])
    v_rel = np.abs(got["virial"] - ref["virial"]).max() / np.abs(ref["virial"]).max()
    assert e_rel <= ENERGY_REL_TOL, e_rel
    assert f_rms <= FORCE_RMS_TOL, f_rms
    assert v_rel <= VIRIAL_REL_TOL, v_rel
    assert abs(got["energy_self"] - ref["energy_self"]) <= 1e-12 * abs(ref["energy_self"])


@pytest.mark.parametrize("order", [4, 6])
def test_reference_fixture(cuda, ref_fixture, order):
    f = ref_fixture
    s = S.PmeSystem("ref", f["xyzq"], tuple(f["box"]), tuple(int(v) for v in f["nfft"]), order,
                    float(f["kappa"]))
    got = _run(cuda, s)
    assert abs(got["energy"] - f[f"energy{order}"]) < f[f"tol_energy{order}"]
    assert np.abs(got["virial"] - f[f"virial{order}"]).max() < f[f"tol_virial{order}"]
    assert np.abs(got["force"] - f[f"force{order}"]).max() < f[f"tol_force{order}"]


@pytest.mark.parametrize("name,schedule", [("water8k_64_p4", 1), ("water8k_64_p4", 2),
                                           ("long_z", 0), ("noncubic_p6", 1), ("bigq", 0),
                                           ("dense_p8", 0)])
def test_staged_calls_equal_fused_eval(cuda, name, schedule):
    """Staged reference-style calls and the fused kernel (either y/z schedule) agree bit for bit.
    The fused tile accumulates its charge rows in one of three exact forms, chosen from the tile's
    candidate count and the largest |q|; water boxes take the 2-sum form, bigq the 3-sum form and
    dense_p8 the carry form, and all must give the staged path's int64 grid."""
    s = _sys(name)
    a = _run(cuda, s, staged=True)
    pme = _pme(cuda, s)
    pme.set_fft_schedule(schedule)
    b = _run(cuda, s, staged=False, pme=pme)
    assert np.array_equal(a["force"], b["force"])
    assert a["energy"] == b["energy"] and a["energy_self"] == b["energy_self"]
    assert np.array_equal(a["virial"], b["virial"])


def test_run_to_run_deterministic(cuda):
    s = _sys("water8k_64_p6")
    a = _run(cuda, s)
    b = _run(cuda, s, pme=a["pme"])
    assert np.array_equal(a["force"], b["force"])
    assert a["energy"] == b["energy"] and np.array_equal(a["virial"], b["virial"])


def test_force_output_kinds(cuda):
    from gpu_recip_b200 import FORCE_SCALE, force_stride, recip_from_box
    torch = cuda
    s = _sys("water1k_32")
    soa = _run(cuda, s, kind="soa")
    aos = _run(cuda, s, kind="aos", pme=soa["pme"])
    assert np.array_equal(soa["force"], aos["force"])
    # int64 fixed point: accumulated (twice -> doubled), equal to rounding the float forces
    pme, x, n = soa["pme"], soa["x"], s.natom
    stride = force_stride(n, 8)
    fi = torch.zeros(3 * stride, dtype=torch.int64, device="cuda")
    recip = recip_from_box(s.box)
    for _ in range(2):
        pme.gather_force(x, n, recip, stride, fi)
    torch.cuda.synchronize()
    got = fi.view(3, stride)[:, :n].T.cpu().numpy()
    want = np.rint(soa["force"].astype(np.float32).astype(np.float64) * FORCE_SCALE).astype(np.int64)
    assert np.array_equal(got, 2 * want)


def test_energy_virial_accumulate(cuda):
    from gpu_recip_b200 import force_stride
    s = _sys("water1k_32")
    a = _run(cuda, s)
    pme, x, n = a["pme"], a["x"], s.natom
    f = cuda.zeros(3 * force_stride(n), dtype=cuda.float32, device="cuda")
    pme.energy_virial.clear()
    for _ in range(2):
        pme.eval_ortho([1.0 / b for b in s.box], x, n, s.kappa, True, True, f, force_stride(n))
    pme.energy_virial.copyToHost()
    assert pme.energy_virial.getEnergy("recip") == 2 * a["energy"]
    assert np.array_equal(pme.energy_virial.getVirial(), 2 * a["virial"])
    assert pme.energy_virial.getEnergy("self") == 2 * a["energy_self"]


@pytest.mark.parametrize("shape", [(64, 64, 64), (24, 25, 27), (30, 36, 40), (216, 16, 8)])
def test_fft_roundtrip_and_spectrum(cuda, shape):
    from gpu_recip_b200 import CudaPMERecip
    nz, ny, nx = shape
    rng = np.random.default_rng(sum(shape))
    g = rng.uniform(-1, 1, size=shape).astype(np.float32)
    pme = CudaPMERecip(nx, ny, nz, 4)
    pme.load_charge_grid(g)
    loaded = pme.charge_grid().astype(np.float64)      # the r2c pass consumes (zeroes) the grid
    pme.r2c_fft()
    spec = pme.fft_grid()
    exact = np.fft.rfftn(loaded)
    scale = np.abs(exact).max()
    assert np.abs(spec - exact).max() <= 2e-6 * scale * np.log2(g.size)
    assert not pme.charge_grid_fixed().any()
    pme.c2r_fft()
    back = pme.solved_grid().astype(np.float64) / g.size
    assert np.abs(back - loaded).max() <= 1e-5


def test_fft_known_answer_vectors(cuda, fft_kat):
    """The reference's 2-D FFT KAT (test_fbfft.cu:188-256) through the 3-D R2C: 4 identical z
    planes, so the kz = 0 plane is 4x the 2-D transform."""
    from gpu_recip_b200 import CudaPMERecip
    for tag in ("64x64",):
        x = fft_kat["in" + tag]
        ny, nx = x.shape
        pme = CudaPMERecip(nx, ny, 4, 4)
        pme.load_charge_grid(np.broadcast_to(x, (4, ny, nx)).astype(np.float32))
        pme.r2c_fft()
        got = pme.fft_grid()[0] / 4.0
        assert np.abs(got - fft_kat["out" + tag][:, : nx // 2 + 1]).max() < 1e-4


def test_invalid_arguments_rejected(cuda):
    from gpu_recip_b200 import CudaPMERecip, _capi
    with pytest.raises(_capi.PMEError) as e:
        CudaPMERecip(64, 64, 64, 5)
    assert e.value.status == _capi.PME_EINVAL
    with pytest.raises(_capi.PMEError) as e:
        CudaPMERecip(64, 49, 64, 4)
    assert e.value.status == _capi.PME_EUNSUPPORTED
    pme = CudaPMERecip(32, 32, 32, 4)
    x = cuda.zeros((4, 4), device="cuda")
    with pytest.raises(_capi.PMEError) as e:   # singular matrix (the first two rows are equal)
        pme.spread_charge(x, 4, [0.1, 0.1, 0, 0.1, 0.1, 0, 0, 0, 0.1])
    assert e.value.status == _capi.PME_EINVAL
    with pytest.raises(_capi.PMEError) as e:   # negative diagonal of an orthorhombic box
        pme.spread_charge(x, 4, [-0.1, 0, 0, 0, 0.1, 0, 0, 0, 0.1])
    assert e.value.status == _capi.PME_EINVAL


def test_nonfinite_coordinates_stay_in_bounds(cuda, oracle):
    """NaN/inf coordinates are mapped to stencil origin 0 (no out-of-grid access)."""
    s = _sys("ragged33")
    x = s.xyzq.copy()
    x[3, 0] = np.nan
    x[5, 2] = np.inf
    x[7, 1] = -1e30
    bad = S.PmeSystem("bad", x, s.box, s.nfft, s.order, s.kappa)
    from gpu_recip_b200 import recip_from_box
    pme = _pme(cuda, bad)
    xd = cuda.from_numpy(x).cuda()
    pme.spread_charge(xd, bad.natom, recip_from_box(bad.box))
    assert np.array_equal(pme.charge_grid_fixed(), oracle.spread_fixed(x, bad.recip3, bad.nfft, bad.order))


def test_atom_count_change_on_one_handle(cuda):
    """The fused path walks atoms in the previous evaluation's bin-sorted order only when that
    order was built for the same atom count: evaluations whose count changes on one handle equal
    those of fresh handles bit for bit."""
    s = _sys("water8k_64_p4")
    fewer = S.PmeSystem("fewer", s.xyzq[:20011].copy(), s.box, s.nfft, s.order, s.kappa)
    pme = _pme(cuda, s)
    for sys_ in (s, fewer, fewer, s, s):
        got = _run(cuda, sys_, pme=pme)
        want = _run(cuda, sys_)
        assert np.array_equal(got["force"], want["force"]), sys_.name
        assert got["energy"] == want["energy"] and np.array_equal(got["virial"], want["virial"])


def _clustered():
    """3,000 atoms, 2,400 of them packed into a 4 A cube: their row blocks overflow the fixed bin
    capacity, so spread and gather go through the overflow list."""
    rng = np.random.default_rng(44)
    box = (30.0, 30.0, 30.0)
    x = np.empty((3000, 4), np.float32)
    x[:2400, :3] = 10.0 + 4.0 * rng.random((2400, 3))
    x[2400:, :3] = 30.0 * rng.random((600, 3))
    x[:, 3] = np.where(np.arange(3000) % 3 == 0, -0.834, 0.417)
    return S.PmeSystem("clustered", x, box, (32, 32, 32), 4, 0.34)


def test_bin_overflow_path(cuda, oracle):
    s = _clustered()
    a = _run(cuda, s, staged=True)
    b = _run(cuda, s)
    c = _run(cuda, s, pme=b["pme"])          # second evaluation walks the bin-sorted order
    ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
    assert _rel_rms(b["force"], ref["force"]) <= FORCE_RMS_TOL
    assert abs(b["energy"] - ref["energy"]) <= ENERGY_REL_TOL * abs(ref["energy"])
    for got in (b, c):
        assert np.array_equal(a["force"], got["force"])
        assert a["energy"] == got["energy"] and np.array_equal(a["virial"], got["virial"])
