"""Triclinic boxes on the GPU (an extension: the reference exits on non-orthorhombic recip,
CudaPMERecip.cu:2042-2045).  Bars as for orthorhombic boxes: the int64 charge grid bit-exact against
the oracle's FP32 mirror, the fused evaluation bit-exact against the staged calls, forces within a
relative RMS of 1e-5, energy within 1e-6 and virial within 1e-5 of the FP64 oracle (whose triclinic
mode is pinned to the exact Ewald sum on the CPU)."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5
ENERGY_REL_TOL = 1e-6
VIRIAL_REL_TOL = 1e-5


def _sys(name):
    if name == "tric_p4":
        return S.config_triclinic_small(4)
    if name == "tric_p6":
        return S.config_triclinic_small(6)
    if name == "tric_p8_odd":     # odd grid lengths and order 8
        s = S.config_triclinic_small(8, seed=7)
        return S.PmeSystem("tric_p8_odd", s.xyzq, s.box, (27, 25, 30), 8, 0.34, s.vectors)
    if name == "dodec_p4":
        return S.config_triclinic(4)
    if name == "tilted_cube":      # a cube's lattice in a skewed basis, Nyquist planes on every axis
        V = ((24.0, 0.0, 0.0), (24.0, 24.0, 0.0), (0.0, -24.0, 24.0))
        return S.PmeSystem("tilted", S.water_cell(450, V, 8), (24.0, 24.0, 24.0), (24, 24, 24), 6, 0.36, V)
    raise KeyError(name)


CASES = ["tric_p4", "tric_p6", "tric_p8_odd", "dodec_p4", "tilted_cube"]


def _run(cuda, s, staged, kind="soa"):
    from gpu_recip_b200 import CudaPMERecip, force_stride
    torch = cuda
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(np.ascontiguousarray(s.xyzq)).cuda()
    n = s.natom
    r9 = s.recip9
    ev = pme.energy_virial
    ev.clear()
    if kind == "soa":
        stride = force_stride(n)
        f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
    elif kind == "f3":
        stride = 1
        f = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    else:
        stride = force_stride(n, 8)
        f = torch.zeros(3 * stride, dtype=torch.int64, device="cuda")
    grid = None
    if staged:
        pme.spread_charge(x, n, r9)
        grid = pme.charge_grid_fixed()     # before R2C, which consumes the fixed-point grid
        pme.r2c_fft()
        pme.scalar_sum(r9, s.kappa, True, True)
        pme.c2r_fft()
        pme.gather_force(x, n, r9, stride, f)
        pme.calc_self_energy(x, n, s.kappa)
    else:
        pme.eval(r9, x, n, s.kappa, True, True, f, stride)
    torch.cuda.synchronize()
    ev.copyToHost()
    if kind == "f3":
        F = f.cpu().numpy()
    else:
        F = f.view(3, stride)[:, :n].T.cpu().numpy()
    out = dict(force=F, energy=ev.getEnergy("recip"), energy_self=ev.getEnergy("self"),
               virial=ev.getVirial(), grid=grid)
    pme.close()
    return out


@pytest.mark.parametrize("name", CASES)
def test_triclinic_spread_grid_bit_exact(cuda, oracle, name):
    s = _sys(name)
    got = _run(cuda, s, staged=True)["grid"]
    want = oracle.spread_fixed(s.xyzq, s.recip9, s.nfft, s.order)
    assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} grid points differ"


@pytest.mark.parametrize("name", CASES)
def test_triclinic_fused_equals_staged_and_matches_fp64_oracle(cuda, oracle, name):
    s = _sys(name)
    st = _run(cuda, s, staged=True)
    fu = _run(cuda, s, staged=False)
    assert np.array_equal(fu["force"], st["force"])
    assert fu["energy"] == st["energy"] and fu["energy_self"] == st["energy_self"]
    assert np.array_equal(fu["virial"], st["virial"])
    ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip9, s.nfft, s.order, s.kappa)
    F = fu["force"].astype(np.float64)
    e_rel = abs(fu["energy"] - ref["energy"]) / abs(ref["energy"])
    f_rms = np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())
    v_rel = np.abs(fu["virial"] - ref["virial"]).max() / np.abs(ref["virial"]).max()
    assert e_rel <= ENERGY_REL_TOL, e_rel
    assert f_rms <= FORCE_RMS_TOL, f_rms
    assert v_rel <= VIRIAL_REL_TOL, v_rel
    assert abs(fu["energy_self"] - ref["energy_self"]) <= 1e-9 * abs(ref["energy_self"])


def test_triclinic_force_kinds_agree(cuda):
    s = _sys("tric_p4")
    soa = _run(cuda, s, staged=False, kind="soa")["force"]
    f3 = _run(cuda, s, staged=False, kind="f3")["force"]
    i64 = _run(cuda, s, staged=False, kind="i64")["force"]
    assert np.array_equal(soa, f3)
    assert np.array_equal(i64, np.rint(soa.astype(np.float64) * 2.0 ** 40).astype(np.int64))


def test_singular_box_rejected(cuda):
    from gpu_recip_b200 import CudaPMERecip, _capi
    pme = CudaPMERecip(16, 16, 16, 4)
    x = cuda.zeros((4, 4), device="cuda")
    f = cuda.zeros((4, 3), device="cuda")
    for bad in ([0.1, 0.1, 0, 0.1, 0.1, 0, 0, 0, 0.1], [0.1, float("nan"), 0, 0, 0.1, 0, 0, 0, 0.1]):
        with pytest.raises(_capi.PMEError) as e:
            pme.eval(bad, x, 4, 0.3, True, True, f, 1)
        assert e.value.status == _capi.PME_EINVAL
        with pytest.raises(_capi.PMEError) as e:
            pme.spread_charge(x, 4, bad)
        assert e.value.status == _capi.PME_EINVAL
    pme.close()
