"""The large configuration: 336,000 TIP3P-geometry waters (1,008,000 atoms), 216 A cube, 216^3
grid (2^3 3^3), order 6, kappa 0.30 -- parity with the FP64 oracle at full size, the bit-exact
fixed-point grid, and staged == fused."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large():
    return S.config_large()


def _fused(torch, s, pme=None):
    from gpu_recip_b200 import CudaPMERecip, force_stride
    pme = pme or CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(s.xyzq).cuda()
    st = force_stride(s.natom)
    f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    pme.energy_virial.clear()
    pme.eval_ortho([1.0 / b for b in s.box], x, s.natom, s.kappa, True, True, f, st)
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    F = f.view(3, st)[:, :s.natom].T.cpu().numpy().astype(np.float64)
    return F, pme.energy_virial.getEnergy("recip"), pme.energy_virial.getVirial(), pme, x, f, st


def test_large_matches_fp64_oracle(cuda, oracle, large):
    s = large
    F, e, v, *_ = _fused(cuda, s)
    ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
    f_rms = np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())
    assert f_rms <= 1e-5, f_rms
    assert abs(e - ref["energy"]) / abs(ref["energy"]) <= 1e-6
    assert np.abs(v - ref["virial"]).max() / np.abs(ref["virial"]).max() <= 1e-5


def test_large_grid_bit_exact_and_staged_equals_fused(cuda, oracle, large):
    from gpu_recip_b200 import recip_from_box
    s = large
    F, e, v, pme, x, f, st = _fused(cuda, s)
    recip = recip_from_box(s.box)
    pme.spread_charge(x, s.natom, recip)
    assert np.array_equal(pme.charge_grid_fixed(), oracle.spread_fixed(s.xyzq, s.recip3, s.nfft, s.order))
    pme.energy_virial.clear()
    pme.r2c_fft()
    pme.scalar_sum(recip, s.kappa, True, True)
    pme.c2r_fft()
    f2 = cuda.zeros_like(f)
    pme.gather_force(x, s.natom, recip, st, f2)
    cuda.cuda.synchronize()
    pme.energy_virial.copyToHost()
    assert np.array_equal(f.cpu().numpy(), f2.cpu().numpy())
    assert pme.energy_virial.getEnergy("recip") == e
    assert np.array_equal(pme.energy_virial.getVirial(), v)
