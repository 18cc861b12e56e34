"""The reference's two-charge probe (gpu_pair.cu:81-140) on the GPU: charges -1 and +1 a distance
r apart along x in a cubic box, staged spread / R2C / solve / C2R / gather, against the exact
reciprocal Ewald sum of the same pair; the forces are equal and opposite along x."""
import numpy as np
import pytest

from tests.test_oracle_triclinic import ewald_recip

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("r", [0.5, 1.5, 4.0, 9.0])
def test_two_charge_probe_matches_exact_ewald(cuda, r):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride, recip_from_box
    L, kappa, nfft, order = 20.0, 0.35, 40, 8
    x = np.array([[-r / 2 + L / 2, L / 2, L / 2, -1.0], [r / 2 + L / 2, L / 2, L / 2, 1.0]])
    pme = CudaPMERecip(nfft, nfft, nfft, order)
    xd = torch.from_numpy(x.astype(np.float32)).cuda()
    st = force_stride(2)
    f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    recip = recip_from_box((L, L, L))
    ev = pme.energy_virial
    ev.clear()
    pme.spread_charge(xd, 2, recip)
    pme.r2c_fft()
    pme.scalar_sum(recip, kappa, True, True)
    pme.c2r_fft()
    pme.gather_force(xd, 2, recip, st, f)
    torch.cuda.synchronize()
    ev.copyToHost()
    F = f.view(3, st)[:, :2].T.cpu().numpy().astype(np.float64)
    E_ref, W_ref, F_ref = ewald_recip(x.astype(np.float32).astype(np.float64), np.diag([L, L, L]), kappa, mmax=16)
    assert abs(ev.getEnergy("recip") - E_ref) <= 1e-5 * abs(E_ref)
    assert np.abs(F - F_ref).max() <= 1e-4 * np.abs(F_ref).max()
    assert np.abs(ev.getVirial() - W_ref).max() <= 1e-4 * np.abs(W_ref).max()
    assert abs(F[0, 0] + F[1, 0]) <= 1e-5 * abs(F[0, 0])          # equal and opposite along x
    assert np.abs(F[:, 1:]).max() <= 1e-4 * abs(F[0, 0])          # nothing across
    pme.close()
