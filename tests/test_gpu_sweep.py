"""Seeded sweep over grid shapes (2/3/5-smooth lengths from 16 to 512, every radix mix), spline
orders, atom counts, box shapes and kappa: the fused evaluation matches the FP64 oracle within
the tolerances and equals the staged reference-style calls bit for bit."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

SMOOTH = [16, 18, 20, 24, 25, 27, 30, 32, 36, 40, 45, 48, 50, 54, 60, 64, 72, 75, 80, 81, 90, 96, 100, 120, 128]


def _case(i):
    rng = np.random.default_rng(1000 + i)
    order = int(rng.choice([4, 6, 8]))
    nfft = [int(rng.choice([n for n in SMOOTH if n >= order])) for _ in range(3)]
    if i == 0:
        nfft = [512, 16, 18]          # longest supported x (8 x 8 x 8 stages), small row blocks
    if i == 1:
        nfft = [20, 480, 16]          # long y: separate y/z passes
    box = tuple(float(n) * float(rng.uniform(0.8, 1.2)) for n in nfft)
    waters = int(rng.integers(30, 1500))
    x = S.water_box(waters, box, 2000 + i)
    kappa = float(rng.uniform(0.25, 0.4))
    return S.PmeSystem(f"sweep{i}_{nfft[0]}x{nfft[1]}x{nfft[2]}_p{order}", x, box, tuple(nfft), order, kappa)


@pytest.mark.parametrize("i", range(14))
def test_sweep(cuda, oracle, i):
    from test_gpu_parity import ENERGY_REL_TOL, FORCE_RMS_TOL, VIRIAL_REL_TOL, _rel_rms, _run
    s = _case(i)
    a = _run(cuda, s, staged=True)
    b = _run(cuda, s)
    assert np.array_equal(a["force"], b["force"]), s.name
    assert a["energy"] == b["energy"] and np.array_equal(a["virial"], b["virial"]), s.name
    ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
    assert _rel_rms(b["force"], ref["force"]) <= FORCE_RMS_TOL, s.name
    assert abs(b["energy"] - ref["energy"]) <= ENERGY_REL_TOL * abs(ref["energy"]), s.name
    v = np.abs(b["virial"] - ref["virial"]).max() / np.abs(ref["virial"]).max()
    assert v <= VIRIAL_REL_TOL, (s.name, v)
