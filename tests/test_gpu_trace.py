"""The profiling hook (pme_set_trace / pme_batch_set_trace): per-CTA phase stamps land inside the
caller's buffer, the 32 step stamps of a single-system trace after them, nothing past the end, and
a buffer too small for the CTAs asked for is refused before any kernel runs."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

GUARD = -7


def test_trace_stays_inside_the_buffer(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride
    from gpu_recip_b200.pme import TRACE_STEP_STAMPS
    s = S.config_small(seed=9)
    n = s.natom
    st = force_stride(n)
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(s.xyzq).cuda()
    f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    ctas = 512
    used = ctas * 14 + TRACE_STEP_STAMPS
    buf = torch.full((used + 64,), GUARD, dtype=torch.int64, device="cuda")
    buf[:used].zero_()
    pme.set_trace(buf[:used], ctas)
    inv = [1.0 / b for b in s.box]
    pme.eval_ortho(inv, x, n, s.kappa, True, True, f, st)
    pme.set_trace(None)
    torch.cuda.synchronize()
    b = buf.cpu().numpy()
    assert np.all(b[used:] == GUARD)
    ph = b[:ctas * 14].reshape(ctas, 7, 2)
    ran = ph[:, :, 0] > 0
    assert ran[0].any()
    assert np.all(ph[:, :, 1][ran] >= ph[:, :, 0][ran])
    assert (b[ctas * 14:used] > 0).any()   # CTA 0's step stamps
    with pytest.raises(ValueError):
        pme.set_trace(buf[:used - 1], ctas)
    with pytest.raises(ValueError):
        pme.set_trace(buf.to(torch.int32))


def test_batch_trace_stays_inside_the_buffer(cuda):
    torch = cuda
    from gpu_recip_b200 import PmeBatch, force_stride
    systems = S.batch_systems(4, seed=12)
    specs = []
    for sy in systems:
        st = force_stride(sy.natom)
        specs.append(dict(nfft=sy.nfft, order=sy.order, box=sy.box, kappa=sy.kappa,
                          xyzq=torch.from_numpy(sy.xyzq).cuda(),
                          force=torch.zeros(3 * st, dtype=torch.float32, device="cuda"), stride=st))
    bt = PmeBatch(specs)
    ctas = 256
    buf = torch.full((ctas * 14 + 64,), GUARD, dtype=torch.int64, device="cuda")
    buf[:ctas * 14].zero_()
    bt.set_trace(buf[:ctas * 14])
    bt.eval()
    bt.set_trace(None)
    torch.cuda.synchronize()
    b = buf.cpu().numpy()
    assert np.all(b[ctas * 14:] == GUARD)
    ph = b[:ctas * 14].reshape(ctas, 7, 2)
    ran = ph[:, :, 0] > 0
    assert ran[0].any()
    assert np.all(ph[:, :, 1][ran] >= ph[:, :, 0][ran])
