"""pme_eval_host: the fused evaluation from page-locked host coordinates to page-locked host
forces.  The evaluation reads the coordinates over the bus in index order instead of the previous
evaluation's bin order; the charge grid is exact int64, so forces, energy and virial must equal
pme_eval's with device buffers bit for bit, in both float force layouts and for any box."""
import ctypes

import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


def _record(pme):
    pme.energy_virial.copyToHost()
    return pme.energy_virial.getEnergy("recip"), pme.energy_virial.getVirial()


@pytest.mark.parametrize("system", ["water8k_64_p4", "dodec_64_p4", "water1k_32"])
def test_eval_host_equals_device_eval(cuda, system):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride, _capi as C
    s = {"water8k_64_p4": lambda: S.config_production(4), "dodec_64_p4": lambda: S.config_triclinic(4),
         "water1k_32": S.config_small}[system]()
    n = s.natom
    st = force_stride(n)
    pme = CudaPMERecip(*s.nfft, s.order)
    x_dev = torch.from_numpy(s.xyzq).cuda()
    f_dev = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    pme.energy_virial.clear()
    pme.eval(s.recip9, x_dev, n, s.kappa, True, True, f_dev, st)
    torch.cuda.synchronize()
    e0, v0 = _record(pme)
    ref = f_dev.cpu().numpy().reshape(3, st)

    x_host = torch.from_numpy(s.xyzq.copy()).pin_memory()
    # SoA with stride padding: the padding is left as the caller had it
    f_host = torch.full((3 * st,), 7.0, dtype=torch.float32).pin_memory()
    for rep in range(3):   # repeated calls: the device eval's bin order is never used for host input
        pme.energy_virial.clear()
        pme.eval_host(s.recip9, x_host, n, s.kappa, True, True, f_host, st)
        torch.cuda.synchronize()
        e1, v1 = _record(pme)
        got = f_host.numpy().reshape(3, st)
        assert np.array_equal(got[:, :n], ref[:, :n]), rep
        assert np.all(got[:, n:] == 7.0)
        assert e1 == e0 and np.array_equal(v1, v0)

    # float3 layout
    f3 = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    pme.eval_host(s.recip9, x_host, n, s.kappa, False, False, f3, 1, kind=C.PME_FORCE_F32X3)
    torch.cuda.synchronize()
    assert np.array_equal(f3.numpy(), ref[:, :n].T)

    # a device evaluation after host ones still matches (the bin order is rebuilt as needed)
    f_dev.zero_()
    pme.eval(s.recip9, x_dev, n, s.kappa, False, False, f_dev, st)
    torch.cuda.synchronize()
    assert np.array_equal(f_dev.cpu().numpy().reshape(3, st)[:, :n], ref[:, :n])


def test_eval_host_rejects_pageable_memory_and_int64(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride, _capi as C
    s = S.config_small()
    n = s.natom
    st = force_stride(n)
    pme = CudaPMERecip(*s.nfft, s.order)
    lib = pme._lib
    x_pageable = np.ascontiguousarray(s.xyzq)
    f_pinned = torch.zeros(3 * st, dtype=torch.float32).pin_memory()
    rc = lib.pme_eval_host(pme._h, C.dbl9(s.recip9), x_pageable.ctypes.data_as(ctypes.c_void_p), n,
                           s.kappa, 1, 1, C.PME_FORCE_F32_SOA, ctypes.c_void_p(f_pinned.data_ptr()), st)
    assert rc == C.PME_EINVAL
    x_pinned = torch.from_numpy(s.xyzq.copy()).pin_memory()
    f_pageable = np.zeros(3 * st, dtype=np.float32)
    rc = lib.pme_eval_host(pme._h, C.dbl9(s.recip9), ctypes.c_void_p(x_pinned.data_ptr()), n, s.kappa, 1, 1,
                           C.PME_FORCE_F32_SOA, f_pageable.ctypes.data_as(ctypes.c_void_p), st)
    assert rc == C.PME_EINVAL
    f64 = torch.zeros(3 * st, dtype=torch.int64).pin_memory()
    with pytest.raises(C.PMEError) as e:
        pme.eval_host(s.recip9, x_pinned, n, s.kappa, True, True, f64, st)
    assert e.value.status == C.PME_EUNSUPPORTED
    with pytest.raises(ValueError):
        pme.eval_host(s.recip9, x_pinned.cuda(), n, s.kappa, True, True, f_pinned, st)


def test_eval_host_without_atoms_is_a_no_op(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip
    s = S.config_small()
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.zeros((1, 4), dtype=torch.float32).pin_memory()
    f = torch.full((3,), 2.0, dtype=torch.float32).pin_memory()
    pme.energy_virial.clear()
    pme.eval_host(s.recip9, x, 0, s.kappa, True, True, f, 1)
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    assert pme.energy_virial.getEnergy("recip") == 0.0
    assert np.all(f.numpy() == 2.0)
