"""GPU test of pme_spread_charge_noalloc, the spreading entry point that allocates no device
memory (for hosts whose own memory manager owns the device and forbids cudaMalloc from plug-ins,
and for latency-critical loops that cannot take allocator locks).  It is compared through the C ABI
with the existing pme_spread_charge grid, exactly as the other grid tests compare (bit for bit),
on two calls in a row, and the device's free memory is checked unchanged around calls after the
first.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


def _noalloc(lib, x, natom, recip, nfft, order, out, stream=0):
    xp = ctypes.c_void_p(x.data_ptr() if natom else 0)
    return lib.pme_spread_charge_noalloc(xp, natom, (ctypes.c_double * 9)(*recip), int(nfft[0]),
                                         int(nfft[1]), int(nfft[2]), int(order),
                                         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def _existing_grid(torch, s, x):
    from gpu_recip_b200 import CudaPMERecip, recip_from_box
    pme = CudaPMERecip(*s.nfft, s.order)
    pme.spread_charge(x, s.natom, recip_from_box(s.box))
    return pme.charge_grid()


def test_noalloc_spread_matches_existing_entry_point(cuda):
    torch = cuda
    from gpu_recip_b200 import _capi, recip_from_box
    lib = _capi.load()
    big = S.config_production(4)
    box = (40.0, 36.0, 33.0)
    small = S.PmeSystem("p6", S.water_box(1500, box, 41), box, (48, 40, 36), 6, 0.32)
    # two calls in a row, alternating sizes, so a stale grid from the previous call would show
    for s in (big, small, big):
        x = torch.from_numpy(s.xyzq).cuda()
        nx, ny, nz = s.nfft
        want = _existing_grid(torch, s, x)
        for call in range(2):
            out = torch.full((nz * ny * nx,), float("nan"), dtype=torch.float32, device="cuda")
            rc = _noalloc(lib, x, s.natom, recip_from_box(s.box), s.nfft, s.order, out)
            assert rc == _capi.PME_OK, lib.pme_last_error_string()
            torch.cuda.synchronize()
            got = out.cpu().numpy().reshape(nz, ny, nx)
            assert np.array_equal(got, want), (s.name, call, np.abs(got - want).max())


def test_noalloc_spread_allocates_no_device_memory(cuda):
    torch = cuda
    from gpu_recip_b200 import _capi, recip_from_box
    lib = _capi.load()
    s = S.config_small()
    x = torch.from_numpy(s.xyzq).cuda()
    nx, ny, nz = s.nfft
    out = torch.empty(nz * ny * nx, dtype=torch.float32, device="cuda")
    recip = recip_from_box(s.box)
    # the first call may load the kernels; the later ones must leave device memory alone
    assert _noalloc(lib, x, s.natom, recip, s.nfft, s.order, out) == _capi.PME_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _noalloc(lib, x, s.natom, recip, s.nfft, s.order, out) == _capi.PME_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_grids_beyond_its_limit(cuda):
    torch = cuda
    from gpu_recip_b200 import _capi
    lib = _capi.load()
    out = torch.zeros(1, dtype=torch.float32, device="cuda")
    x = torch.zeros((1, 4), dtype=torch.float32, device="cuda")
    rc = _noalloc(lib, x, 1, [0.01, 0, 0, 0, 0.01, 0, 0, 0, 0.01], (128, 128, 128), 4, out)
    assert rc == _capi.PME_EINVAL
    assert b"1048576" in lib.pme_last_error_string()
