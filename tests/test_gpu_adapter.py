"""The MD-side callers of the path: CudaDomdecRecip::calc with its three force outputs
(CudaDomdecRecip.h:50-81), the int64 output accumulating onto forces already there (as direct-space
forces would be), and the recip node's request loop (CudaDomdecRecipLooper::run) in process."""
import ctypes
import threading

import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


def _fixed(f):
    return np.rint(f.astype(np.float64) * 2.0 ** 40).astype(np.int64)


def test_domdec_recip_three_force_kinds_and_int64_accumulate(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaDomdecRecip, force_stride
    s = S.config_small(seed=5)
    n = s.natom
    rec = CudaDomdecRecip(*s.nfft, s.order, s.kappa)
    x = torch.from_numpy(s.xyzq).cuda()
    inv = [1.0 / b for b in s.box]
    f3 = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    rec.calc(*inv, x, n, True, True, f3)
    st = force_stride(n)
    fs = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    rec.calc(*inv, x, n, True, True, fs, st)
    st8 = force_stride(n, 8)
    prior = np.random.default_rng(3).integers(-2 ** 45, 2 ** 45, size=(3, st8)).astype(np.int64)
    fi = torch.from_numpy(prior.copy().reshape(-1)).cuda()
    rec.calc(*inv, x, n, True, True, fi, st8)
    torch.cuda.synchronize()
    a = f3.cpu().numpy()
    b = fs.view(3, st)[:, :n].T.cpu().numpy()
    assert np.array_equal(a, b)
    got = fi.view(3, st8).cpu().numpy()
    want = prior.copy()
    want[:, :n] += _fixed(a).T
    assert np.array_equal(got, want)


def test_int64_accumulate_then_convert_as_the_md_step(cuda):
    """The end of an MD step (CudaPMEForcefield.cu:514): reciprocal forces accumulated in int64
    onto forces already there, then Force<long long>::convert to double (in place and out of
    place), to float, and convert_add of a float force array: every value is the accumulated
    int64 rounded once to the type times 2^-40, bit for bit."""
    torch = cuda
    from gpu_recip_b200 import CudaDomdecRecip, force_convert, force_convert_add, force_stride
    s = S.config_small(seed=7)
    n = s.natom
    rec = CudaDomdecRecip(*s.nfft, s.order, s.kappa)
    x = torch.from_numpy(s.xyzq).cuda()
    inv = [1.0 / b for b in s.box]
    f3 = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    rec.calc(*inv, x, n, True, True, f3)
    st8 = force_stride(n, 8)
    prior = np.random.default_rng(4).integers(-2 ** 45, 2 ** 45, size=(3, st8)).astype(np.int64)
    fi = torch.from_numpy(prior.copy().reshape(-1)).cuda()
    rec.calc(*inv, x, n, True, True, fi, st8)
    torch.cuda.synchronize()
    acc = prior.copy()
    acc[:, :n] += _fixed(f3.cpu().numpy()).T          # prior + rint(F 2^40)
    assert np.array_equal(fi.view(3, st8).cpu().numpy(), acc)
    want64 = acc[:, :n].astype(np.float64) * 2.0 ** -40
    want32 = acc[:, :n].astype(np.float32) * np.float32(2.0 ** -40)
    # out of place, other strides; the padding of the output is left alone
    so = force_stride(n, 8) + 64
    out64 = torch.full((3 * so,), -7.0, dtype=torch.float64, device="cuda")
    force_convert(fi, st8, n, out64, so)
    out32 = torch.full((3 * so,), -7.0, dtype=torch.float32, device="cuda")
    force_convert(fi, st8, n, out32, so)
    torch.cuda.synchronize()
    o64 = out64.view(3, so).cpu().numpy()
    o32 = out32.view(3, so).cpu().numpy()
    assert np.array_equal(o64[:, :n], want64) and np.all(o64[:, n:] == -7.0)
    assert np.array_equal(o32[:, :n], want32) and np.all(o32[:, n:] == -7.0)
    # convert_add of a float32 array (the reference's reduce_add_force<long long, double, float>)
    add = torch.from_numpy(np.random.default_rng(5).standard_normal((3, st8)).astype(np.float32).reshape(-1)).cuda()
    fa = fi.clone()
    d = force_convert_add(fa, st8, n, add)
    # in place: convert<double>() of the int64 array itself
    d2 = force_convert(fi, st8, n)
    torch.cuda.synchronize()
    assert np.array_equal(d2.view(3, st8)[:, :n].cpu().numpy(), want64)
    want_add = want64 + add.view(3, st8)[:, :n].cpu().numpy().astype(np.float64)
    assert np.array_equal(d.view(3, st8)[:, :n].cpu().numpy(), want_add)


def test_force_convert_rejects_bad_arguments(cuda):
    torch = cuda
    from gpu_recip_b200 import _capi, force_convert
    fi = torch.zeros(3 * 64, dtype=torch.int64, device="cuda")
    f32 = fi.view(torch.float64)[:96].view(torch.float32)   # overlaps fi
    with pytest.raises(_capi.PMEError):
        force_convert(fi, 64, 32, f32, 64)                  # overlapping float output
    with pytest.raises(_capi.PMEError):
        force_convert(fi, 64, 65)                           # ncoord beyond the stride
    out = torch.zeros(3 * 64, dtype=torch.float32, device="cuda")
    with pytest.raises(_capi.PMEError):
        force_convert(fi, 64, 32, out, 16)                  # output stride below ncoord


@pytest.mark.parametrize("native", [False, True])
def test_recip_looper_serves_a_direct_node(cuda, native):
    """The recip node's loop (CudaDomdecRecipLooper::run) in Python and in C++ behind the C ABI
    (pme_recip_loop_run): every reply equals the MD adapter's own evaluation bit for bit."""
    torch = cuda
    from gpu_recip_b200 import CudaDomdecRecip
    from gpu_recip_b200.looper import InProcessRecipComm, NativeRecipLooper, RecipLooper
    s = S.config_small(seed=9)
    comm = InProcessRecipComm(timeout=120.0)
    looper = (NativeRecipLooper if native else RecipLooper)(comm, *s.nfft, s.order, s.kappa)
    out = {}
    th = threading.Thread(target=lambda: out.setdefault("steps", looper.run()))
    th.start()
    rng = np.random.default_rng(11)
    ref = CudaDomdecRecip(*s.nfft, s.order, s.kappa)
    try:
        for step, (scale, e, v) in enumerate([(1.0, True, True), (1.01, False, True), (0.995, True, False)]):
            box = [b * scale for b in s.box]
            x = s.xyzq.copy()
            x[:, :3] += rng.normal(0.0, 0.05, size=(s.natom, 3)).astype(np.float32)
            n = s.natom - 7 * step                      # the coordinate count may change per step
            xd = torch.from_numpy(x[:n].copy()).cuda()
            comm.send_header(n, *[1.0 / b for b in box], e, v)
            comm.send_coord(xd)
            reply = comm.recv_force()
            want = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
            ev = ref.pme.energy_virial
            ev.clear()
            ref.calc(*[1.0 / b for b in box], xd, n, e, v, want)
            torch.cuda.synchronize()
            ev.copyToHost()
            assert np.array_equal(reply.force.cpu().numpy(), want.cpu().numpy())
            assert reply.energy_virial[0] == ev.getEnergy("recip")
            assert np.array_equal(reply.energy_virial[2:].reshape(3, 3), ev.getVirial())
    finally:
        comm.send_stop()
        th.join(timeout=120)
    assert not th.is_alive() and out["steps"] == 3


def test_energy_virial_mirror_holds_each_evaluations_own_record(cuda):
    """pme_set_energy_virial_mirror: each fused evaluation writes its own record to pinned host
    memory while the device record keeps accumulating."""
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, _capi, force_stride
    s = S.config_small(seed=12)
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(s.xyzq).cuda()
    st = force_stride(s.natom)
    f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    inv = [1.0 / b for b in s.box]
    mirror = torch.zeros(11, dtype=torch.float64).pin_memory()
    pme.set_energy_virial_mirror(mirror)
    ev = pme.energy_virial
    ev.clear()
    pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, st)
    torch.cuda.synchronize()
    first = mirror.numpy().copy()
    ev.copyToHost()
    assert first[0] == ev.getEnergy("recip") and first[1] == ev.getEnergy("self")
    assert np.array_equal(first[2:].reshape(3, 3), ev.getVirial())
    pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, st)   # no clear: the record doubles
    torch.cuda.synchronize()
    ev.copyToHost()
    assert np.array_equal(mirror.numpy(), first)
    assert ev.getEnergy("recip") == 2 * first[0]
    pme.eval_ortho(inv, x, s.natom, s.kappa, False, False, f, st)   # nothing asked: zeros
    torch.cuda.synchronize()
    assert not mirror.numpy().any()
    pme.set_energy_virial_mirror(None)
    with pytest.raises(_capi.PMEError) as e:   # device memory is not a host mirror
        _capi.check(pme._lib.pme_set_energy_virial_mirror(pme._h, ctypes.c_void_p(f.data_ptr())), "mirror")
    assert e.value.status == _capi.PME_EINVAL
    pme.close()
