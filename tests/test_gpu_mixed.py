"""Batches and served requests that mix every spline order and force-output kind, plus an empty
system: each system's results equal the plain single-system path bit for bit."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

KINDS = {"soa": 0, "aos": 1, "i64": 2}


def _systems():
    b = S.batch_systems(5, seed=29, min_waters=216, max_waters=1500)
    out = []
    for i, (s, order) in enumerate(zip(b, (4, 6, 8, 6, 4))):
        out.append(S.PmeSystem(f"{s.name}_p{order}", s.xyzq, s.box, s.nfft, order, 0.33))
    out.append(S.PmeSystem("empty", np.zeros((0, 4), np.float32), (20.0, 20.0, 20.0), (24, 24, 24), 6, 0.3))
    return out


def _force(torch, s, kind):
    from gpu_recip_b200 import force_stride
    n = max(s.natom, 1)
    if kind == "aos":
        return torch.zeros((n, 3), dtype=torch.float32, device="cuda"), 1
    st = force_stride(n, 8 if kind == "i64" else 4)
    dt = torch.int64 if kind == "i64" else torch.float32
    return torch.zeros(3 * st, dtype=dt, device="cuda"), st


def _host(f, kind, n, st):
    if kind == "aos":
        return f.cpu().numpy()[:n]
    return f.view(3, st)[:, :n].T.cpu().numpy()


def test_batch_mixing_orders_and_force_kinds(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, PmeBatch
    systems = _systems()
    kinds = ["soa", "aos", "i64", "i64", "aos", "soa"]
    specs, outs = [], []
    for s, k in zip(systems, kinds):
        f, st = _force(torch, s, k)
        x = torch.from_numpy(np.ascontiguousarray(s.xyzq)).cuda() if s.natom else torch.zeros((1, 4), device="cuda")
        outs.append((f, st, x))
        specs.append(dict(nfft=s.nfft, order=s.order, box=s.box, kappa=s.kappa, xyzq=x, natom=s.natom,
                          force=f, stride=st, force_kind=KINDS[k]))
    b = PmeBatch(specs)
    b.clear_energy_virial()
    b.eval()
    ev = b.energy_virial()
    for i, (s, k) in enumerate(zip(systems, kinds)):
        f, st, x = outs[i]
        pme = CudaPMERecip(*s.nfft, s.order)
        g, gst = _force(torch, s, k)
        pme.energy_virial.clear()
        pme.eval_ortho([1.0 / v for v in s.box], x, s.natom, s.kappa, True, True, g, gst, KINDS[k])
        torch.cuda.synchronize()
        pme.energy_virial.copyToHost()
        assert ev[i, 0] == pme.energy_virial.getEnergy("recip"), s.name
        assert ev[i, 1] == pme.energy_virial.getEnergy("self"), s.name
        assert np.array_equal(ev[i, 2:].reshape(3, 3), pme.energy_virial.getVirial()), s.name
        assert np.array_equal(_host(f, k, s.natom, st), _host(g, k, s.natom, gst)), s.name
    assert ev[5, 0] == 0.0 and ev[5, 1] == 0.0


def test_server_mixing_orders_without_energy(cuda):
    from gpu_recip_b200 import PmeServer
    systems = [s for s in _systems() if s.natom]
    srv = PmeServer(1 << 30, max_active=3)
    ids = [srv.submit(s, n_evals=2, sigma=0.02, seed=7 + i) for i, s in enumerate(systems)]
    res = [srv.wait(r, timeout=120) for r in ids]
    srv.close()
    # again, alone and with energies off: the forces are the same bits
    srv = PmeServer(1 << 30, max_active=1)
    for i, (s, r) in enumerate(zip(systems, res)):
        import ctypes
        from gpu_recip_b200 import _capi as C
        ev = np.zeros((2, 11))
        force = np.zeros((s.natom, 3), np.float32)
        req, _x = srv._request(s, 2, 0.02, 7 + i, ev, force, calc_energy=False, calc_virial=False)
        rid = ctypes.c_longlong()
        C.check(srv._lib.pme_server_submit(srv._h, ctypes.byref(req), ctypes.byref(rid)), "submit")
        C.check(srv._lib.pme_server_wait(srv._h, rid, 120.0, None), "wait")
        assert np.array_equal(force, r["force"]), s.name
        assert not ev.any()
    srv.close()
