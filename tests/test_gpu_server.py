"""The request server (pme_server_*): continuous batching of PME evaluations.

Each request's results depend only on the request: the same request gives the same bits alone
and in a mix of requests that arrive while others run; with no jitter every evaluation equals
the plain single-system path (pme_eval_ortho) exactly."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _plain(torch, s):
    from gpu_recip_b200 import CudaPMERecip
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(np.ascontiguousarray(s.xyzq)).cuda()
    f = torch.zeros((s.natom, 3), dtype=torch.float32, device="cuda")
    pme.energy_virial.clear()
    pme.eval_ortho([1.0 / b for b in s.box], x, s.natom, s.kappa, True, True, f, 1)
    torch.cuda.synchronize()
    rec = np.zeros(11)
    pme.energy_virial.copyToHost()
    rec[0] = pme.energy_virial.getEnergy("recip")
    rec[1] = pme.energy_virial.getEnergy("self")
    rec[2:] = pme.energy_virial.getVirial().reshape(-1)
    return rec, f.cpu().numpy()


def test_server_without_jitter_equals_plain_path(cuda):
    from gpu_recip_b200 import PmeServer
    systems = S.batch_systems(6, seed=13)
    srv = PmeServer(2 * GiB, max_active=8)
    ids = [srv.submit(s, n_evals=3, sigma=0.0, seed=i) for i, s in enumerate(systems)]
    for s, rid in zip(systems, ids):
        got = srv.wait(rid, timeout=120)
        rec, force = _plain(cuda, s)
        for k in range(3):       # every evaluation of an unjittered request is the same
            assert np.array_equal(got["ev"][k], rec), (s.name, k)
        assert np.array_equal(got["force"], force)
    st = srv.stats()
    assert st["completed"] == 6 and st["evals"] == 18
    srv.close()


def test_each_result_same_alone_and_in_the_mix(cuda):
    from gpu_recip_b200 import PmeServer
    rng = np.random.default_rng(5)
    systems = S.batch_systems(24, seed=17)
    n_evals = [int(v) for v in rng.integers(1, 12, size=len(systems))]
    # alone: one request at a time
    alone = []
    srv = PmeServer(2 * GiB, max_active=1)
    for i, s in enumerate(systems[:8]):
        alone.append(srv.wait(srv.submit(s, n_evals=n_evals[i], sigma=0.05, seed=100 + i), timeout=120))
    srv.close()
    # in the mix: all 24 submitted together, uneven evaluation counts, a memory budget that makes
    # later requests wait for earlier ones to leave
    budget = sum(sorted(PmeServer.request_device_bytes(s, n) for s, n in zip(systems, n_evals))[-6:])
    srv = PmeServer(budget, max_active=5)
    ids = [srv.submit(s, n_evals=n_evals[i], sigma=0.05, seed=100 + i) for i, s in enumerate(systems)]
    mixed = [srv.wait(rid, timeout=300) for rid in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(systems)
    assert st["steps"] < sum(n_evals)          # requests shared steps
    for a, m in zip(alone, mixed[:8]):
        assert np.array_equal(a["ev"], m["ev"])
        assert np.array_equal(a["force"], m["force"])
    # jitter changes the evaluations of a request (and differs between seeds)
    multi = [m for m, n in zip(mixed, n_evals) if n >= 2]
    assert all(not np.array_equal(m["ev"][0], m["ev"][1]) for m in multi)


_M64 = (1 << 64) - 1


def _mix64(z):
    """splitmix64 finaliser on Python ints (mod 2^64), as the server's jitter generator."""
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def _jittered(xyzq, seed, k, sigma):
    """The coordinates of a request's evaluation k, restated on the host: each coordinate plus
    sigma times a Box-Muller deviate of the counter (seed, k, atom, axis).  The deviate is formed
    in FP64 here (FP32 on the device), so a coordinate can differ by one FP32 ulp, far inside the
    FP64 tolerances the results are checked against."""
    x = np.array(xyzq, dtype=np.float32, copy=True)
    sig = np.float32(sigma)
    for i in range(x.shape[0]):
        for axis in range(3):
            h = _mix64(seed ^ _mix64(((k & 0xFFFFFFFF) << 34) ^ ((i & 0xFFFFFFFF) << 2) ^ axis))
            u1 = ((h >> 40) + 1.0) / 16777216.0
            u2 = ((h >> 16) & 0xFFFFFF) / 16777216.0
            g = np.float32(np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2))
            x[i, axis] = np.float32(x[i, axis] + np.float32(sig * g))
    return x


def test_jittered_evaluations_match_the_fp64_oracle(cuda, oracle):
    """Each evaluation of a jittered request, against the FP64 oracle on the same jittered
    coordinates (restated on the host): energy, virial and the last evaluation's forces."""
    from gpu_recip_b200 import PmeServer
    systems = [S.batch_systems(3, seed=29, min_waters=216, max_waters=900)[i] for i in (0, 2)]
    srv = PmeServer(2 * GiB, max_active=4)
    seeds = [0x5EED0001, 0x0BADC0DE12345]
    ids = [srv.submit(s, n_evals=3, sigma=0.05, seed=sd) for s, sd in zip(systems, seeds)]
    got = [srv.wait(rid, timeout=120) for rid in ids]
    srv.close()
    for s, sd, g in zip(systems, seeds, got):
        for k in range(3):
            xk = _jittered(s.xyzq, sd, k, 0.05)
            assert not np.array_equal(xk, s.xyzq)
            ref = oracle.evaluate(xk.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
            e = g["ev"][k]
            assert abs(e[0] - ref["energy"]) <= 1e-6 * abs(ref["energy"]), (s.name, k, e[0], ref["energy"])
            vir = e[2:].reshape(3, 3)
            assert np.abs(vir - ref["virial"]).max() <= 1e-5 * np.abs(ref["virial"]).max(), (s.name, k)
            if k == 2:
                F = g["force"].astype(np.float64)
                rms = np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())
                assert rms <= 1e-5, (s.name, rms)


def test_server_rejects_requests_larger_than_its_memory(cuda):
    from gpu_recip_b200 import PmeServer, _capi
    srv = PmeServer(8 << 20, max_active=2)
    with pytest.raises(_capi.PMEError) as e:
        srv.submit(S.config_production(4), n_evals=1)
    assert e.value.status == _capi.PME_ENOMEM
    srv.close()
