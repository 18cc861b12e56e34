"""GPU tests of the fused persistent evaluation: batches of uneven systems in one launch, results
identical alone and in the mix, CUDA-graph capture, and bounded-wait failure detection."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


def _mixed_systems():
    b = S.batch_systems(6, seed=17, min_waters=216, max_waters=2000)
    b[1] = S.PmeSystem(b[1].name, b[1].xyzq, b[1].box, b[1].nfft, 6, 0.35)   # mixed orders
    b.append(S.PmeSystem("odd", S.water_box(400, (22.0, 23.5, 25.0), 5), (22.0, 23.5, 25.0), (25, 24, 27), 4, 0.32))
    return b


def _single(torch, s):
    from gpu_recip_b200 import CudaPMERecip, force_stride
    pme = CudaPMERecip(*s.nfft, s.order)
    x = torch.from_numpy(s.xyzq).cuda()
    stride = force_stride(s.natom)
    f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
    pme.energy_virial.clear()
    pme.eval_ortho([1.0 / b for b in s.box], x, s.natom, s.kappa, True, True, f, stride)
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    ev = pme.energy_virial
    F = f.view(3, stride)[:, : s.natom].T.cpu().numpy()
    return F, ev.getEnergy("recip"), ev.getEnergy("self"), ev.getVirial()


def _batch(torch, systems):
    from gpu_recip_b200 import PmeBatch, force_stride
    specs, fs = [], []
    for s in systems:
        x = torch.from_numpy(s.xyzq).cuda()
        stride = force_stride(s.natom)
        f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
        fs.append((f, stride))
        specs.append(dict(nfft=s.nfft, order=s.order, box=s.box, kappa=s.kappa, xyzq=x, force=f,
                          stride=stride))
    b = PmeBatch(specs)
    b.clear_energy_virial()
    b.eval()
    ev = b.energy_virial()
    out = []
    for i, s in enumerate(systems):
        f, stride = fs[i]
        out.append((f.view(3, stride)[:, : s.natom].T.cpu().numpy(), ev[i, 0], ev[i, 1], ev[i, 2:].reshape(3, 3)))
    return out, b, specs


def test_batch_results_identical_alone_and_in_mix(cuda):
    systems = _mixed_systems()
    mixed, _, _ = _batch(cuda, systems)
    for s, got in zip(systems, mixed):
        alone = _single(cuda, s)
        assert np.array_equal(got[0], alone[0]), s.name
        assert got[1] == alone[1] and got[2] == alone[2], s.name
        assert np.array_equal(got[3], alone[3]), s.name


def test_batch_matches_oracle(cuda, oracle):
    systems = _mixed_systems()
    mixed, _, _ = _batch(cuda, systems)
    for s, got in zip(systems, mixed):
        ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
        F = got[0].astype(np.float64)
        rms = np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())
        assert rms <= 1e-5, (s.name, rms)
        assert abs(got[1] - ref["energy"]) <= 1e-6 * abs(ref["energy"]), s.name
        assert abs(got[2] - ref["energy_self"]) <= 1e-12 * abs(ref["energy_self"]), s.name


def test_batch_repeat_and_update(cuda):
    """Repeated launches give the same answer; a changed box/coordinate set takes effect after commit."""
    systems = _mixed_systems()[:3]
    first, b, specs = _batch(cuda, systems)
    b.clear_energy_virial()
    b.eval()
    again = b.energy_virial()
    for i in range(len(systems)):
        assert again[i, 0] == first[i][1]
    s = systems[0]
    new_box = tuple(1.01 * v for v in s.box)
    b.set_system(0, box=new_box)
    b.commit()
    b.clear_energy_virial()
    b.eval()
    upd = b.energy_virial()
    alone = _single(cuda, S.PmeSystem("u", s.xyzq, new_box, s.nfft, s.order, s.kappa))
    assert upd[0, 0] == alone[1]
    assert upd[1, 0] == first[1][1]


def test_eval_captured_in_cuda_graph(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride
    s = S.config_small(seed=8)
    eager = _single(torch, s)
    stream = torch.cuda.Stream()
    pme = CudaPMERecip(*s.nfft, s.order, stream=stream)
    x = torch.from_numpy(s.xyzq).cuda()
    stride = force_stride(s.natom)
    f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
    inv = [1.0 / b for b in s.box]
    with torch.cuda.stream(stream):     # warm up (module load) outside the capture
        pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, stride)
    stream.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        pme.energy_virial.clear()
        pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, stride)
    for _ in range(3):
        f.zero_()
        g.replay()
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    assert np.array_equal(f.view(3, stride)[:, : s.natom].T.cpu().numpy(), eager[0])
    assert pme.energy_virial.getEnergy("recip") == eager[1]
    del g


def test_barrier_timeout_is_reported_not_hung(cuda):
    """A CTA that never arrives at a grid barrier: the others' bounded waits run out, the device
    status says so, the host gets PME_ETIMEOUT, and after the reset the handle works again."""
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, _capi, force_stride
    s = S.config_small(seed=9)
    eager = _single(torch, s)
    pme = CudaPMERecip(*s.nfft, s.order)
    pme.set_barrier_spin_limit(20000)
    x = torch.from_numpy(s.xyzq).cuda()
    stride = force_stride(s.natom)
    f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
    inv = [1.0 / b for b in s.box]
    pme.set_fault_injection(_capi.PME_INJECT_SKIP_BARRIER)
    pme.energy_virial.clear()
    pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, stride)
    # the sticky status makes the next evaluation a no-op and is reported on read-back
    pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, stride)
    with pytest.raises(_capi.PMEError) as e:
        pme.energy_virial.copyToHost()
    assert e.value.status == _capi.PME_ETIMEOUT
    with pytest.raises(_capi.PMEError) as e:
        pme.get_status()
    assert e.value.status == _capi.PME_ETIMEOUT
    # recovered
    pme.set_fault_injection(_capi.PME_INJECT_NONE)
    pme.set_barrier_spin_limit(1 << 22)
    assert pme.get_status() == 0
    pme.energy_virial.clear()
    pme.eval_ortho(inv, x, s.natom, s.kappa, True, True, f, stride)
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    assert np.array_equal(f.view(3, stride)[:, : s.natom].T.cpu().numpy(), eager[0])
    assert pme.energy_virial.getEnergy("recip") == eager[1]


def test_benched_256_system_batch_matches_oracle(cuda, oracle):
    """The batched workload exactly as the benchmark times it: 256 water boxes of 648-24,000 atoms
    and 24^3-64^3 grids (seed 4), the launch shape picked by the batch autotuner, the step replayed
    from a CUDA graph.  A seeded subset of 32 systems (with the smallest and largest atom counts
    and grids, chosen as the benchmark's own parity block chooses them) against the FP64 oracle;
    every system's energy is finite."""
    torch = cuda
    import bench
    from gpu_recip_b200 import PmeBatch, force_stride
    systems = S.batch_systems(256, seed=4)
    specs, fs = [], []
    for s in systems:
        x = torch.from_numpy(s.xyzq).cuda()
        stride = force_stride(s.natom)
        f = torch.zeros(3 * stride, dtype=torch.float32, device="cuda")
        fs.append((f, stride))
        specs.append(dict(nfft=s.nfft, order=s.order, box=s.box, kappa=s.kappa, xyzq=x, force=f, stride=stride))
    stream = torch.cuda.Stream()
    b = PmeBatch(specs, stream=stream)
    tune = b.autotune(reps=3)
    assert tune["candidates"] >= 1
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        b.clear_energy_virial()
        b.eval()
    for f, _ in fs:
        f.zero_()
    torch.cuda.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    ev = b.energy_virial()
    del graph
    assert np.all(np.isfinite(ev))
    idx = bench.parity_subset(systems)
    assert len(idx) == 32
    natoms = [s.natom for s in systems]
    assert natoms.index(min(natoms)) in idx and natoms.index(max(natoms)) in idx
    for i in idx:
        s = systems[i]
        f, stride = fs[i]
        F = f.view(3, stride)[:, : s.natom].T.cpu().numpy().astype(np.float64)
        ref = oracle.evaluate(s.xyzq.astype(np.float64), s.recip3, s.nfft, s.order, s.kappa)
        rms = np.sqrt(((F - ref["force"]) ** 2).sum() / (ref["force"] ** 2).sum())
        assert rms <= 1e-5, (s.name, s.natom, s.nfft, rms)
        assert abs(ev[i, 0] - ref["energy"]) <= 1e-6 * abs(ref["energy"]), (s.name, ev[i, 0], ref["energy"])
        assert abs(ev[i, 1] - ref["energy_self"]) <= 1e-12 * abs(ref["energy_self"]), s.name
        vir = ev[i, 2:].reshape(3, 3)
        assert np.abs(vir - ref["virial"]).max() <= 1e-5 * np.abs(ref["virial"]).max(), s.name

