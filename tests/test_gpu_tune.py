"""The autotuner (pme_autotune / pme_batch_autotune): every launch shape it may pick computes the
same bits, so tuned evaluations must equal untuned ones exactly; the chosen shape is kept in the
handle and reused by new handles of the same grid."""
import numpy as np
import pytest

from gpu_recip_b200 import systems as S

pytestmark = pytest.mark.gpu


def _eval(torch, pme, s, x):
    from gpu_recip_b200 import force_stride
    n = s.natom
    st = force_stride(n)
    f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
    pme.energy_virial.clear()
    pme.eval_ortho([1.0 / b for b in s.box], x, n, s.kappa, True, True, f, st)
    torch.cuda.synchronize()
    pme.energy_virial.copyToHost()
    return f.cpu().numpy(), pme.energy_virial.getEnergy("recip"), pme.energy_virial.getVirial()


def test_autotune_keeps_results_and_caches_shape(cuda):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip
    from gpu_recip_b200.pme import tune_cache_clear
    tune_cache_clear()
    s = S.config_production(4)
    x = torch.from_numpy(s.xyzq).cuda()
    pme = CudaPMERecip(*s.nfft, s.order)
    f0, e0, v0 = _eval(torch, pme, s, x)
    pme.energy_virial.clear()
    cfg = pme.autotune([1.0 / b for b in s.box], x, s.natom, s.kappa, reps=3)
    assert cfg["candidates"] >= 2 and cfg["us_per_eval"] > 0
    # the energy/virial record is left as it was (cleared above)
    pme.energy_virial.copyToHost()
    assert pme.energy_virial.getEnergy("recip") == 0.0
    f1, e1, v1 = _eval(torch, pme, s, x)
    assert np.array_equal(f0, f1) and e0 == e1 and np.array_equal(v0, v1)
    got = pme.get_tune_config()
    for k in ("schedule", "x_lines", "y_lines", "z_columns", "grid_ctas"):
        assert got[k] == cfg[k]
    other = CudaPMERecip(*s.nfft, s.order)     # same grid: starts from the tuned shape
    assert {k: other.get_tune_config()[k] for k in got if k not in ("us_per_eval", "candidates")} == \
           {k: got[k] for k in got if k not in ("us_per_eval", "candidates")}
    tune_cache_clear()


@pytest.mark.parametrize("shape", [dict(schedule=2, x_lines=4, y_lines=32, z_columns=4, grid_ctas=148),
                                   dict(schedule=1, x_lines=32, y_lines=4, z_columns=32, grid_ctas=0),
                                   dict(schedule=2, x_lines=8, y_lines=8, z_columns=8, grid_ctas=37)])
def test_every_launch_shape_gives_the_same_bits(cuda, shape):
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip
    s = S.config_production(6)
    x = torch.from_numpy(s.xyzq).cuda()
    ref = _eval(torch, CudaPMERecip(*s.nfft, s.order), s, x)
    pme = CudaPMERecip(*s.nfft, s.order)
    pme.set_tune_config(**shape)
    got = _eval(torch, pme, s, x)
    assert np.array_equal(ref[0], got[0]) and ref[1] == got[1] and np.array_equal(ref[2], got[2])


def test_set_tune_config_rejects_oversized_tiles(cuda):
    from gpu_recip_b200 import CudaPMERecip, _capi
    pme = CudaPMERecip(512, 64, 64, 4)
    with pytest.raises(_capi.PMEError) as e:
        pme.set_tune_config(x_lines=64)
    assert e.value.status == _capi.PME_EINVAL


def test_batch_autotune_keeps_results(cuda):
    torch = cuda
    from gpu_recip_b200 import PmeBatch, force_stride
    systems = S.batch_systems(12, seed=9)
    specs, forces = [], []
    for sy in systems:
        st = force_stride(sy.natom)
        f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
        forces.append(f)
        specs.append(dict(nfft=sy.nfft, order=sy.order, box=sy.box, kappa=sy.kappa,
                          xyzq=torch.from_numpy(sy.xyzq).cuda(), force=f, stride=st))
    b = PmeBatch(specs)
    b.clear_energy_virial()
    b.eval()
    ev0 = b.energy_virial()
    f0 = [f.cpu().numpy().copy() for f in forces]
    cfg = b.autotune(reps=2)
    assert cfg["candidates"] == 12
    b.clear_energy_virial()
    b.eval()
    ev1 = b.energy_virial()
    assert np.array_equal(ev0, ev1)
    for a, f in zip(f0, forces):
        assert np.array_equal(a, f.cpu().numpy())


@pytest.mark.parametrize("system", ["water8k_64_p4", "water8k_64_p6", "water1k_32", "dodec_64_p4", "odd_p4"])
def test_inverse_x_in_the_gather_gives_the_same_bits(cuda, system):
    """The fused evaluation with the inverse x pass inside the gather tiles (each tile transforms
    the rows its atoms reach) equals the one with a separate x-inverse phase bit for bit: forces of
    every kind, energy, virial and the stored solved grid; repeated evaluations too."""
    torch = cuda
    from gpu_recip_b200 import CudaPMERecip, force_stride, _capi as C
    s = {"water8k_64_p4": lambda: S.config_production(4), "water8k_64_p6": lambda: S.config_production(6),
         "water1k_32": S.config_small, "dodec_64_p4": lambda: S.config_triclinic(4),
         "odd_p4": lambda: S.PmeSystem("odd", S.config_small().xyzq, S.config_small().box, (30, 36, 25), 4, 0.34)}[system]()
    n = s.natom
    st = force_stride(n)
    x = torch.from_numpy(s.xyzq).cuda()

    def run(mode):
        pme = CudaPMERecip(*s.nfft, s.order)
        pme.set_x_gather_fusion(mode)
        outs = []
        for rep in range(2):
            f = torch.zeros(3 * st, dtype=torch.float32, device="cuda")
            fi = torch.full((3 * st,), 5, dtype=torch.int64, device="cuda")
            pme.energy_virial.clear()
            pme.eval(s.recip9, x, n, s.kappa, True, True, f, st)
            pme.eval(s.recip9, x, n, s.kappa, False, False, fi, st)
            torch.cuda.synchronize()
            pme.energy_virial.copyToHost()
            outs.append((f.cpu().numpy(), fi.cpu().numpy(), pme.energy_virial.getEnergy("recip"),
                         pme.energy_virial.getEnergy("self"), pme.energy_virial.getVirial(),
                         pme.solved_grid()))   # the whole solved grid is stored either way
        return outs

    fused, separate = run(C.PME_XGATHER_AUTO), run(C.PME_XGATHER_OFF)
    for a, b in zip(fused, separate):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert a[2] == b[2] and a[3] == b[3] and np.array_equal(a[4], b[4])
        assert np.array_equal(a[5], b[5])
    assert np.abs(fused[0][0]).max() > 0


def test_x_gather_fusion_rejects_unknown_modes(cuda):
    from gpu_recip_b200 import CudaPMERecip, _capi as C
    pme = CudaPMERecip(32, 32, 32, 4)
    with pytest.raises(C.PMEError) as e:
        pme.set_x_gather_fusion(7)
    assert e.value.status == C.PME_EINVAL
