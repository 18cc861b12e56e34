"""Direct-space PME on the GPU (include/pme_direct.h) against the reference's direct test and
the FP64 oracle.  Bars: the reference driver's own tolerances on its 23,558-atom fixture
(gpu_direct.cu:158-222: forces 7.72e-4 / 7.73e-4, energies 0.007, virial 3.13); against the
oracle a force relative RMS of 1e-5 and energies within 1e-6 relative; identical int64 forces
and energies from run to run."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FORCE_SCALE = 2.0 ** 40


@pytest.fixture(scope="module")
def fx():
    from tests.conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "ref_direct_23558.npz")))


def _make(torch, d, with14=False):
    from gpu_recip_b200.direct import CudaPMEDirectForce
    n = d["xyzq"].shape[0]
    dr = CudaPMEDirectForce()
    dr.setup(*d["box"], float(d["kappa"]), float(d["roff"]), float(d.get("ron", 0.0)), float(d.get("e14fac", 1.0)))
    dr.set_vdwparam(d["vdwparam"])
    dr.set_vdwtype(d["vdwtype"])
    if "iblo14" in d:
        dr.set_exclusions(d["iblo14"], d["inb14"], d.get("loc2glo"))
    if with14:
        dr.set_vdwparam14(d["vdwparam14"])
        dr.set_14_list(d["in14"], d["ex14"])
    x = torch.from_numpy(np.ascontiguousarray(d["xyzq"], dtype=np.float32)).cuda()
    stride = ((n + 63) // 64) * 64
    return dr, x, n, stride


def _run(torch, dr, x, n, stride, with14=False):
    f = torch.zeros(3 * stride, dtype=torch.int64, device="cuda")
    dr.energy_virial.clear()
    dr.calc_force(x, n, True, True, stride, f)
    if with14:
        dr.calc_14_force(x, True, True, stride, f)
    torch.cuda.synchronize()
    ev = dr.energy_virial
    ev.copyToHost()
    fi = f.view(3, stride)[:, :n].T.cpu().numpy()
    return fi, dict(vdw=ev.getEnergy("vdw"), elec=ev.getEnergy("elec"), excl=ev.getEnergy("excl")), ev.getVirial()


def test_direct_reference_fixture_main_list(cuda, fx):
    dr, x, n, stride = _make(cuda, fx)
    fi, e, vir = _run(cuda, dr, x, n, stride)
    f = fi.astype(np.float64) / FORCE_SCALE
    assert np.abs(f - fx["force_main"]).max() <= fx["tol_force_main"]
    assert abs(e["vdw"] - fx["energy_vdw"]) < fx["tol_energy"]
    assert abs(e["elec"] - fx["energy_elec"]) < fx["tol_energy"]
    assert np.abs(vir - fx["virial"]).max() < fx["tol_virial"]
    # run to run: the same int64 forces and energies
    fi2, e2, vir2 = _run(cuda, dr, x, n, stride)
    assert np.array_equal(fi, fi2) and e == e2 and np.array_equal(vir, vir2)
    dr.close()


def test_direct_reference_fixture_total_with_14_lists(cuda, fx, oracle):
    dr, x, n, stride = _make(cuda, fx, with14=True)
    fi, e, _ = _run(cuda, dr, x, n, stride, with14=True)
    f = fi.astype(np.float64) / FORCE_SCALE
    assert np.abs(f - fx["force_total"]).max() <= fx["tol_force_total"]
    _, ev14, ee14, ex14, _ = oracle.direct_14(fx["xyzq"].astype(np.float64), fx["box"], float(fx["kappa"]),
                                              float(fx["roff"]), float(fx["e14fac"]), fx["vdwparam14"],
                                              fx["vdwtype"], fx["in14"], fx["ex14"])
    assert abs(e["excl"] - ex14) < 1e-6 * abs(ex14)
    assert abs(e["vdw"] - (fx["energy_vdw"] + ev14)) < fx["tol_energy"]
    assert abs(e["elec"] - (fx["energy_elec"] + ee14)) < fx["tol_energy"]
    dr.close()


def test_direct_matches_fp64_oracle_on_fixture(cuda, fx, oracle):
    dr, x, n, stride = _make(cuda, fx)
    fi, e, vir = _run(cuda, dr, x, n, stride)
    ptr, idx = oracle.exclusions_csr(fx["iblo14"], fx["inb14"], n, fx["loc2glo"])
    vp32 = fx["vdwparam"].astype(np.float32).astype(np.float64)   # the library holds FP32 parameters
    fo, ev, ee, vo = oracle.direct_force(fx["xyzq"].astype(np.float32).astype(np.float64), fx["box"],
                                         float(fx["kappa"]), float(fx["roff"]), vp32, fx["vdwtype"], ptr, idx)
    f = fi.astype(np.float64) / FORCE_SCALE
    rms = np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum())
    assert rms <= 1e-5, rms
    assert abs(e["vdw"] - ev) <= 1e-6 * abs(ev)
    assert abs(e["elec"] - ee) <= 1e-6 * abs(ee)
    assert np.abs(vir - vo).max() <= 1e-5 * np.abs(vo).max()
    dr.close()


def _lattice(box=24.0, per=6, seed=3):
    """Charges on a jittered lattice with exclusions to the +x lattice neighbour (wrapping pairs sit
    180 indices apart: the explicit far-list path), two vdW types."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(per)] * 3, indexing="ij"), -1).reshape(-1, 3)
    n = per ** 3
    sp = box / per
    x = np.empty((n, 4))
    x[:, :3] = g * sp + rng.uniform(-0.3, 0.3, (n, 3))
    x[:, 3] = rng.choice([-0.8, 0.4], n)
    iblo, inb = [], []
    for i in range(n):
        gx, gy, gz = g[i]
        j = int(((gx + 1) % per) * per * per + gy * per + gz)
        inb.append(j + 1)
        iblo.append(len(inb))
    return dict(xyzq=x.astype(np.float32), box=np.array([box, box, box]), kappa=np.array(0.35),
                roff=np.array(9.0), vdwparam=np.array([1.0e2, 1.2e5, 6.0e1, 1.6e5, 2.9e2, 5.0e5]),
                vdwtype=(np.arange(n) % 2).astype(np.int32), iblo14=np.array(iblo, np.int32),
                inb14=np.array(inb, np.int32))


@pytest.mark.parametrize("box", [24.0, 40.0])   # 24 A: fewer cells than offsets on every axis
def test_direct_lattice_with_far_exclusions_matches_oracle(cuda, oracle, box):
    d = _lattice(box=box, per=6 if box == 24.0 else 10)
    dr, x, n, stride = _make(cuda, d)
    fi, e, vir = _run(cuda, dr, x, n, stride)
    ptr, idx = oracle.exclusions_csr(d["iblo14"], d["inb14"], n)
    vp32 = d["vdwparam"].astype(np.float32).astype(np.float64)
    fo, ev, ee, vo = oracle.direct_force(d["xyzq"].astype(np.float64), d["box"], float(d["kappa"]),
                                         float(d["roff"]), vp32, d["vdwtype"], ptr, idx)
    f = fi.astype(np.float64) / FORCE_SCALE
    assert np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum()) <= 1e-5
    assert abs(e["vdw"] - ev) <= 1e-6 * abs(ev) + 1e-6 and abs(e["elec"] - ee) <= 1e-6 * abs(ee)
    assert np.abs(vir - vo).max() <= 1e-5 * np.abs(vo).max()
    dr.close()


def test_direct_electrostatics_only_and_no_exclusions(cuda, oracle):
    from gpu_recip_b200.direct import CudaPMEDirectForce, ELEC_NONE, EWALD, VDW_NONE
    d = _lattice()
    n = d["xyzq"].shape[0]
    dr = CudaPMEDirectForce()
    dr.setup(24.0, 24.0, 24.0, 0.35, 9.0, 7.5, 1.0, VDW_NONE, EWALD)
    x = cuda.from_numpy(d["xyzq"]).cuda()
    fi, e, _ = _run(cuda, dr, x, n, n)
    ptr = np.zeros(n + 1, np.int32)
    fo, ev, ee, _ = oracle.direct_force(d["xyzq"].astype(np.float64), d["box"], 0.35, 9.0, np.zeros(2),
                                        np.zeros(n, np.int32), ptr, np.zeros(0, np.int32))
    f = fi.astype(np.float64) / FORCE_SCALE
    assert np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum()) <= 1e-5
    assert e["vdw"] == 0.0 and abs(e["elec"] - ee) <= 1e-6 * abs(ee)
    dr.close()


def test_direct_argument_checks(cuda):
    from gpu_recip_b200 import _capi
    from gpu_recip_b200.direct import CudaPMEDirectForce
    dr = CudaPMEDirectForce()
    x = cuda.zeros((4, 4), device="cuda")
    f = cuda.zeros(12, dtype=cuda.int64, device="cuda")
    with pytest.raises(_capi.PMEError) as e:       # before setup
        dr.calc_force(x, 4, True, True, 4, f)
    assert e.value.status == _capi.PME_ESTATE
    with pytest.raises(_capi.PMEError) as e:       # roff beyond half the box
        dr.setup(10.0, 10.0, 10.0, 0.3, 9.0, 7.5, 1.0)
    assert e.value.status == _capi.PME_EINVAL
    with pytest.raises(_capi.PMEError) as e:       # a model that is not built
        dr.setup(30.0, 30.0, 30.0, 0.3, 9.0, 7.5, 1.0, 2, 101)
    assert e.value.status == _capi.PME_EUNSUPPORTED
    dr.setup(30.0, 30.0, 30.0, 0.3, 9.0, 7.5, 1.0)
    dr.set_vdwparam([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])          # 2 types
    dr.set_vdwtype([0, 1, 2, 0])                             # type 2 is beyond the table
    with pytest.raises(_capi.PMEError) as e:
        dr.calc_force(x, 4, True, True, 4, f)
    assert e.value.status == _capi.PME_EINVAL
    dr.set_vdwtype([0, 1, 1, 0])
    dr.set_vdwparam14([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    dr.set_14_list([[0, 9, 13]], [])                         # atom 9 of 4
    with pytest.raises(_capi.PMEError) as e:
        dr.calc_14_force(x, True, True, 4, f)
    assert e.value.status == _capi.PME_EINVAL
    with pytest.raises(_capi.PMEError) as e:                 # loc2glo not a permutation
        dr.set_exclusions([1, 1, 1, 1], [2], [0, 0, 1, 2])
    assert e.value.status == _capi.PME_EINVAL
    dr.close()


@pytest.mark.parametrize("box,n", [(20.0, 3000), (40.0, 24000)])   # every axis with too few cells; shifts
def test_direct_dense_cells_many_chunks(cuda, oracle, box, n):
    """About 90 atoms per cell (three 32-atom chunks each): electrostatics only (random charges
    closer than any vdW model would allow), against the FP64 oracle."""
    from gpu_recip_b200.direct import CudaPMEDirectForce, EWALD, VDW_NONE
    rng = np.random.default_rng(n)
    x = np.empty((n, 4), np.float32)
    x[:, :3] = rng.random((n, 3)) * box
    x[:, 3] = rng.normal(0.0, 0.3, n)
    dr = CudaPMEDirectForce()
    dr.setup(box, box, box, 0.35, 9.0, 7.5, 1.0, VDW_NONE, EWALD)
    xd = cuda.from_numpy(x).cuda()
    fi, e, vir = _run(cuda, dr, xd, n, n)
    fo, _, ee, vo = oracle.direct_force(x.astype(np.float64), np.array([box] * 3), 0.35, 9.0, np.zeros(2),
                                        np.zeros(n, np.int32), np.zeros(n + 1, np.int32), np.zeros(0, np.int32))
    f = fi.astype(np.float64) / FORCE_SCALE
    assert np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum()) <= 1e-6
    assert abs(e["elec"] - ee) <= 1e-7 * abs(ee) + 1e-6
    assert np.abs(vir - vo).max() <= 1e-6 * np.abs(vo).max()
    dr.close()


def test_direct_vdw_only(cuda, oracle):
    """ELEC_NONE: only the shifted Lennard-Jones terms (the oracle with the charges set to 0)."""
    from gpu_recip_b200.direct import CudaPMEDirectForce, ELEC_NONE, VDW_VSH
    d = _lattice()
    n = d["xyzq"].shape[0]
    dr = CudaPMEDirectForce()
    dr.setup(24.0, 24.0, 24.0, 0.35, 9.0, 7.5, 1.0, VDW_VSH, ELEC_NONE)
    dr.set_vdwparam(d["vdwparam"])
    dr.set_vdwtype(d["vdwtype"])
    dr.set_exclusions(d["iblo14"], d["inb14"])
    x = cuda.from_numpy(d["xyzq"]).cuda()
    fi, e, vir = _run(cuda, dr, x, n, n)
    xq0 = d["xyzq"].astype(np.float64).copy()
    xq0[:, 3] = 0.0
    ptr, idx = oracle.exclusions_csr(d["iblo14"], d["inb14"], n)
    fo, ev, ee, vo = oracle.direct_force(xq0, d["box"], 0.35, 9.0, d["vdwparam"].astype(np.float32).astype(np.float64),
                                         d["vdwtype"], ptr, idx)
    f = fi.astype(np.float64) / FORCE_SCALE
    assert e["elec"] == 0.0 and ee == 0.0
    assert np.sqrt(((f - fo) ** 2).sum() / (fo ** 2).sum()) <= 1e-6
    assert abs(e["vdw"] - ev) <= 1e-6 * abs(ev)
    dr.close()
