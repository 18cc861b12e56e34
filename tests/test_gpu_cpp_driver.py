"""A C++ program that uses only include/pme_recip.h (and the CUDA runtime for its buffers) runs the
reference driver's call sequence on the reference's own 23,558-atom fixture: the staged calls and
the fused call agree bit for bit and pass the reference driver's tolerances (gpu_recip.cu)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _build(tmp, name="recip_driver"):
    from gpu_recip_b200 import build
    lib = build.build()
    exe = os.path.join(tmp, name)
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           "-L", os.path.dirname(lib), "-lpme_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.dirname(lib), "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


@pytest.mark.parametrize("name", ["recip_driver", "direct_driver", "looper_driver"])
def test_cpp_driver_compiles_against_the_header(name):
    with tempfile.TemporaryDirectory() as tmp:
        obj = os.path.join(tmp, "d.o")
        subprocess.run(["g++", "-std=c++17", "-c", os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), "-o", obj],
                       check=True)
        assert os.path.getsize(obj) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 6])
def test_cpp_driver_on_reference_fixture(cuda, ref_fixture, order):
    f = ref_fixture
    n = f["xyzq"].shape[0]
    with tempfile.TemporaryDirectory() as tmp:
        exe = _build(tmp)
        inp, out = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(inp, "wb") as fh:
            fh.write(np.array([n, order, *[int(v) for v in f["nfft"]]], np.int32).tobytes())
            fh.write(np.asarray(f["box"], np.float64).tobytes())
            fh.write(np.array([float(f["kappa"])], np.float64).tobytes())
            fh.write(np.ascontiguousarray(f["xyzq"], np.float32).tobytes())
        subprocess.run([exe, inp, out], check=True, timeout=120)
        raw = open(out, "rb").read()
    per = 8 * 10 + 4 * 3 * n
    res = []
    for seq in range(2):
        chunk = raw[seq * per:(seq + 1) * per]
        e = np.frombuffer(chunk[:8], np.float64)[0]
        vir = np.frombuffer(chunk[8:80], np.float64).reshape(3, 3)
        force = np.frombuffer(chunk[80:], np.float32).reshape(n, 3)
        res.append((e, vir, force))
    (e0, v0, f0), (e1, v1, f1) = res
    assert e0 == e1 and np.array_equal(v0, v1) and np.array_equal(f0, f1)
    assert abs(e0 - f[f"energy{order}"]) < f[f"tol_energy{order}"]
    assert np.abs(v0 - f[f"virial{order}"]).max() < f[f"tol_virial{order}"]
    assert np.abs(f0 - f[f"force{order}"]).max() < f[f"tol_force{order}"]


@pytest.mark.gpu
def test_cpp_direct_driver_on_reference_fixture(cuda):
    """The reference's direct test sequence from C++ (gpu_direct.cu:151-233) on its own fixture:
    main-list forces, energies and virial, then the total with the 1-4 lists, within the driver's
    tolerances."""
    from tests.conftest import GOLDEN
    d = dict(np.load(os.path.join(GOLDEN, "ref_direct_23558.npz")))
    n = d["xyzq"].shape[0]
    with tempfile.TemporaryDirectory() as tmp:
        exe = _build(tmp, "direct_driver")
        inp, out = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(inp, "wb") as fh:
            fh.write(np.array([n, d["vdwparam"].size, d["vdwparam14"].size, d["in14"].shape[0],
                               d["ex14"].shape[0], d["inb14"].size], np.int32).tobytes())
            fh.write(np.array([*d["box"], float(d["kappa"]), float(d["roff"]), float(d["ron"]),
                               float(d["e14fac"])], np.float64).tobytes())
            fh.write(np.ascontiguousarray(d["xyzq"], np.float32).tobytes())
            fh.write(d["vdwparam"].astype(np.float32).tobytes())
            fh.write(d["vdwparam14"].astype(np.float32).tobytes())
            for key in ("vdwtype", "iblo14", "inb14", "loc2glo", "in14", "ex14"):
                fh.write(np.ascontiguousarray(d[key], np.int32).tobytes())
        subprocess.run([exe, inp, out], check=True, timeout=120)
        raw = np.fromfile(out, dtype=np.float64)
    per = 12 + 3 * n
    main, total = raw[:per], raw[per:2 * per]
    assert np.abs(main[12:].reshape(n, 3) - d["force_main"]).max() <= d["tol_force_main"]
    assert abs(main[0] - d["energy_vdw"]) < d["tol_energy"] and abs(main[1] - d["energy_elec"]) < d["tol_energy"]
    assert np.abs(main[3:12].reshape(3, 3) - d["virial"]).max() < d["tol_virial"]
    assert np.abs(total[12:].reshape(n, 3) - d["force_total"]).max() <= d["tol_force_total"]


@pytest.mark.gpu
def test_cpp_recip_node_loop(cuda):
    """A C++ recip node on pme_recip_loop_run (CudaDomdecRecipLooper::run): three steps with
    changing box, coordinate count and flags, then STOP; every step's forces and record equal the
    MD adapter's evaluation of the same step bit for bit."""
    torch = cuda
    from gpu_recip_b200 import CudaDomdecRecip
    from gpu_recip_b200 import systems as S
    s = S.config_small(seed=12)
    n = s.natom
    with tempfile.TemporaryDirectory() as tmp:
        exe = _build(tmp, "looper_driver")
        inp, out = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(inp, "wb") as fh:
            fh.write(np.array([n, s.order, *s.nfft], np.int32).tobytes())
            fh.write(np.asarray(s.box, np.float64).tobytes())
            fh.write(np.array([s.kappa], np.float64).tobytes())
            fh.write(np.ascontiguousarray(s.xyzq, np.float32).tobytes())
        subprocess.run([exe, inp, out], check=True, timeout=120)
        raw = open(out, "rb").read()
    steps = int(np.frombuffer(raw[:8], np.int64)[0])
    assert steps == 3
    pos = 8
    ref = CudaDomdecRecip(*s.nfft, s.order, s.kappa)
    for k, (scale, drop, e, v) in enumerate([(1.0, 0, True, True), (1.01, 7, False, True), (0.995, 14, True, False)]):
        cnt = int(np.frombuffer(raw[pos:pos + 4], np.int32)[0])
        pos += 4
        rec = np.frombuffer(raw[pos:pos + 88], np.float64)
        pos += 88
        force = np.frombuffer(raw[pos:pos + 12 * cnt], np.float32).reshape(cnt, 3)
        pos += 12 * cnt
        assert cnt == n - drop
        x = torch.from_numpy(np.ascontiguousarray(s.xyzq[:cnt])).cuda()
        want = torch.zeros((cnt, 3), dtype=torch.float32, device="cuda")
        ev = ref.pme.energy_virial
        ev.clear()
        ref.calc(*[1.0 / (b * scale) for b in s.box], x, cnt, e, v, want)
        torch.cuda.synchronize()
        ev.copyToHost()
        assert np.array_equal(force, want.cpu().numpy()), k
        assert rec[0] == ev.getEnergy("recip") and np.array_equal(rec[2:].reshape(3, 3), ev.getVirial()), k

