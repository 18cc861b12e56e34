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


def _build(tmp):
    from gpu_recip_b200 import build
    lib = build.build()
    exe = os.path.join(tmp, "recip_driver")
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "recip_driver.cpp"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           "-L", os.path.dirname(lib), "-lpme_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.dirname(lib), "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_driver_compiles_against_the_header():
    with tempfile.TemporaryDirectory() as tmp:
        obj = os.path.join(tmp, "d.o")
        subprocess.run(["g++", "-std=c++17", "-c", os.path.join(ROOT, "tests", "cpp", "recip_driver.cpp"),
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
