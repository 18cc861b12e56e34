"""Builds the committed golden fixtures from the reference's own test data.

Run once, in a checkout that has the reference tree (read-only) beside it:

    python tests/golden/make_golden.py /path/to/gpu_recip

It writes, next to this script:

* ``ref_recip_23558.npz`` -- the reference recip test system (test_data/xyzq.txt: 23,558 atoms,
  cubic 62.23 A box, kappa 0.32, 64^3 grid) with its expected forces for spline order 4
  (test_data/force_recip_4.txt) and 6 (test_data/force_recip_6.txt), and the expected energy and
  virial that the reference test driver hard-codes (gpu_recip.cu:71-84 for order 4,
  gpu_recip.cu:300-314 for order 6) together with that driver's tolerances
  (gpu_recip.cu:146-174, :286-291 and :373-384, :515).
* ``fft_kat.npz`` -- the forward-FFT known-answer vectors of the reference
  (test_data/dataFFT{in,out}{64,64x2,64x64,4x4}.txt, used by test_fbfft.cu:188-256): real
  inputs (rows, x fastest) and their full complex DFTs (sign -1, unnormalised).

* ``ref_direct_23558.npz`` -- the reference direct-space test (gpu_direct.cu:55-207): the same
  23,558 atoms with their vdW types (test_data/vdwtype.txt) and parameters
  (test_data/vdwparam.txt, vdwparam14.txt: (c6, c12) pairs of 35 types), the CHARMM exclusion
  lists (iblo14.txt, inb14.txt, in the original atom order), the map from the coordinates'
  order to that order (loc2glo.txt, stored 0-based; xyzq.txt is the reference's neighbour-list
  order), the 1-4 inclusion and exclusion lists (in14list.txt,
  ex14list.txt), the settings of gpu_direct.cu:58-66 (box 62.23 A, kappa 0.32, roff 9, ron 7.5,
  e14fac 1.5, VDW_VSH + EWALD), the expected main-list and total forces (force_direct_main.txt,
  force_direct.txt), energies, virial and the driver's tolerances (gpu_direct.cu:67-76, 158,
  171, 203-207, 222).

Nothing at run time reads the reference tree: the tests load these .npz files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Expected values hard-coded in the reference test driver (gpu_recip.cu:71-84, :300-314).
REF_CONSTANTS = {
    4: dict(
        energy=0.5939730270e03,
        virial=[-0.5282341105e03, 0.5596133994e01, -0.6254453157e01,
                0.5596133994e01, -0.5054581254e03, -0.7652312605e-01,
                -0.6254453157e01, -0.7652312605e-01, -0.5575246246e03],
        tol_energy=2.0e-3, tol_virial=4.0e-3, tol_force=1.0e-3),
    6: dict(
        energy=0.5951144996e03,
        virial=[-0.5314776507e03, 0.5670623182e01, -0.6175456643e01,
                0.5670623182e01, -0.5086150173e03, -0.1026251692e00,
                -0.6175456643e01, -0.1026251692e00, -0.5606459148e03],
        tol_energy=1.3e-3, tol_virial=2.0e-3, tol_force=3.6e-4),
}


def main(ref_root: str) -> None:
    td = os.path.join(ref_root, "test_data")
    xyzq = np.loadtxt(os.path.join(td, "xyzq.txt"), dtype=np.float32)
    f4 = np.loadtxt(os.path.join(td, "force_recip_4.txt"), dtype=np.float64)
    f6 = np.loadtxt(os.path.join(td, "force_recip_6.txt"), dtype=np.float64)
    assert xyzq.shape == (23558, 4) and f4.shape == (23558, 3) and f6.shape == (23558, 3)
    out = dict(xyzq=xyzq, box=np.array([62.23, 62.23, 62.23]), kappa=np.array(0.320),
               nfft=np.array([64, 64, 64]), force4=f4, force6=f6)
    for p, c in REF_CONSTANTS.items():
        out[f"energy{p}"] = np.array(c["energy"])
        out[f"virial{p}"] = np.array(c["virial"]).reshape(3, 3)
        out[f"tol_energy{p}"] = np.array(c["tol_energy"])
        out[f"tol_virial{p}"] = np.array(c["tol_virial"])
        out[f"tol_force{p}"] = np.array(c["tol_force"])
    np.savez_compressed(os.path.join(HERE, "ref_recip_23558.npz"), **out)

    kat = {}
    for tag, shape in (("64", (1, 64)), ("64x2", (2, 64)), ("64x64", (64, 64)), ("4x4", (4, 4))):
        xin = np.loadtxt(os.path.join(td, f"dataFFTin{tag}.txt"), dtype=np.float64).reshape(shape)
        raw = np.loadtxt(os.path.join(td, f"dataFFTout{tag}.txt"), dtype=np.float64).reshape(-1)
        xout = (raw[0::2] + 1j * raw[1::2]).reshape(shape)
        kat[f"in{tag}"] = xin
        kat[f"out{tag}"] = xout
    np.savez_compressed(os.path.join(HERE, "fft_kat.npz"), **kat)

    def ints(name, cols=1):
        a = np.loadtxt(os.path.join(td, name), dtype=np.int64)
        return a.reshape(-1, cols).astype(np.int32) if cols > 1 else a.astype(np.int32)

    direct = dict(
        xyzq=xyzq, box=np.array([62.23, 62.23, 62.23]), kappa=np.array(0.320), roff=np.array(9.0),
        ron=np.array(7.5), e14fac=np.array(1.5),
        vdwparam=np.loadtxt(os.path.join(td, "vdwparam.txt"), dtype=np.float64),
        vdwparam14=np.loadtxt(os.path.join(td, "vdwparam14.txt"), dtype=np.float64),
        vdwtype=ints("vdwtype.txt"), iblo14=ints("iblo14.txt"), inb14=ints("inb14.txt"),
        loc2glo=ints("loc2glo.txt") - 1,
        in14=ints("in14list.txt", 3), ex14=ints("ex14list.txt", 3),
        force_main=np.loadtxt(os.path.join(td, "force_direct_main.txt"), dtype=np.float64),
        force_total=np.loadtxt(os.path.join(td, "force_direct.txt"), dtype=np.float64),
        energy_vdw=np.array(8198.14425), energy_elec=np.array(-73396.45998),
        virial=np.array([58748.2766568620, 159.656334638237, 483.080609561938,
                         159.656334638202, 57272.9410562695, 894.635309171291,
                         483.080609561938, 894.635309171288, 56639.3675265570]).reshape(3, 3),
        tol_force_main=np.array(7.72e-4), tol_force_total=np.array(7.73e-4),
        tol_energy=np.array(0.007), tol_virial=np.array(3.13))
    assert direct["vdwparam"].shape == (1260,) and direct["in14"].shape == (6556, 3)
    assert direct["force_main"].shape == (23558, 3) and direct["inb14"].shape == (34709,)
    np.savez_compressed(os.path.join(HERE, "ref_direct_23558.npz"), **direct)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference source tree>")
    main(sys.argv[1])
