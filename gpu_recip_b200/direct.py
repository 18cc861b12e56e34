"""Direct-space (real-space) PME nonbonded terms: the Python mirror of CudaPMEDirectForce.

``CudaPMEDirectForce`` keeps the reference's method names and argument meaning
(CudaPMEDirectForce.h:137-205): setup, set_vdwparam(14), set_vdwtype, set_14_list, calc_force,
calc_14_force, and an energy/virial record with the names "vdw", "elec" and "excl".  The
topological exclusions that the reference hands to its neighbour-list build (CudaTopExcl) go to
``set_exclusions``; calc_force takes no neighbour list (the library bins the atoms itself).
Forces are gradients added to an int64 SoA array at 2^40 (Force<long long>).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from .pme import _ptr, _stream_handle, _xyzq_ptr

VDW_NONE, VDW_VSH = C.PME_VDW_NONE, C.PME_VDW_VSH
ELEC_NONE, EWALD = C.PME_ELEC_NONE, C.PME_ELEC_EWALD


def _host(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


class DirectEnergyVirial:
    """The record calc_force / calc_14_force accumulate into (CudaEnergyVirial's "vdw", "elec",
    "excl" energies and virial)."""

    def __init__(self, owner: "CudaPMEDirectForce"):
        self._owner = owner
        self._e = {"vdw": 0.0, "elec": 0.0, "excl": 0.0}
        self._v = np.zeros((3, 3))

    def clear(self):
        C.check(C.load().pme_direct_clear_energy_virial(self._owner._h), "direct clear")
        self._e = {k: 0.0 for k in self._e}
        self._v[:] = 0.0

    def copyToHost(self):
        e = [ctypes.c_double() for _ in range(3)]
        v = (ctypes.c_double * 9)()
        C.check(C.load().pme_direct_get_energy_virial(self._owner._h, *[ctypes.byref(x) for x in e], v),
                "direct energies")
        self._e = {"vdw": e[0].value, "elec": e[1].value, "excl": e[2].value}
        self._v = np.array(v[:]).reshape(3, 3)

    def getEnergy(self, name: str) -> float:
        return float(self._e[name])

    def getVirial(self) -> np.ndarray:
        return self._v.copy()


class CudaPMEDirectForce:
    def __init__(self, stream=None):
        self._lib = C.load()
        self._h = ctypes.c_void_p()
        C.check(self._lib.pme_direct_create(_stream_handle(stream), ctypes.byref(self._h)), "direct create")
        self.energy_virial = DirectEnergyVirial(self)

    def close(self):
        if self._h:
            self._lib.pme_direct_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        C.check(self._lib.pme_direct_set_stream(self._h, _stream_handle(stream)), "direct set_stream")

    def setup(self, boxx, boxy, boxz, kappa, roff, ron, e14fac, vdw_model=VDW_VSH, elec_model=EWALD):
        C.check(self._lib.pme_direct_setup(self._h, float(boxx), float(boxy), float(boxz), float(kappa),
                                           float(roff), float(ron), float(e14fac), int(vdw_model),
                                           int(elec_model)), "direct setup")

    def set_box_size(self, boxx, boxy, boxz):
        C.check(self._lib.pme_direct_set_box_size(self._h, float(boxx), float(boxy), float(boxz)), "box")

    def set_vdwparam(self, vdwparam):
        a = _host(vdwparam, np.float32)
        C.check(self._lib.pme_direct_set_vdwparam(self._h, a.size, a.ctypes.data_as(ctypes.c_void_p)), "vdwparam")

    def set_vdwparam14(self, vdwparam14):
        a = _host(vdwparam14, np.float32)
        C.check(self._lib.pme_direct_set_vdwparam14(self._h, a.size, a.ctypes.data_as(ctypes.c_void_p)),
                "vdwparam14")

    def set_vdwtype(self, vdwtype):
        a = _host(vdwtype, np.int32)
        C.check(self._lib.pme_direct_set_vdwtype(self._h, a.size, a.ctypes.data_as(ctypes.c_void_p)), "vdwtype")

    def set_exclusions(self, iblo14, inb14, loc2glo=None):
        """CHARMM exclusion lists (CudaTopExcl(ncoord, iblo14, inb14)) in the original atom order;
        loc2glo (0-based) maps each coordinate to that order."""
        ib = _host(iblo14, np.int32)
        nb = _host(inb14, np.int32)
        lg = None if loc2glo is None else _host(loc2glo, np.int32)
        C.check(self._lib.pme_direct_set_exclusions(
            self._h, ib.size, ib.ctypes.data_as(ctypes.c_void_p),
            nb.ctypes.data_as(ctypes.c_void_p) if nb.size else None,
            None if lg is None else lg.ctypes.data_as(ctypes.c_void_p)), "exclusions")

    def set_14_list(self, in14, ex14):
        """(i, j, ishift) triples of the 1-4 inclusion and exclusion lists (xx14list_t)."""
        a = _host(in14, np.int32).reshape(-1, 3)
        b = _host(ex14, np.int32).reshape(-1, 3)
        C.check(self._lib.pme_direct_set_14_list(self._h, a.shape[0], b.shape[0],
                                                 a.ctypes.data_as(ctypes.c_void_p) if a.size else None,
                                                 b.ctypes.data_as(ctypes.c_void_p) if b.size else None), "14 list")

    def calc_force(self, xyzq, ncoord: int, calc_energy: bool, calc_virial: bool, stride: int, force):
        """Main-list forces added to ``force`` (device int64 tensor of 3 * stride)."""
        C.check(self._lib.pme_direct_calc_force(self._h, _xyzq_ptr(xyzq, ncoord), int(ncoord), int(calc_energy),
                                                int(calc_virial), int(stride), _ptr(force)), "calc_force")

    def calc_14_force(self, xyzq, calc_energy: bool, calc_virial: bool, stride: int, force):
        C.check(self._lib.pme_direct_calc_14_force(self._h, _ptr(xyzq), int(calc_energy), int(calc_virial),
                                                   int(stride), _ptr(force)), "calc_14_force")
