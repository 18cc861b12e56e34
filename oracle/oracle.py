"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may import this
module: it is the checker of the CUDA path, never part of it.  The C++ restatement it loads
(``pme_oracle.cpp``, built by the ``Makefile`` beside it) follows the reference operator
CudaPMERecip (ap-hynninen/gpu_recip, CudaPMERecip.cu); each C function cites the reference
lines it restates.

Array conventions (numpy):
  xyzq      (N, 4)  x, y, z [A], q [e]
  recip3    (3,)    diagonal of the reciprocal box (1/Lx, 1/Ly, 1/Lz)
  real grid (nz, ny, nx)            x fastest, as the reference's unpadded grid
  half grid (nz, ny, nx//2+1) complex128
  forces    (N, 3)  +dE/dx (the reference's gradient convention)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

CCELEC = 332.0716


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++; no GPU needed)."""
    src = os.path.join(_HERE, "pme_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        L.orc_bspline.argtypes = [I, D, P, P]
        L.orc_spread_f64.argtypes = [P, I, P, I, I, I, I, P, I]
        L.orc_spread_fixed.argtypes = [P, I, P, I, I, I, I, P, I]
        L.orc_fixed_to_float.argtypes = [P, ctypes.c_size_t, P]
        L.orc_fft1d.argtypes = [P, I, I]
        L.orc_dft1d.argtypes = [P, P, I, I]
        L.orc_fft3d_r2c.argtypes = [P, I, I, I, P, I]
        L.orc_fft3d_c2r.argtypes = [P, I, I, I, P, I]
        L.orc_bspline_moduli.argtypes = [I, I, P]
        L.orc_scalar_sum.argtypes = [P, I, I, I, I, P, D, I, P, P, I]
        L.orc_gather.argtypes = [P, I, P, P, I, I, I, I, P, I]
        L.orc_self_energy.argtypes = [P, I, D]
        L.orc_self_energy.restype = D
        L.orc_eval.argtypes = [P, I, P, I, I, I, I, D, P, P, P, P, I]
        L.orc_hardware_threads.argtypes = []
        L.orc_spread_f64_tric.argtypes = [P, I, P, I, I, I, I, P, I]
        L.orc_spread_fixed_tric.argtypes = [P, I, P, I, I, I, I, P, I]
        L.orc_scalar_sum_tric.argtypes = [P, I, I, I, I, P, D, I, P, P, I]
        L.orc_gather_tric.argtypes = [P, I, P, P, I, I, I, I, P, I]
        L.orc_eval_tric.argtypes = [P, I, P, I, I, I, I, D, P, P, P, P, I]
        L.orc_direct_force.argtypes = [P, I, P, D, D, P, P, P, P, P, P, P, P, I]
        L.orc_direct_14.argtypes = [P, P, D, D, D, P, P, P, I, P, I, P, P, P, P, P]
        for name in ("orc_direct_force", "orc_direct_14"):
            getattr(L, name).restype = I
        for name in ("orc_bspline", "orc_spread_f64", "orc_spread_fixed", "orc_fixed_to_float",
                     "orc_fft1d", "orc_dft1d", "orc_fft3d_r2c", "orc_fft3d_c2r",
                     "orc_bspline_moduli", "orc_scalar_sum", "orc_gather", "orc_eval",
                     "orc_hardware_threads", "orc_spread_f64_tric", "orc_spread_fixed_tric",
                     "orc_scalar_sum_tric", "orc_gather_tric", "orc_eval_tric"):
            if name not in ("orc_fixed_to_float",):
                getattr(L, name).restype = I
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int, what: str):
    if rc != 0:
        raise ValueError(f"oracle {what} rejected its arguments (rc={rc})")


def hardware_threads() -> int:
    return int(lib().orc_hardware_threads())


def bspline(order: int, u: float):
    th = np.zeros(order)
    dth = np.zeros(order)
    _check(lib().orc_bspline(order, float(u), _p(th), _p(dth)), "bspline")
    return th, dth


def bspline_moduli(order: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    _check(lib().orc_bspline_moduli(order, n, _p(out)), "moduli")
    return out


def _box(recip):
    """(suffix, array): recip given as the reciprocal diagonal (3 values) or the row-major 3x3
    reciprocal matrix (9 values); a diagonal matrix takes the orthorhombic functions, anything
    else the triclinic (*_tric) ones."""
    r = np.ascontiguousarray(recip, dtype=np.float64).reshape(-1)
    if r.size == 3:
        return "", r
    if r.size != 9:
        raise ValueError("recip must hold 3 (diagonal) or 9 (matrix) values")
    if np.all(r[[1, 2, 3, 5, 6, 7]] == 0.0):
        return "", np.ascontiguousarray(r[[0, 4, 8]])
    return "_tric", r


def spread_f64(xyzq, recip3, nfft, order, nthreads=0) -> np.ndarray:
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    sfx, r = _box(recip3)
    nx, ny, nz = nfft
    g = np.zeros((nz, ny, nx))
    _check(getattr(lib(), "orc_spread_f64" + sfx)(_p(x), x.shape[0], _p(r), nx, ny, nz, order, _p(g),
                                                   nthreads), "spread_f64")
    return g


def spread_fixed(xyzq, recip3, nfft, order, nthreads=0) -> np.ndarray:
    """int64 fixed-point grid (scale 2^40) from the FP32 mirror of the GPU spreading."""
    x = np.ascontiguousarray(xyzq, dtype=np.float32).reshape(-1, 4)
    sfx, r = _box(recip3)
    nx, ny, nz = nfft
    g = np.zeros((nz, ny, nx), dtype=np.int64)
    _check(getattr(lib(), "orc_spread_fixed" + sfx)(_p(x), x.shape[0], _p(r), nx, ny, nz, order, _p(g),
                                                     nthreads), "spread_fixed")
    return g


def fixed_to_float(g: np.ndarray) -> np.ndarray:
    g = np.ascontiguousarray(g, dtype=np.int64)
    out = np.empty(g.shape, dtype=np.float32)
    lib().orc_fixed_to_float(_p(g), g.size, _p(out))
    return out


def fft1d(x, sign=-1) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    _check(lib().orc_fft1d(_p(a), a.size, sign), "fft1d")
    return a


def dft1d(x, sign=-1) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(a)
    _check(lib().orc_dft1d(_p(a), _p(out), a.size, sign), "dft1d")
    return out


def fft3d_r2c(grid: np.ndarray, nthreads=0) -> np.ndarray:
    g = np.ascontiguousarray(grid, dtype=np.float64)
    nz, ny, nx = g.shape
    out = np.empty((nz, ny, nx // 2 + 1), dtype=np.complex128)
    _check(lib().orc_fft3d_r2c(_p(g), nx, ny, nz, _p(out), nthreads), "fft3d_r2c")
    return out


def fft3d_c2r(half: np.ndarray, nx: int, nthreads=0) -> np.ndarray:
    h = np.ascontiguousarray(half, dtype=np.complex128)
    nz, ny, hx = h.shape
    assert hx == nx // 2 + 1
    out = np.empty((nz, ny, nx))
    _check(lib().orc_fft3d_c2r(_p(h), nx, ny, nz, _p(out), nthreads), "fft3d_c2r")
    return out


def scalar_sum(half: np.ndarray, nx: int, order: int, recip3, kappa: float, calc_ev=True,
               nthreads=0):
    """Returns (solved half grid, energy, virial 3x3)."""
    h = np.ascontiguousarray(half, dtype=np.complex128).copy()
    nz, ny, hx = h.shape
    sfx, r = _box(recip3)
    e = np.zeros(1)
    v = np.zeros(9)
    _check(getattr(lib(), "orc_scalar_sum" + sfx)(_p(h), nx, ny, nz, order, _p(r), float(kappa),
                                                   int(calc_ev), _p(e), _p(v), nthreads), "scalar_sum")
    return h, float(e[0]), v.reshape(3, 3)


def gather(xyzq, grid: np.ndarray, recip3, order, nthreads=0) -> np.ndarray:
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    g = np.ascontiguousarray(grid, dtype=np.float64)
    nz, ny, nx = g.shape
    sfx, r = _box(recip3)
    f = np.zeros((x.shape[0], 3))
    _check(getattr(lib(), "orc_gather" + sfx)(_p(x), x.shape[0], _p(g), _p(r), nx, ny, nz, order, _p(f),
                                               nthreads), "gather")
    return f


def self_energy(xyzq, kappa) -> float:
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    return float(lib().orc_self_energy(_p(x), x.shape[0], float(kappa)))


def evaluate(xyzq, recip3, nfft, order, kappa, nthreads=0):
    """Full FP64 evaluation.  Returns dict(force (N,3), energy, energy_self, virial (3,3))."""
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    sfx, r = _box(recip3)
    nx, ny, nz = nfft
    f = np.zeros((x.shape[0], 3))
    e = np.zeros(1)
    es = np.zeros(1)
    v = np.zeros(9)
    _check(getattr(lib(), "orc_eval" + sfx)(_p(x), x.shape[0], _p(r), nx, ny, nz, order, float(kappa),
                                             _p(f), _p(e), _p(es), _p(v), nthreads), "eval")
    return {"force": f, "energy": float(e[0]), "energy_self": float(es[0]),
            "virial": v.reshape(3, 3)}


# ---------------------------------------------------------------------------------------------
# Direct-space nonbonded terms (VDW_VSH + EWALD, the reference's direct test models)
# ---------------------------------------------------------------------------------------------
def exclusions_csr(iblo14, inb14, natom, loc2glo=None):
    """Symmetric 0-based exclusion lists (CSR ptr, idx) from CHARMM's iblo14/inb14 (atom i's
    partners are |inb14[iblo14[i-1] .. iblo14[i]-1]| - 1, negative entries marking 1-4 pairs;
    CudaTopExcl.cu:22-80 reads them the same way).  The lists number atoms in their original
    order; loc2glo[i] (0-based) is the original index of coordinate i, and the result is in the
    coordinates' order."""
    iblo14 = np.asarray(iblo14, dtype=np.int64)
    inb14 = np.asarray(inb14, dtype=np.int64)
    start = np.r_[0, iblo14[:-1]]
    ii = np.repeat(np.arange(natom), iblo14 - start)
    jj = np.abs(inb14) - 1
    if loc2glo is not None:
        glo2loc = np.empty(natom, dtype=np.int64)
        glo2loc[np.asarray(loc2glo, dtype=np.int64)] = np.arange(natom)
        ii, jj = glo2loc[ii], glo2loc[jj]
    a = np.r_[ii, jj]
    b = np.r_[jj, ii]
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    keep = np.r_[True, (a[1:] != a[:-1]) | (b[1:] != b[:-1])]
    a, b = a[keep], b[keep]
    ptr = np.zeros(natom + 1, dtype=np.int32)
    np.add.at(ptr, a + 1, 1)
    return np.cumsum(ptr).astype(np.int32), b.astype(np.int32)


def direct_force(xyzq, box3, kappa, roff, vdwparam, vdwtype, excl_ptr, excl_idx, nthreads=0):
    """Main-list pair forces (gradient, (N, 3)), E_vdw, E_elec and the virial (3x3)."""
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    b = np.ascontiguousarray(box3, dtype=np.float64)
    vp = np.ascontiguousarray(vdwparam, dtype=np.float64)
    vt = np.ascontiguousarray(vdwtype, dtype=np.int32)
    ep = np.ascontiguousarray(excl_ptr, dtype=np.int32)
    ei = np.ascontiguousarray(excl_idx, dtype=np.int32)
    f = np.zeros((x.shape[0], 3))
    ev, ee, v = np.zeros(1), np.zeros(1), np.zeros(9)
    _check(lib().orc_direct_force(_p(x), x.shape[0], _p(b), float(kappa), float(roff), _p(vp), _p(vt),
                                  _p(ep), _p(ei), _p(f), _p(ev), _p(ee), _p(v), nthreads), "direct_force")
    return f, float(ev[0]), float(ee[0]), v.reshape(3, 3)


def direct_14(xyzq, box3, kappa, roff, e14fac, vdwparam14, vdwtype, in14, ex14):
    """1-4 inclusion and exclusion terms: forces (N, 3), E_vdw, E_elec, E_excl, virial."""
    x = np.ascontiguousarray(xyzq, dtype=np.float64).reshape(-1, 4)
    b = np.ascontiguousarray(box3, dtype=np.float64)
    vp = np.ascontiguousarray(vdwparam14, dtype=np.float64)
    vt = np.ascontiguousarray(vdwtype, dtype=np.int32)
    i14 = np.ascontiguousarray(in14, dtype=np.int32).reshape(-1, 3)
    e14 = np.ascontiguousarray(ex14, dtype=np.int32).reshape(-1, 3)
    f = np.zeros((x.shape[0], 3))
    ev, ee, ex, v = np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(9)
    _check(lib().orc_direct_14(_p(x), _p(b), float(kappa), float(roff), float(e14fac), _p(vp), _p(vt),
                               _p(i14), i14.shape[0], _p(e14), e14.shape[0], _p(f), _p(ev), _p(ee), _p(ex),
                               _p(v)), "direct_14")
    return f, float(ev[0]), float(ee[0]), float(ex[0]), v.reshape(3, 3)
