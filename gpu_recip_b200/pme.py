"""Python mirror of the reference operator interface for the PME reciprocal path.

``CudaPMERecip`` follows CudaPMERecip<AT,CT,CT2> (ap-hynninen/gpu_recip, CudaPMERecip.h:166-203)
method for method -- spread_charge, r2c_fft, scalar_sum, c2r_fft, gather_force,
calc_self_energy, set_stream, set_order, get_nfft{x,y,z}, get_order, print_info -- and
``CudaDomdecRecip`` follows the MD adapter (CudaDomdecRecip.h:9-83).  Energy and virial live in
an ``EnergyVirial`` record that accumulates like CudaEnergyVirial (insert/clear/copyToHost/
getEnergy/getVirial, CudaEnergyVirial.h:13-53).

All compute runs in libpme_b200.so (hand-written sm_100a kernels) through the C ABI of
include/pme_recip.h; torch is used only to hold device memory and streams.  Device arrays are
torch CUDA tensors: xyzq float32 (N, 4) [x, y, z, q]; forces float32 SoA (3*stride,) or
(3, stride), float32 AoS (N, 3), or int64 SoA fixed point (accumulated, scale 2^40).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _capi as C

FFT_COLUMN, FFT_SLAB, FFT_BOX = C.PME_FFT_COLUMN, C.PME_FFT_SLAB, C.PME_FFT_BOX
CCELEC = 332.0716
FORCE_SCALE = float(1 << 40)


def recip_from_box(box: Sequence[float]) -> list:
    """Row-major 3x3 reciprocal box of an orthorhombic box (CudaDomdecRecip.h:17-23)."""
    bx, by, bz = (float(b) for b in box)
    return [1.0 / bx, 0.0, 0.0, 0.0, 1.0 / by, 0.0, 0.0, 0.0, 1.0 / bz]


def recip_from_box_vectors(vectors) -> list:
    """Row-major reciprocal matrix R[j][d] (recip[3 j + d]) of a box whose vectors a, b, c are the
    rows of ``vectors``: R is the inverse of that matrix, so the fractional coordinate along d is
    sum_j x_j R[j][d].  A diagonal result is the orthorhombic case."""
    B = np.asarray(vectors, dtype=np.float64).reshape(3, 3)
    if not np.all(np.isfinite(B)) or abs(np.linalg.det(B)) == 0.0:
        raise ValueError("box vectors must be finite and span a volume")
    return [float(v) for v in np.linalg.inv(B).reshape(-1)]


def force_stride(n: int, itemsize: int = 4) -> int:
    """SoA force stride padded to 256 bytes, as Force<T> (Force.h:63-69)."""
    return ((((n - 1 + 32) * itemsize) - 1) // 256 + 1) * 256 // itemsize


TRACE_STEP_STAMPS = 32   # entries after the per-CTA phase stamps of a single-system trace


def _trace_ctas(buf, max_ctas: int, extra: int) -> int:
    """CTAs a trace buffer of buf.numel() int64 entries holds (14 each, then `extra`); a
    max_ctas that does not fit raises instead of letting the kernel write past the buffer."""
    import torch
    if buf.dtype != torch.int64 or not buf.is_cuda:
        raise ValueError("trace buffer must be an int64 CUDA tensor")
    fit = (buf.numel() - extra) // 14
    n = int(max_ctas) if max_ctas else fit
    if n < 1 or n > fit:
        raise ValueError(f"trace buffer of {buf.numel()} entries holds {max(fit, 0)} CTAs (14 entries each"
                         f" + {extra}); asked for {n}")
    return n


def _stream_handle(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)  # torch.cuda.Stream


def _ptr(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    if isinstance(t, int):
        return ctypes.c_void_p(t)
    if not t.is_cuda:
        raise ValueError("device tensor expected")
    if not t.is_contiguous():
        raise ValueError("contiguous tensor expected")
    return ctypes.c_void_p(t.data_ptr())


def _xyzq_ptr(xyzq, ncoord: int):
    import torch
    if isinstance(xyzq, int):
        return ctypes.c_void_p(xyzq)
    if xyzq.dtype != torch.float32:
        raise ValueError("xyzq must be float32 (x, y, z, q)")
    if xyzq.numel() < 4 * ncoord:
        raise ValueError("xyzq holds fewer than ncoord atoms")
    return _ptr(xyzq)


class EnergyVirial:
    """Energy/virial record (accumulating), the CudaEnergyVirial role for the PME terms."""

    def __init__(self):
        self._owner: Optional["CudaPMERecip"] = None
        self._names = {}
        self._host = np.zeros(C.PME_EV_COUNT)

    def insert(self, name: str, slot: int):
        self._names[name] = slot

    def _bind(self, owner: "CudaPMERecip"):
        self._owner = owner

    def clear(self):
        if self._owner is not None:
            C.check(C.load().pme_clear_energy_virial(self._owner._h), "clear")
        self._host[:] = 0.0

    def copyToHost(self):
        e = ctypes.c_double()
        s = ctypes.c_double()
        v = (ctypes.c_double * 9)()
        C.check(C.load().pme_get_energy_virial(self._owner._h, ctypes.byref(e), ctypes.byref(s), v),
                "copyToHost")
        self._host[C.PME_EV_RECIP] = e.value
        self._host[C.PME_EV_SELF] = s.value
        self._host[C.PME_EV_VIRIAL:] = np.array(v[:])

    def getEnergy(self, name: str) -> float:
        return float(self._host[self._names[name]])

    def getVirial(self) -> np.ndarray:
        return self._host[C.PME_EV_VIRIAL:].reshape(3, 3).copy()

    def copy_async(self, dst) -> None:
        """Enqueue a copy of the record (11 doubles) into ``dst`` (pinned host or device tensor)."""
        C.check(C.load().pme_copy_energy_virial_async(self._owner._h, ctypes.c_void_p(dst.data_ptr())),
                "copy_async")

    def device_ptr(self) -> int:
        p = ctypes.c_void_p()
        C.check(C.load().pme_energy_virial_device_ptr(self._owner._h, ctypes.byref(p)), "ev ptr")
        return int(p.value)


class CudaPMERecip:
    """B200 smooth-PME reciprocal operator (int64 fixed-point grid, FP32 FFT/solve/gather)."""

    def __init__(self, nfftx: int, nffty: int, nfftz: int, order: int, fft_type: int = FFT_BOX,
                 nnode: int = 1, mynode: int = 0, energy_virial: Optional[EnergyVirial] = None,
                 name_recip: str = "recip", name_self: str = "self", stream=None):
        lib = C.load()
        h = ctypes.c_void_p()
        C.check(lib.pme_create(nfftx, nffty, nfftz, order, fft_type, nnode, mynode,
                               ctypes.c_void_p(_stream_handle(stream)), ctypes.byref(h)),
                "CudaPMERecip")
        self._h = h
        self._lib = lib
        self.nfft = (nfftx, nffty, nfftz)
        self.energy_virial = energy_virial if energy_virial is not None else EnergyVirial()
        self.energy_virial.insert(name_recip, C.PME_EV_RECIP)
        self.energy_virial.insert(name_self, C.PME_EV_SELF)
        self.energy_virial._bind(self)

    # -- lifetime -------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.pme_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration --------------------------------------------------------------------------
    def set_stream(self, stream):
        C.check(self._lib.pme_set_stream(self._h, ctypes.c_void_p(_stream_handle(stream))), "set_stream")

    def set_order(self, order: int):
        C.check(self._lib.pme_set_order(self._h, order), "set_order")

    def get_nfftx(self):
        return self.nfft[0]

    def get_nffty(self):
        return self.nfft[1]

    def get_nfftz(self):
        return self.nfft[2]

    def get_order(self) -> int:
        o = ctypes.c_int()
        C.check(self._lib.pme_get_order(self._h, ctypes.byref(o)), "get_order")
        return o.value

    def print_info(self):
        C.check(self._lib.pme_print_info(self._h), "print_info")

    # -- stages ---------------------------------------------------------------------------------
    def spread_charge(self, xyzq, ncoord: int, recip):
        C.check(self._lib.pme_spread_charge(self._h, _xyzq_ptr(xyzq, ncoord), ncoord, C.dbl9(recip)),
                "spread_charge")

    def r2c_fft(self):
        C.check(self._lib.pme_r2c_fft(self._h), "r2c_fft")

    def scalar_sum(self, recip, kappa: float, calc_energy: bool, calc_virial: bool):
        C.check(self._lib.pme_scalar_sum(self._h, C.dbl9(recip), float(kappa), int(calc_energy),
                                         int(calc_virial)), "scalar_sum")

    def c2r_fft(self):
        C.check(self._lib.pme_c2r_fft(self._h), "c2r_fft")

    @staticmethod
    def _force_kind(force, stride: int):
        import torch
        if force.dtype == torch.int64:
            return C.PME_FORCE_I64_SOA_ACCUM
        if force.dtype != torch.float32:
            raise ValueError("force must be float32 or int64")
        if force.dim() == 2 and force.shape[1] == 3 and stride in (1, 0):
            return C.PME_FORCE_F32X3
        return C.PME_FORCE_F32_SOA

    def gather_force(self, xyzq, ncoord: int, recip, stride: int, force, kind: Optional[int] = None):
        k = self._force_kind(force, stride) if kind is None else kind
        if k != C.PME_FORCE_F32X3 and force.numel() < 2 * stride + ncoord:
            raise ValueError("force too small for 3 strided blocks")
        C.check(self._lib.pme_gather_force(self._h, _xyzq_ptr(xyzq, ncoord), ncoord, C.dbl9(recip),
                                           int(stride), k, _ptr(force)), "gather_force")

    def calc_self_energy(self, xyzq, ncoord: int, kappa: float):
        C.check(self._lib.pme_calc_self_energy(self._h, _xyzq_ptr(xyzq, ncoord), ncoord, float(kappa)),
                "calc_self_energy")

    # -- fused evaluation (CudaDomdecRecip::calc) -----------------------------------------------
    def set_energy_virial_mirror(self, host_tensor=None):
        """Each later fused evaluation also writes its own [E_recip, E_self, W(9)] record into
        ``host_tensor`` (a pinned float64 CPU tensor of 11 values), or stop with None."""
        if host_tensor is not None and (host_tensor.numel() < 11 or not host_tensor.is_pinned()):
            raise ValueError("the mirror must be a pinned tensor of at least 11 float64 values")
        self._mirror = host_tensor   # keep it alive
        ptr = None if host_tensor is None else ctypes.c_void_p(host_tensor.data_ptr())
        C.check(self._lib.pme_set_energy_virial_mirror(self._h, ptr), "set_energy_virial_mirror")

    def eval(self, recip, xyzq, ncoord: int, kappa: float, calc_energy: bool, calc_virial: bool,
             force, stride: int = 0, kind: Optional[int] = None):
        """Fused evaluation for any box (pme_eval): recip is the row-major reciprocal matrix,
        orthorhombic (diagonal) or triclinic."""
        k = self._force_kind(force, stride) if kind is None else kind
        C.check(self._lib.pme_eval(self._h, C.dbl9(recip), _xyzq_ptr(xyzq, ncoord), ncoord,
                                   float(kappa), int(calc_energy), int(calc_virial), k, _ptr(force),
                                   int(stride)), "eval")

    def eval_host(self, recip, xyzq, ncoord: int, kappa: float, calc_energy: bool, calc_virial: bool,
                  force, stride: int = 0, kind: Optional[int] = None):
        """pme_eval from and to page-locked host tensors (``tensor.pin_memory()``): the evaluation
        reads the coordinates over the bus itself and the forces come back by one copy on the
        stream; they are in ``force`` once the stream has passed the call."""
        import torch
        for t, what in ((xyzq, "xyzq"), (force, "force")):
            if not isinstance(t, torch.Tensor) or t.is_cuda or not t.is_pinned() or not t.is_contiguous():
                raise ValueError(f"{what} must be a contiguous pinned host tensor")
        if xyzq.dtype != torch.float32 or xyzq.numel() < 4 * ncoord:
            raise ValueError("xyzq must be float32 (x, y, z, q) for ncoord atoms")
        k = self._force_kind(force, stride) if kind is None else kind
        C.check(self._lib.pme_eval_host(self._h, C.dbl9(recip), ctypes.c_void_p(xyzq.data_ptr()), ncoord,
                                        float(kappa), int(calc_energy), int(calc_virial), k,
                                        ctypes.c_void_p(force.data_ptr()), int(stride)), "eval_host")

    def eval_ortho(self, inv_box, xyzq, ncoord: int, kappa: float, calc_energy: bool,
                   calc_virial: bool, force, stride: int = 0, kind: Optional[int] = None):
        k = self._force_kind(force, stride) if kind is None else kind
        C.check(self._lib.pme_eval_ortho(self._h, float(inv_box[0]), float(inv_box[1]),
                                         float(inv_box[2]), _xyzq_ptr(xyzq, ncoord), ncoord,
                                         float(kappa), int(calc_energy), int(calc_virial), k,
                                         _ptr(force), int(stride)), "eval_ortho")

    # -- grid read-back (synchronising) ---------------------------------------------------------
    def charge_grid_fixed(self) -> np.ndarray:
        nx, ny, nz = self.nfft
        out = np.empty((nz, ny, nx), dtype=np.int64)
        C.check(self._lib.pme_copy_charge_grid_fixed(self._h, out.ctypes.data_as(ctypes.c_void_p)),
                "charge_grid_fixed")
        return out

    def charge_grid(self) -> np.ndarray:
        nx, ny, nz = self.nfft
        out = np.empty((nz, ny, nx), dtype=np.float32)
        C.check(self._lib.pme_copy_charge_grid(self._h, out.ctypes.data_as(ctypes.c_void_p)),
                "charge_grid")
        return out

    def fft_grid(self) -> np.ndarray:
        nx, ny, nz = self.nfft
        out = np.empty((nz, ny, nx // 2 + 1, 2), dtype=np.float32)
        C.check(self._lib.pme_copy_fft_grid(self._h, out.ctypes.data_as(ctypes.c_void_p)), "fft_grid")
        return out.view(np.complex64)[..., 0]

    def load_charge_grid(self, grid: np.ndarray):
        nx, ny, nz = self.nfft
        g = np.ascontiguousarray(grid, dtype=np.float32).reshape(nz, ny, nx)
        C.check(self._lib.pme_load_charge_grid(self._h, g.ctypes.data_as(ctypes.c_void_p)),
                "load_charge_grid")

    # -- failure detection ----------------------------------------------------------------------
    def get_status(self) -> int:
        """Synchronise; raise PMEError(PME_ETIMEOUT) if a fused evaluation's barrier wait gave up
        (the sticky device status is cleared and the handle reset), else return 0."""
        st = ctypes.c_int()
        C.check(self._lib.pme_get_status(self._h, ctypes.byref(st)), "get_status")
        return st.value

    def reserve_atoms(self, natom: int):
        """Pre-size the fused evaluation's atom bins (call before CUDA-graph capture)."""
        C.check(self._lib.pme_reserve_atoms(self._h, int(natom)), "reserve_atoms")

    def set_barrier_spin_limit(self, polls: int):
        C.check(self._lib.pme_set_barrier_spin_limit(self._h, int(polls)), "set_barrier_spin_limit")

    def set_trace(self, buf, max_ctas: int = 0):
        """Record per-CTA, per-phase %globaltimer stamps of fused evaluations into ``buf`` (int64
        device tensor of max_ctas*14 entries plus 32 step stamps of CTA 0); None turns it off."""
        if buf is None:
            C.check(self._lib.pme_set_trace(self._h, None, 0), "set_trace")
        else:
            n = _trace_ctas(buf, max_ctas, TRACE_STEP_STAMPS)
            C.check(self._lib.pme_set_trace(self._h, _ptr(buf), n), "set_trace")

    def set_fft_schedule(self, schedule: int):
        """PME_SCHED_AUTO / PME_SCHED_PLANES / PME_SCHED_PASSES / PME_SCHED_CLUSTER (identical results)."""
        C.check(self._lib.pme_set_fft_schedule(self._h, int(schedule)), "set_fft_schedule")

    def set_x_gather_fusion(self, mode: int):
        """PME_XGATHER_AUTO (default) / PME_XGATHER_OFF (identical results)."""
        C.check(self._lib.pme_set_x_gather_fusion(self._h, int(mode)), "set_x_gather_fusion")

    def autotune(self, inv_box, xyzq, ncoord: int, kappa: float, reps: int = 10) -> dict:
        """Measure launch shapes of the fused evaluation on this system and keep the fastest
        (pme_autotune); returns the chosen shape and its time per evaluation."""
        c = C.TuneConfig()
        C.check(self._lib.pme_autotune(self._h, _xyzq_ptr(xyzq, ncoord), int(ncoord), float(inv_box[0]),
                                       float(inv_box[1]), float(inv_box[2]), float(kappa), int(reps),
                                       ctypes.byref(c)), "autotune")
        return c.as_dict()

    def get_tune_config(self) -> dict:
        c = C.TuneConfig()
        C.check(self._lib.pme_get_tune_config(self._h, ctypes.byref(c)), "get_tune_config")
        return c.as_dict()

    def set_tune_config(self, **cfg):
        c = C.TuneConfig()
        C.check(self._lib.pme_get_tune_config(self._h, ctypes.byref(c)), "get_tune_config")
        for k, v in cfg.items():
            setattr(c, k, v)
        C.check(self._lib.pme_set_tune_config(self._h, ctypes.byref(c)), "set_tune_config")

    def set_fault_injection(self, what: int):
        C.check(self._lib.pme_set_fault_injection(self._h, int(what)), "set_fault_injection")

    def solved_grid(self) -> np.ndarray:
        nx, ny, nz = self.nfft
        out = np.empty((nz, ny, nx), dtype=np.float32)
        C.check(self._lib.pme_copy_solved_grid(self._h, out.ctypes.data_as(ctypes.c_void_p)),
                "solved_grid")
        return out


class CudaDomdecRecip:
    """MD adapter: calc(inv_box..., coord, ncoord, calc_energy, calc_virial, force) runs the whole
    reciprocal evaluation (CudaDomdecRecip.h:50-81).  ``force`` may be an int64 SoA fixed-point
    array (accumulated), a float32 SoA array (overwritten) or a float32 (N, 3) array."""

    def __init__(self, nfftx, nffty, nfftz, order, kappa, energy_virial=None, name_recip="recip",
                 name_self="self", stream=None):
        self.kappa = float(kappa)
        self.pme = CudaPMERecip(nfftx, nffty, nfftz, order, FFT_BOX, 1, 0, energy_virial,
                                name_recip, name_self, stream)

    def set_stream(self, stream):
        self.pme.set_stream(stream)

    def calc(self, inv_boxx, inv_boxy, inv_boxz, coord, ncoord, calc_energy, calc_virial, force,
             stride: Optional[int] = None):
        if stride is None:
            stride = 1 if (force.dim() == 2 and force.shape[1] == 3) else force.numel() // 3
        self.pme.eval_ortho((inv_boxx, inv_boxy, inv_boxz), coord, ncoord, self.kappa, calc_energy,
                            calc_virial, force, stride)


class PmeBatch:
    """Many independent systems evaluated by one persistent launch (pme_batch_* of the C ABI).

    ``systems`` is a sequence of dicts with keys nfft (3,), order, box (3,), kappa, xyzq (device
    float32 (N,4) tensor), force (device tensor) and optionally force_kind, stride, calc_energy,
    calc_virial.  Device tensors must stay alive while the batch is used."""

    def __init__(self, systems, stream=None):
        lib = C.load()
        n = len(systems)
        arr = (C.SystemDesc * n)()
        self._keep = []
        for i, s in enumerate(systems):
            x, f = s["xyzq"], s["force"]
            natom = int(s.get("natom", x.shape[0]))
            kind = s.get("force_kind")
            stride = int(s.get("stride", 0))
            if kind is None:
                kind = CudaPMERecip._force_kind(f, stride)
            nx, ny, nz = s["nfft"]
            arr[i].nfftx, arr[i].nffty, arr[i].nfftz = int(nx), int(ny), int(nz)
            arr[i].order = int(s["order"])
            arr[i].natom = natom
            for d in range(3):
                arr[i].box[d] = float(s["box"][d])
            arr[i].kappa = float(s["kappa"])
            arr[i].xyzq = _xyzq_ptr(x, natom).value
            arr[i].force = _ptr(f).value
            arr[i].force_kind = int(kind)
            arr[i].stride = stride
            arr[i].calc_energy = int(s.get("calc_energy", True))
            arr[i].calc_virial = int(s.get("calc_virial", True))
            self._keep.append((x, f))
        h = ctypes.c_void_p()
        C.check(lib.pme_batch_create(ctypes.cast(arr, ctypes.c_void_p), n,
                                     ctypes.c_void_p(_stream_handle(stream)), ctypes.byref(h)),
                "pme_batch_create")
        self._h = h
        self._lib = lib
        self.nsys = n

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.pme_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        C.check(self._lib.pme_batch_set_stream(self._h, ctypes.c_void_p(_stream_handle(stream))), "set_stream")

    def set_system(self, i: int, box=None, xyzq=None, force=None):
        b = (ctypes.c_double * 3)(*[float(v) for v in box]) if box is not None else None
        C.check(self._lib.pme_batch_set_system(self._h, int(i), b, _ptr(xyzq) if xyzq is not None else None,
                                               _ptr(force) if force is not None else None), "set_system")

    def commit(self):
        C.check(self._lib.pme_batch_commit(self._h), "commit")

    def eval(self):
        C.check(self._lib.pme_batch_eval(self._h), "batch eval")

    def clear_energy_virial(self):
        C.check(self._lib.pme_batch_clear_energy_virial(self._h), "batch clear")

    def energy_virial(self) -> np.ndarray:
        """(nsys, 11): [E_recip, E_self, W_xx .. W_zz] per system (synchronising)."""
        out = np.zeros((self.nsys, C.PME_EV_COUNT))
        C.check(self._lib.pme_batch_get_energy_virial(self._h, out.ctypes.data_as(C._DP)), "batch ev")
        return out

    def set_trace(self, buf, max_ctas: int = 0):
        """Per-CTA, per-phase stamps of the batch launch into ``buf`` (int64 device tensor of at
        least max_ctas*14 entries); None turns it off."""
        if buf is None:
            C.check(self._lib.pme_batch_set_trace(self._h, None, 0), "set_trace")
        else:
            C.check(self._lib.pme_batch_set_trace(self._h, _ptr(buf), _trace_ctas(buf, max_ctas, 0)), "set_trace")

    def autotune(self, reps: int = 5) -> dict:
        """Measure the batch's y/z schedule and launch size and keep the fastest."""
        c = C.TuneConfig()
        C.check(self._lib.pme_batch_autotune(self._h, int(reps), ctypes.byref(c)), "batch autotune")
        return c.as_dict()

    def info(self):
        n = ctypes.c_int()
        g = ctypes.c_int()
        b = ctypes.c_size_t()
        C.check(self._lib.pme_batch_info(self._h, ctypes.byref(n), ctypes.byref(g), ctypes.byref(b)), "info")
        return {"nsys": n.value, "grid_ctas": g.value, "device_bytes": b.value}


def _real_type(t) -> int:
    import torch
    if t.dtype == torch.float64:
        return C.PME_REAL_F64
    if t.dtype == torch.float32:
        return C.PME_REAL_F32
    raise ValueError("float32 or float64 force array expected")


def force_convert(force_i64, stride: int, ncoord: int, out=None, out_stride: Optional[int] = None, stream=None):
    """Force<long long>::convert (Force.cu:103-157): int64 SoA forces at 2^40 (rows of ``stride``)
    to float32 or float64 SoA rows of ``out_stride`` in ``out``; with ``out`` None the conversion
    is in place to float64 and the float64 view of the same storage is returned (convert<double>(),
    as CudaPMEForcefield.cu:514 does at the end of an MD step)."""
    import torch
    if force_i64.dtype != torch.int64:
        raise ValueError("int64 fixed-point force array expected")
    if out is None:
        out, out_stride = force_i64.view(torch.float64), stride
    if out_stride is None:
        out_stride = stride
    C.check(C.load().pme_force_convert(_ptr(force_i64), int(stride), int(ncoord), _ptr(out), int(out_stride),
                                       _real_type(out), _stream_handle(stream)), "force_convert")
    return out


def force_convert_add(force_i64, stride: int, ncoord: int, add, add_stride: Optional[int] = None, stream=None):
    """Force<long long>::convert_add (Force.cu:167-184): in place, int64 SoA forces at 2^40 become
    float64 v 2^-40 + add (float32 or float64 SoA rows); returns the float64 view."""
    import torch
    if force_i64.dtype != torch.int64:
        raise ValueError("int64 fixed-point force array expected")
    C.check(C.load().pme_force_convert_add(_ptr(force_i64), int(stride), int(ncoord), _ptr(add),
                                           int(add_stride if add_stride is not None else stride), _real_type(add),
                                           _stream_handle(stream)), "force_convert_add")
    return force_i64.view(torch.float64)


def system_device_bytes(nfft) -> int:
    return int(C.load().pme_system_device_bytes(int(nfft[0]), int(nfft[1]), int(nfft[2])))


def tune_cache_clear() -> None:
    """Forget the launch shapes pme_autotune stored for later handles of the same grid."""
    C.check(C.load().pme_tune_cache_clear(), "tune_cache_clear")


class PmeServer:
    """Request loop with continuous batching (pme_server_* of the C ABI).

    submit() takes one system (a PmeSystem-like object with xyzq, box, nfft, order, kappa) and a
    number of evaluations on its coordinates plus a seeded Gaussian jitter of sigma (A); wait()
    returns that request's per-evaluation energy/virial records, the last evaluation's forces and
    its submit / admission / completion times."""

    def __init__(self, device_bytes: int, max_active: int = 256, stream=None):
        self._lib = C.load()
        h = ctypes.c_void_p()
        C.check(self._lib.pme_server_create(int(device_bytes), int(max_active),
                                            ctypes.c_void_p(_stream_handle(stream)), ctypes.byref(h)),
                "pme_server_create")
        self._h = h
        self._live = {}

    @staticmethod
    def _request(system, n_evals, sigma, seed, ev, force, calc_energy=True, calc_virial=True):
        x = np.ascontiguousarray(system.xyzq, dtype=np.float32)
        r = C.Request()
        r.nfftx, r.nffty, r.nfftz = (int(v) for v in system.nfft)
        r.order = int(system.order)
        r.natom = int(x.shape[0])
        for d in range(3):
            r.box[d] = float(system.box[d])
        r.kappa = float(system.kappa)
        r.xyzq = x.ctypes.data
        r.n_evals = int(n_evals)
        r.sigma = float(sigma)
        r.seed = int(seed)
        r.calc_energy, r.calc_virial = int(calc_energy), int(calc_virial)
        r.ev_out = ev.ctypes.data
        r.force_out = force.ctypes.data if force is not None else None
        return r, x

    @staticmethod
    def request_device_bytes(system, n_evals: int = 1) -> int:
        ev = np.zeros((max(int(n_evals), 1), C.PME_EV_COUNT))
        r, _ = PmeServer._request(system, n_evals, 0.0, 0, ev, None)
        return int(C.load().pme_request_device_bytes(ctypes.byref(r)))

    def submit(self, system, n_evals: int = 1, sigma: float = 0.0, seed: int = 0, forces: bool = True) -> int:
        ev = np.zeros((int(n_evals), C.PME_EV_COUNT), dtype=np.float64)
        force = np.zeros((system.xyzq.shape[0], 3), dtype=np.float32) if forces else None
        r, x = self._request(system, n_evals, sigma, seed, ev, force)
        rid = ctypes.c_longlong()
        C.check(self._lib.pme_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)), "server submit")
        self._live[rid.value] = (ev, force, x)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> dict:
        t = (ctypes.c_double * 3)()
        rc = self._lib.pme_server_wait(self._h, ctypes.c_longlong(rid), float(timeout), t)
        ev, force, _ = self._live.pop(rid) if rc == C.PME_OK else self._live.get(rid, (None, None, None))
        C.check(rc, "server wait")
        return {"ev": ev, "force": force, "t_submit": t[0], "t_admit": t[1], "t_done": t[2],
                "latency": t[2] - t[0]}

    def stats(self) -> dict:
        st = C.ServerStats()
        C.check(self._lib.pme_server_get_stats(self._h, ctypes.byref(st)), "server stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.pme_server_destroy(self._h)
            self._h = ctypes.c_void_p()
        self._live = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
