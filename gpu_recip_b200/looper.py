"""The recip node's request loop, in process.

The reference runs the reciprocal part on pure recip nodes (CudaDomdecRecipLooper::run,
CudaDomdecRecipLooper.cu:3-36): each step it receives a header from the direct nodes
(DomdecRecipComm.h:11-15: inverse box edges, the coordinate count and whether to compute energy
and virial; a negative count means STOP, DomdecRecipComm.cpp:144-179), then the coordinates, runs
CudaDomdecRecip::calc and sends back float3 forces.  Here the two sides share a process: the
direct side posts messages on one queue and reads replies from another; the recip side runs the
same loop over CudaDomdecRecip (one fused evaluation per step).
"""
from __future__ import annotations

import ctypes
import queue
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .pme import CudaDomdecRecip


@dataclass
class RecipHeader:
    """The per-step header of the direct -> recip exchange (DomdecRecipComm.h:11-15)."""
    inv_boxx: float
    inv_boxy: float
    inv_boxz: float
    ncoord: int
    calc_energy: bool
    calc_virial: bool


@dataclass
class RecipReply:
    """What goes back to the direct side: float3 forces (N, 3) and this step's energy/virial
    record [E_recip, E_self, W_xx ... W_zz] (zeros where not asked for)."""
    force: object
    energy_virial: np.ndarray


class InProcessRecipComm:
    """Both ends of the direct <-> recip exchange over two queues (the role of
    CudaDomdecRecipComm without MPI).  Coordinates and forces are device tensors."""

    def __init__(self, timeout: float = 60.0):
        self._to_recip: queue.Queue = queue.Queue()
        self._to_direct: queue.Queue = queue.Queue()
        self.timeout = timeout

    # ---- direct side (DomdecRecipComm::send_header / send_coord / recv_force / send_stop)
    def send_header(self, ncoord: int, inv_boxx: float, inv_boxy: float, inv_boxz: float,
                    calc_energy: bool, calc_virial: bool) -> None:
        self._to_recip.put(RecipHeader(float(inv_boxx), float(inv_boxy), float(inv_boxz), int(ncoord),
                                       bool(calc_energy), bool(calc_virial)))

    def send_coord(self, xyzq) -> None:
        self._to_recip.put(xyzq)

    def recv_force(self) -> RecipReply:
        return self._to_direct.get(timeout=self.timeout)

    def send_stop(self) -> None:
        self.send_header(-1, 1.0, 1.0, 1.0, False, False)

    # ---- recip side (recv_header / recv_coord / send_force)
    def recv_header(self) -> Optional[RecipHeader]:
        """The next header, or None on STOP (a negative coordinate count)."""
        h = self._to_recip.get(timeout=self.timeout)
        return None if h.ncoord < 0 else h

    def recv_coord(self):
        return self._to_recip.get(timeout=self.timeout)

    def send_force(self, reply: RecipReply) -> None:
        self._to_direct.put(reply)


class RecipLooper:
    """CudaDomdecRecipLooper: receive header, stop on STOP, receive coordinates, evaluate, send
    forces, until STOP.  The force buffer grows with the coordinate count as the reference's
    reallocate<float3> does; every reply carries a fresh copy of the forces."""

    def __init__(self, comm: InProcessRecipComm, nfftx: int, nffty: int, nfftz: int, order: int,
                 kappa: float, stream=None):
        self.comm = comm
        self.recip = CudaDomdecRecip(nfftx, nffty, nfftz, order, kappa, stream=stream)
        self._force = None
        self.steps = 0

    def run(self) -> int:
        import torch
        while True:
            h = self.comm.recv_header()
            if h is None:
                break
            xyzq = self.comm.recv_coord()
            n = h.ncoord
            if self._force is None or self._force.shape[0] < n:
                self._force = torch.zeros((max(n, 1), 3), dtype=torch.float32, device=xyzq.device)
            ev = self.recip.pme.energy_virial
            ev.clear()
            self.recip.calc(h.inv_boxx, h.inv_boxy, h.inv_boxz, xyzq, n, h.calc_energy, h.calc_virial,
                            self._force, 1)
            torch.cuda.synchronize()
            ev.copyToHost()
            rec = np.zeros(11)
            rec[0] = ev.getEnergy("recip")
            rec[1] = ev.getEnergy("self")
            rec[2:] = ev.getVirial().reshape(-1)
            self.comm.send_force(RecipReply(self._force[:n].clone(), rec))
            self.steps += 1
        return self.steps


_CUDART = None


def _cudart():
    """The CUDA runtime library, for a device-to-device copy of the loop's force buffer."""
    global _CUDART
    if _CUDART is None:
        import ctypes.util
        for name in ("libcudart.so", "libcudart.so.12", ctypes.util.find_library("cudart"),
                     "/usr/local/cuda/lib64/libcudart.so"):
            if not name:
                continue
            try:
                _CUDART = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if _CUDART is None:
            raise RuntimeError("the CUDA runtime library was not found")
    return _CUDART


class NativeRecipLooper:
    """The same loop run by the library itself (pme_recip_loop_run, C++ behind the C ABI): its
    three transport callbacks read headers and coordinates from an InProcessRecipComm and post
    the replies to it, so a direct side written against the queue protocol talks to the native
    loop unchanged.  Each reply carries a copy of the step's float3 forces and its own
    energy/virial record."""

    def __init__(self, comm: InProcessRecipComm, nfftx: int, nffty: int, nfftz: int, order: int,
                 kappa: float, stream=None):
        from . import _capi as C
        from .pme import CudaPMERecip
        self.comm = comm
        self.kappa = float(kappa)
        self.pme = CudaPMERecip(nfftx, nffty, nfftz, order, stream=stream)
        self._coords = None
        self.steps = 0

        def recv_header(user, hdr):
            try:
                h = comm._to_recip.get(timeout=comm.timeout)
            except Exception:
                return 1
            hdr.contents.inv_boxx, hdr.contents.inv_boxy, hdr.contents.inv_boxz = h.inv_boxx, h.inv_boxy, h.inv_boxz
            hdr.contents.ncoord = h.ncoord
            hdr.contents.calc_energy, hdr.contents.calc_virial = int(h.calc_energy), int(h.calc_virial)
            return 0

        def recv_coord(user, ncoord, stream_ptr, out):
            try:
                self._coords = comm.recv_coord()
            except Exception:
                return 1
            out[0] = self._coords.data_ptr() if ncoord > 0 else None
            return 0

        def send_force(user, ncoord, force_ptr, ev):
            import torch
            f = torch.empty((max(ncoord, 0), 3), dtype=torch.float32, device=self._coords.device)
            if ncoord > 0 and _cudart().cudaMemcpy(ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(force_ptr),
                                                  ctypes.c_size_t(12 * ncoord), 3) != 0:   # device to device
                return 1
            comm.send_force(RecipReply(f, np.ctypeslib.as_array(ev, shape=(11,)).copy()))
            return 0

        self._cb = C.RecipComm(None, C.RECV_HEADER(recv_header), C.RECV_COORD(recv_coord), C.SEND_FORCE(send_force))

    def run(self) -> int:
        from . import _capi as C
        n = ctypes.c_longlong(0)
        C.check(C.load().pme_recip_loop_run(self.pme._h, self.kappa, ctypes.byref(self._cb), ctypes.byref(n)),
                "pme_recip_loop_run")
        self.steps = n.value
        return self.steps

