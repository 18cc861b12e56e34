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
