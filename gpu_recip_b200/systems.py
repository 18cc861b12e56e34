"""Seeded synthetic PME workloads: rigid TIP3P-geometry water boxes.

Every workload is generated from a seed (numpy PCG64), so the same call gives the same atoms on
any machine.  Waters: O-H 0.9572 A, H-O-H 104.52 deg, charges O -0.834 e, H +0.417 e (neutral);
oxygen positions uniform in the box, orientations uniform (random unit quaternions); all atoms
wrapped into [0, L) and stored as float32 (x, y, z, q).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

R_OH = 0.9572
ANGLE_HOH = 104.52
Q_O = -0.834
Q_H = 0.417


def water_box(n_waters: int, box: Sequence[float], seed: int) -> np.ndarray:
    """(3*n_waters, 4) float32 xyzq, atoms ordered O, H, H per water."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64).reshape(3)
    o = rng.random((n_waters, 3)) * box
    h = _hydrogens(rng, o)
    out = np.empty((n_waters, 3, 4))
    out[:, 0, :3] = o
    out[:, 1:, :3] = h
    out[:, :, :3] = np.mod(out[:, :, :3], box)
    out[:, 0, 3] = Q_O
    out[:, 1:, 3] = Q_H
    out = out.reshape(-1, 4).astype(np.float32)
    # float32 rounding of a coordinate just below L can give exactly L: fold it back to 0
    for d in range(3):
        col = out[:, d]
        col[col >= np.float32(box[d])] = 0.0
    return out


def water_cell(n_waters: int, vectors, seed: int) -> np.ndarray:
    """Waters in a triclinic cell whose box vectors are the rows of ``vectors``: oxygens uniform in
    the cell (uniform fractional coordinates), orientations as water_box, every atom wrapped into
    the cell (fractional coordinates in [0, 1)).  (3*n_waters, 4) float32 xyzq."""
    rng = np.random.default_rng(seed)
    B = np.asarray(vectors, dtype=np.float64).reshape(3, 3)
    R = np.linalg.inv(B)
    o = rng.random((n_waters, 3)) @ B
    h = _hydrogens(rng, o)
    xyz = np.concatenate([o[:, None, :], h], axis=1).reshape(-1, 3)
    frac = xyz @ R
    frac -= np.floor(frac)
    out = np.empty((3 * n_waters, 4))
    out[:, :3] = frac @ B
    out[:, 3] = np.tile([Q_O, Q_H, Q_H], n_waters)
    return out.astype(np.float32)


def _hydrogens(rng, o: np.ndarray) -> np.ndarray:
    """(n, 2, 3) hydrogen positions of waters with oxygens at ``o`` and uniform random orientations
    (unit quaternions from ``rng``)."""
    n_waters = o.shape[0]
    q = rng.normal(size=(n_waters, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    rot = np.empty((n_waters, 3, 3))
    rot[:, 0, 0] = 1 - 2 * (y * y + z * z)
    rot[:, 0, 1] = 2 * (x * y - z * w)
    rot[:, 0, 2] = 2 * (x * z + y * w)
    rot[:, 1, 0] = 2 * (x * y + z * w)
    rot[:, 1, 1] = 1 - 2 * (x * x + z * z)
    rot[:, 1, 2] = 2 * (y * z - x * w)
    rot[:, 2, 0] = 2 * (x * z - y * w)
    rot[:, 2, 1] = 2 * (y * z + x * w)
    rot[:, 2, 2] = 1 - 2 * (x * x + y * y)
    half = math.radians(ANGLE_HOH) / 2
    body = np.array([[R_OH * math.sin(half), R_OH * math.cos(half), 0.0],
                     [-R_OH * math.sin(half), R_OH * math.cos(half), 0.0]])
    return o[:, None, :] + np.einsum("nij,kj->nki", rot, body)


def smooth235(lo: int, hi: int) -> List[int]:
    res = []
    for n in range(lo, hi + 1):
        m = n
        for f in (2, 3, 5):
            while m % f == 0:
                m //= f
        if m == 1:
            res.append(n)
    return res


@dataclass
class PmeSystem:
    name: str
    xyzq: np.ndarray
    box: tuple
    nfft: tuple
    order: int
    kappa: float
    vectors: tuple = None     # triclinic box vectors (rows); None for the orthorhombic `box`

    @property
    def recip9(self) -> list:
        """Row-major reciprocal matrix R[j][d] (the inverse of the box-vector matrix)."""
        if self.vectors is None:
            return [1.0 / self.box[0], 0.0, 0.0, 0.0, 1.0 / self.box[1], 0.0, 0.0, 0.0, 1.0 / self.box[2]]
        return [float(v) for v in np.linalg.inv(np.asarray(self.vectors, dtype=np.float64)).reshape(-1)]

    @property
    def natom(self) -> int:
        return self.xyzq.shape[0]

    @property
    def recip3(self):
        return tuple(1.0 / b for b in self.box)

    def alg_bytes(self) -> int:
        """Algorithmic HBM bytes of one evaluation: 44 N + 16 G + 32 H (each stage reads its
        input once and writes its output once, FP32 real and complex grids)."""
        nx, ny, nz = self.nfft
        G = nx * ny * nz
        H = (nx // 2 + 1) * ny * nz
        return 44 * self.natom + 16 * G + 32 * H


def config_small(seed: int = 1) -> PmeSystem:
    """1,000 waters (3,000 atoms), 31.04 A cube, 32^3, order 4, kappa 0.34."""
    L = 31.04
    return PmeSystem("water1k_32", water_box(1000, (L, L, L), seed), (L, L, L), (32, 32, 32), 4, 0.34)


def config_production(order: int = 4, seed: int = 2) -> PmeSystem:
    """8,000 waters (24,000 atoms), 62.1 A cube, 64^3, order 4 or 6, kappa 0.32."""
    L = 62.1
    return PmeSystem(f"water8k_64_p{order}", water_box(8000, (L, L, L), seed), (L, L, L),
                     (64, 64, 64), order, 0.32)


def config_large(seed: int = 3) -> PmeSystem:
    """336,000 waters (1,008,000 atoms), 216 A cube, 216^3, order 6, kappa 0.30."""
    L = 216.0
    return PmeSystem("water336k_216_p6", water_box(336000, (L, L, L), seed), (L, L, L),
                     (216, 216, 216), 6, 0.30)


def config_triclinic_small(order: int = 4, seed: int = 5) -> PmeSystem:
    """1,000 waters (3,000 atoms) in a general triclinic cell a = (32, 0, 0), b = (6, 31, 0),
    c = (-5, 7, 30.5) A (angles 77-101 deg, volume equal to a 31.2 A cube), 32^3, kappa 0.34."""
    V = ((32.0, 0.0, 0.0), (6.0, 31.0, 0.0), (-5.0, 7.0, 30.5))
    return PmeSystem(f"water1k_tric_32_p{order}", water_cell(1000, V, seed), (32.0, 31.0, 30.5),
                     (32, 32, 32), order, 0.34, V)


def config_triclinic(order: int = 4, seed: int = 6) -> PmeSystem:
    """8,000 waters (24,000 atoms) in a rhombic dodecahedron (xy-square form: a = (L, 0, 0),
    b = (0, L, 0), c = (L/2, L/2, L/sqrt 2), L = 69.73 A; the volume of the 62.1 A cube), 64^3,
    order 4 or 6, kappa 0.32."""
    L = 69.73
    V = ((L, 0.0, 0.0), (0.0, L, 0.0), (L / 2, L / 2, L / math.sqrt(2.0)))
    return PmeSystem(f"water8k_dodec_64_p{order}", water_cell(8000, V, seed), (L, L, L / math.sqrt(2.0)),
                     (64, 64, 64), order, 0.32, V)


def batch_systems(count: int = 256, seed: int = 4, order: int = 4, kappa: float = 0.32,
                  min_waters: int = 216, max_waters: int = 8000) -> List[PmeSystem]:
    """Independent orthorhombic water boxes: seeded sizes min..max waters, edges from
    18.6 A (216 waters) to 62.1 A (8,000 waters) at constant density, each axis scaled by up to
    +-10%, grid per axis the 2/3/5-smooth length nearest to 1 A spacing within [24, 64]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(min_waters), math.log(max_waters), size=count))
    sizes = np.round(sizes).astype(int)
    cands = np.array(smooth235(24, 64))
    out = []
    for i, nw in enumerate(sizes):
        L0 = 62.1 * (nw / 8000.0) ** (1.0 / 3.0)
        box = tuple(float(L0 * rng.uniform(0.9, 1.1)) for _ in range(3))
        nfft = tuple(int(cands[np.argmin(np.abs(cands - b))]) for b in box)
        xyzq = water_box(int(nw), box, seed * 100003 + i)
        out.append(PmeSystem(f"batch{i}", xyzq, box, nfft, order, kappa))
    return out
