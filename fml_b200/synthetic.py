"""Seeded synthetic molecules standing in for QM7-like data.

No public dataset is used. Molecules are drawn as follows, identically for
every workload:

* atom count ``n ~ U{4..nmax}``;
* charges ``Z ~ Cat{1: .50, 6: .35, 7: .07, 8: .07, 16: .01}``;
* positions uniform in a ball of radius ``1.5 * n**(1/3)`` Angstrom, by
  rejection with a minimum pair distance of 0.9 Angstrom;
* target ``y = sum_{i<j} Z_i Z_j / r_ij + N(0, 0.1**2)``.

Molecules are returned packed and ragged: ``charges`` (total_atoms,),
``coords`` (total_atoms, 3) and ``offsets`` (nmol + 1,) int32, which is the
layout the batched descriptor kernels take.
"""

from dataclasses import dataclass

import numpy as np

_Z_VALUES = np.array([1, 6, 7, 8, 16], dtype=np.float64)
_Z_PROBS = np.array([0.50, 0.35, 0.07, 0.07, 0.01])
MIN_PAIR_DIST = 0.9


@dataclass
class MoleculeBatch:
    charges: np.ndarray  # (total_atoms,) float64
    coords: np.ndarray  # (total_atoms, 3) float64
    offsets: np.ndarray  # (nmol + 1,) int32
    energies: np.ndarray  # (nmol,) float64 target y

    @property
    def nmol(self):
        return len(self.offsets) - 1

    @property
    def natoms(self):
        return np.diff(self.offsets)

    def molecule(self, i):
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return self.charges[a:b], self.coords[a:b]

    def subset(self, idx):
        idx = np.asarray(idx)
        counts = self.natoms[idx]
        offs = np.zeros(len(idx) + 1, dtype=np.int32)
        np.cumsum(counts, out=offs[1:])
        sel = np.concatenate([np.arange(self.offsets[i], self.offsets[i + 1]) for i in idx]) \
            if len(idx) else np.zeros(0, dtype=np.int64)
        return MoleculeBatch(self.charges[sel], self.coords[sel], offs, self.energies[idx])


def generate(nmol, nmax=23, seed=0, nmin=4):
    """Generate ``nmol`` molecules with ``nmin..nmax`` atoms from ``seed``."""
    rng = np.random.default_rng(seed)
    n = rng.integers(nmin, nmax + 1, size=nmol)
    radius = 1.5 * np.cbrt(n.astype(np.float64))
    Z = rng.choice(_Z_VALUES, size=(nmol, nmax), p=_Z_PROBS)
    pos = np.zeros((nmol, nmax, 3))
    min2 = MIN_PAIR_DIST * MIN_PAIR_DIST
    for slot in range(nmax):
        need = np.nonzero(n > slot)[0]
        while len(need):
            # uniform point in the ball of each molecule's radius
            u = rng.standard_normal((len(need), 3))
            u /= np.linalg.norm(u, axis=1, keepdims=True)
            r = radius[need] * np.cbrt(rng.random(len(need)))
            cand = u * r[:, None]
            if slot:
                d2 = ((pos[need, :slot, :] - cand[:, None, :]) ** 2).sum(-1)
                ok = (d2 >= min2).all(axis=1)
            else:
                ok = np.ones(len(need), dtype=bool)
            pos[need[ok], slot] = cand[ok]
            need = need[~ok]
    offsets = np.zeros(nmol + 1, dtype=np.int32)
    np.cumsum(n, out=offsets[1:])
    mask = np.arange(nmax)[None, :] < n[:, None]
    charges = Z[mask]
    coords = pos[mask]
    # target: Coulomb sum over atom pairs plus noise
    diff = pos[:, :, None, :] - pos[:, None, :, :]
    r = np.sqrt((diff ** 2).sum(-1))
    pair = np.triu(mask[:, :, None] & mask[:, None, :], k=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        e = np.where(pair, Z[:, :, None] * Z[:, None, :] / np.where(pair, r, 1.0), 0.0)
    y = e.sum(axis=(1, 2)) + rng.normal(0.0, 0.1, size=nmol)
    return MoleculeBatch(charges.astype(np.float64), coords.astype(np.float64), offsets, y)


#: seeds of the standard synthetic workloads
SEEDS = {"cm_small": 0, "arad": 1, "cm_large": 2, "batched": 1000, "serving": 4}
