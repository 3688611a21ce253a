"""Seeded synthetic molecular Hamiltonians for the benchmark shapes.

No public molecular data set travels with this package, so the benchmark and
parity workloads use Hamiltonians built from a fixed recipe:

* each Cholesky vector ``L_g`` is a symmetric N x N matrix whose upper
  triangle is N(0, 1), mirrored, then scaled by ``exp(-g / N) / sqrt(N)``;
* ``h1`` is symmetric N(0, 0.1^2) plus ``diag(linspace(-3, 1, N))``;
* the RHF trial is the lowest ``No`` eigenvectors of ``h1``; the UHF trial
  uses ``h1 +/- 0.05 R`` with R a random symmetric matrix;
* ``h0 = ene0 = 0``.

With N = 200 the scale factor is ``exp(-g/200)/sqrt(200)``.  Everything is
drawn from ``numpy.random.default_rng(seed)`` in a fixed order, so a seed
names one Hamiltonian exactly.  Construction happens once per solve on the
host; the walker path itself never touches these NumPy arrays.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Tuple

import numpy as np


@dataclass
class SyntheticSystem:
    norb: int
    nelec: Tuple[int, int]
    nchol: int
    h1: np.ndarray          # (2, N, N) float64
    chol: np.ndarray        # (G, N*N) float64
    h0: float
    mo_coeff: object        # (N, Na) for RHF, [(N, Na), (N, Nb)] for UHF
    trial: str              # "rhf" or "uhf"

    def ham_data(self) -> Dict:
        # chol is shared read-only (nothing writes it; copying it cost more than the solve setup)
        chol = self.chol.view()
        chol.flags.writeable = False
        return {"h0": self.h0, "h1": self.h1.copy(), "chol": chol, "ene0": 0.0}

    def pin(self) -> "SyntheticSystem":
        """Move chol into page-locked host memory (a torch pinned buffer that
        this object keeps alive), so its host-to-device copy runs at full PCIe
        bandwidth and asynchronously on the copying stream."""
        import torch

        buf = torch.empty(self.chol.shape, dtype=torch.float64, pin_memory=True)
        buf.numpy()[...] = self.chol
        self._pinned = buf
        self.chol = buf.numpy()
        return self

    def wave_data(self) -> Dict:
        if self.trial == "rhf":
            mo = self.mo_coeff
            return {"mo_coeff": mo.copy(), "rdm1": np.array([mo @ mo.T] * 2)}
        mo = [m.copy() for m in self.mo_coeff]
        return {"mo_coeff": mo, "rdm1": np.array([mo[0] @ mo[0].T, mo[1] @ mo[1].T])}


def _sym_normal(rng, n):
    a = rng.standard_normal((n, n))
    up = np.triu(a)
    return up + np.triu(up, 1).T


def make_system(norb: int, nelec: Tuple[int, int], nchol: int, seed: int,
                trial: str = "rhf", chol_scale: float = 1.0) -> SyntheticSystem:
    """``chol_scale`` multiplies every Cholesky vector.  With the prescribed
    scale (1.0) at N=200 the one-step propagator is far from identity
    (||VHS|| ~ 1.4) and the phaseless clamps kill the whole population within
    a few steps; 0.25 gives a same-shape system whose population survives,
    used where block energies must be meaningful (precision comparisons)."""
    rng = np.random.default_rng(seed)
    n = norb
    chol = np.empty((nchol, n * n))
    for g in range(nchol):
        chol[g] = (_sym_normal(rng, n) * (chol_scale * np.exp(-g / n) / np.sqrt(n))).reshape(-1)
    h1 = 0.1 * _sym_normal(rng, n)
    h1 = (h1 + h1.T) / 2.0 + np.diag(np.linspace(-3.0, 1.0, n))
    h1 = np.array([h1, h1])
    if trial == "rhf":
        assert nelec[0] == nelec[1]
        _, v = np.linalg.eigh(h1[0])
        mo = v[:, : nelec[0]].copy()
    else:
        r = _sym_normal(rng, n)
        r = (r + r.T) / 2.0
        _, va = np.linalg.eigh(h1[0] + 0.05 * r)
        _, vb = np.linalg.eigh(h1[1] - 0.05 * r)
        mo = [va[:, : nelec[0]].copy(), vb[:, : nelec[1]].copy()]
    return SyntheticSystem(n, tuple(nelec), nchol, h1, chol, 0.0, mo, trial)


# Named workloads (sizes of the benchmark configurations).
CONFIGS = {
    # stand-in for H10 / STO-6G: Norb=10, 5a/5b, ~50 Cholesky vectors
    "h10_sto6g_synthetic": dict(norb=10, nelec=(5, 5), nchol=50, seed=1001, trial="rhf",
                                n_walkers=100, dt=0.005, n_prop_steps=10, n_blocks=20),
    "rhf_n200_g1000": dict(norb=200, nelec=(40, 40), nchol=1000, seed=1002, trial="rhf",
                           n_walkers=512, dt=0.005, n_prop_steps=10, n_blocks=20),
    "uhf_n300_g1500": dict(norb=300, nelec=(60, 58), nchol=1500, seed=1003, trial="uhf",
                           n_walkers=1024, dt=0.005, n_prop_steps=10, n_blocks=20),
}


def make_config(name: str, chol_scale: float = 1.0) -> Tuple[SyntheticSystem, dict]:
    c = dict(CONFIGS[name])
    sys_ = make_system(c.pop("norb"), c.pop("nelec"), c.pop("nchol"), c.pop("seed"), c.pop("trial"),
                       chol_scale=chol_scale)
    return sys_, c


def fragment_chol_scale(norb: int) -> float:
    """Two-body scale of a served fragment: 0.035 * sqrt(100 / N).  The block
    energy variance of these synthetic systems grows steeply with N and with
    the Cholesky scale; this scale puts the 0.5 mHa standard error within tens
    of blocks at every fragment size (about 0.1-0.2 mHa after 40 blocks at
    N = 40 ... 250).  The arithmetic per block does not depend on it."""
    return 0.035 * float(np.sqrt(100.0 / norb))


def make_fragment_batch(n_fragments: int = 64, seed: int = 1004, large_frac: float = 0.0):
    """Uneven fragment shapes: N ~ U[30,160], No = round(N/4), G ~ U[4N, 6N],
    W ~ U[64, 256]; with ``large_frac`` of them at N=250, G=1250."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_fragments):
        if large_frac > 0 and rng.random() < large_frac:
            n, g = 250, 1250
        else:
            n = int(rng.integers(30, 161))
            g = int(rng.integers(4 * n, 6 * n + 1))
        no = int(round(n / 4))
        w = int(rng.integers(64, 257))
        out.append(dict(norb=n, nelec=(no, no), nchol=g, n_walkers=w, seed=int(seed * 1000 + i)))
    return out
