"""Per-solve Hamiltonian intermediates on this library's kernels.

The set-up half of a solve — symmetrized h1, the half-rotated integrals
``rot_h1`` / ``rot_chol`` (wavefunctions.py:1215-1232, 1472-1496), the
mean-field shifts, ``h0_prop``, ``v0``, ``v1`` and ``exp_h1``
(propagation.py:378-438), and the natural orbitals of the initial walkers
(wavefunctions.py:427-466) — as calls into libafqmc_b200 (FP64 DMMA GEMMs,
Taylor scaling and squaring, a Jacobi eigensolver).  Every call runs on the
current torch stream; the scratch comes from torch's caching allocator.
"""

from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import torch

from . import _lib
from ._engine import to_dev


def workspace(norb: int, nchol: int, dev) -> torch.Tensor:
    n = C.c_size_t()
    _lib.check(_lib.lib().afq_intermediates_workspace_size(int(norb), int(nchol), C.byref(n)),
               "afq_intermediates_workspace_size")
    return torch.empty((n.value + 7) // 8, dtype=torch.float64, device=dev)


def measurement(norb: int, nelec: Tuple[int, int], h1, chol, mos: Sequence[torch.Tensor],
                uhf: bool) -> Tuple[torch.Tensor, List[torch.Tensor], List[torch.Tensor]]:
    """Symmetrized h1 (2, N, N), rot_h1 per sector and rot_chol per sector
    (one sector for an RHF trial, two for UHF)."""
    h1 = to_dev(h1).clone().contiguous()
    chol = to_dev(chol)
    dev = h1.device
    G = int(chol.shape[0])
    ns = 2 if uhf else 1
    nocc = (C.c_int32 * 2)(int(nelec[0]), int(nelec[1]))
    rh1 = [torch.empty(int(nelec[s]), norb, dtype=torch.float64, device=dev) for s in range(ns)]
    rc = [torch.empty(G, int(nelec[s]), norb, dtype=torch.float64, device=dev) for s in range(ns)]
    mo = [m.contiguous() for m in mos]
    work = workspace(norb, G, dev)
    _lib.check(_lib.lib().afq_measurement_intermediates(
        int(norb), nocc, G, _lib.AFQ_TRIAL_UHF if uhf else _lib.AFQ_TRIAL_RHF,
        _lib.pair(mo[0].data_ptr(), mo[-1].data_ptr()), h1.data_ptr(), chol.data_ptr(),
        _lib.pair(rh1[0].data_ptr(), rh1[-1].data_ptr()), _lib.pair(rc[0].data_ptr(), rc[-1].data_ptr()),
        work.data_ptr(), work.numel() * 8, _lib.stream_handle()), "afq_measurement_intermediates")
    return h1, rh1, rc


def propagation(norb: int, h1, rdm1, chol, h0: float, dt: float, unrestricted: bool):
    """(mf_shifts (G,) complex128, h0_prop 0-d complex128, exp_h1 (N, N) or (2, N, N))."""
    h1 = to_dev(h1).contiguous()
    rdm1 = to_dev(rdm1).contiguous()
    chol = to_dev(chol)
    dev = h1.device
    G = int(chol.shape[0])
    mf = torch.empty(G, dtype=torch.complex128, device=dev)
    h0p = torch.empty((), dtype=torch.complex128, device=dev)
    np_ = 2 if unrestricted else 1
    exp_h1 = torch.empty(np_, norb, norb, dtype=torch.float64, device=dev)
    work = workspace(norb, G, dev)
    _lib.check(_lib.lib().afq_propagation_intermediates(
        int(norb), G, _lib.AFQ_UNRESTRICTED if unrestricted else _lib.AFQ_RESTRICTED, h1.data_ptr(),
        rdm1.data_ptr(), chol.data_ptr(), float(h0), float(dt), mf.data_ptr(), h0p.data_ptr(),
        exp_h1.data_ptr(), work.data_ptr(), work.numel() * 8, _lib.stream_handle()),
        "afq_propagation_intermediates")
    return mf, h0p, (exp_h1 if unrestricted else exp_h1[0])


def expm(a: torch.Tensor, scale: float = 1.0) -> torch.Tensor:
    """expm(scale * a) for a real square matrix (afq_expm)."""
    a = to_dev(a).contiguous()
    n = int(a.shape[0])
    out = torch.empty_like(a)
    work = workspace(n, 1, a.device)  # covers the exponential's scratch
    _lib.check(_lib.lib().afq_expm(n, a.data_ptr(), float(scale), out.data_ptr(), work.data_ptr(),
                                   work.numel() * 8, _lib.stream_handle()), "afq_expm")
    return out


def eigh_desc(a: torch.Tensor, return_sweeps: bool = False):
    """(eigenvalues descending, eigenvectors as columns in that order); with
    ``return_sweeps`` also the number of Jacobi sweeps (synchronizes)."""
    a = to_dev(a).contiguous()
    n = int(a.shape[0])
    vals = torch.empty(n, dtype=torch.float64, device=a.device)
    vecs = torch.empty(n, n, dtype=torch.float64, device=a.device)
    work = torch.empty(2 * n * n + 16, dtype=torch.float64, device=a.device)
    _lib.check(_lib.lib().afq_eigh_desc(n, a.data_ptr(), vals.data_ptr(), vecs.data_ptr(), work.data_ptr(),
                                        work.numel() * 8, _lib.stream_handle()), "afq_eigh_desc")
    if return_sweeps:
        nn2 = 2 * ((n * n + 1) // 2 * 2)  # the sweep count follows the two (n x n) buffers
        return vals, vecs, int(work.view(torch.int32)[2 * nn2].item())
    return vals, vecs


def natural_orbitals(rdm: torch.Tensor, k: int, return_occ: bool = False):
    """The k natural orbitals of largest occupation, (N, k) float64
    (afq_natural_orbitals: subspace iteration with Rayleigh-Ritz, the full
    Jacobi eigensolver when the occupations at the cut are too close)."""
    rdm = to_dev(rdm).contiguous()
    n = int(rdm.shape[0])
    size = C.c_size_t()
    _lib.check(_lib.lib().afq_natural_orbitals_workspace_size(n, int(k), C.byref(size)),
               "afq_natural_orbitals_workspace_size")
    work = torch.empty((size.value + 7) // 8, dtype=torch.float64, device=rdm.device)
    orbs = torch.empty(n, int(k), dtype=torch.float64, device=rdm.device)
    occ = torch.empty(int(k), dtype=torch.float64, device=rdm.device)
    _lib.check(_lib.lib().afq_natural_orbitals(n, int(k), rdm.data_ptr(), orbs.data_ptr(), occ.data_ptr(),
                                               work.data_ptr(), work.numel() * 8, _lib.stream_handle()),
               "afq_natural_orbitals")
    return (orbs, occ) if return_occ else orbs
