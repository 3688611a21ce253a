"""Walker batches on the device (mirror of ad_afqmc/walkers.py).

``RHFWalkers.data`` is a (W, N, No) complex128 CUDA tensor and
``UHFWalkers.data`` a list of (W, N, Na) and (W, N, Nb) tensors, the layouts
of walkers.py:85-284.  The reference's ``apply_chunked`` memory chunking
(walkers.py:95-137) is replaced by the kernels' own tiling and is not needed
by callers; QR and reconfiguration run in libafqmc_b200.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, List, Tuple, Union

import numpy as np
import torch

from . import _lib
from ._engine import small_work, to_dev


def _dims(norb, nocc, W, walker_type):
    wt = _lib.AFQ_RESTRICTED if walker_type == "restricted" else _lib.AFQ_UNRESTRICTED
    # trial type does not matter for QR / reconfiguration; rhf needs Na == Nb
    tt = _lib.AFQ_TRIAL_RHF if walker_type == "restricted" or nocc[0] == nocc[1] else _lib.AFQ_TRIAL_UHF
    return _lib.make_dims(norb, nocc, 1, W, wt, tt, 6, _lib.AFQ_FP64, 0.01)


def _as_weights(weights) -> torch.Tensor:
    return to_dev(weights, torch.float64)


def _multi_rank(comm) -> bool:
    """True for a torch.distributed group of more than one rank.  An MPI-style
    communicator (Get_size) of one rank keeps the single-rank path; the
    reconfiguration across ranks runs on torch.distributed groups."""
    if comm is None:
        return False
    if hasattr(comm, "Get_size"):
        if comm.Get_size() == 1:
            return False
        raise ValueError("reconfiguration across ranks takes a torch.distributed process group "
                         "(one rank per GPU), not an MPI communicator")
    import torch.distributed as dist

    return dist.is_initialized() and dist.get_world_size(comm) > 1


class walker_batch:
    """Common interface (walkers.py:11-82)."""

    def _sr(self, tensors: List[torch.Tensor], weights, zeta, mode, walker_type):
        W = tensors[0].shape[0]
        N = tensors[0].shape[1]
        nocc = (tensors[0].shape[2], tensors[-1].shape[2])
        d = _dims(N, nocc, W, walker_type)
        w_in = _as_weights(weights)
        w_out = torch.empty_like(w_in)
        idx = torch.empty(W, dtype=torch.int32, device=w_in.device)
        outs = [torch.empty_like(t) for t in tensors]
        ins = _lib.pair(tensors[0].data_ptr(), tensors[-1].data_ptr() if len(tensors) > 1 else None)
        ous = _lib.pair(outs[0].data_ptr(), outs[-1].data_ptr() if len(outs) > 1 else None)
        z = float(torch.as_tensor(zeta).item()) if isinstance(zeta, torch.Tensor) else float(zeta)
        _lib.check(
            _lib.lib().afq_stochastic_reconfiguration(
                C.byref(d), w_in.data_ptr(), z, mode, ins, ous, w_out.data_ptr(), idx.data_ptr(),
                _lib.stream_handle()),
            "afq_stochastic_reconfiguration",
        )
        return outs, w_out, idx

    def _qr(self, tensors: List[torch.Tensor], walker_type, want_norms: bool):
        W, N = tensors[0].shape[0], tensors[0].shape[1]
        nocc = (tensors[0].shape[2], tensors[-1].shape[2])
        d = _dims(N, nocc, W, walker_type)
        out = [t.clone() for t in tensors]
        norms = torch.empty(W, dtype=torch.complex128, device=out[0].device) if want_norms else None
        work = small_work(W)
        _lib.check(
            _lib.lib().afq_orthonormalize(
                C.byref(d),
                _lib.pair(out[0].data_ptr(), out[-1].data_ptr() if len(out) > 1 else None),
                norms.data_ptr() if norms is not None else None,
                work.data_ptr(), work.numel() * 8, _lib.stream_handle()),
            "afq_orthonormalize",
        )
        return out, norms


@dataclass
class RHFWalkers(walker_batch):
    """Restricted walkers, data (W, N, No) complex128 (walkers.py:85-177)."""

    data: Any

    def __post_init__(self):
        self.data = to_dev(self.data, torch.complex128)

    @property
    def n_walkers(self) -> int:
        return self.data.shape[0]

    def stochastic_reconfiguration_local(self, weights, zeta) -> Tuple["RHFWalkers", torch.Tensor]:
        """walkers.py:139-145 -> sr.py:24-34."""
        outs, w, _ = self._sr([self.data], weights, zeta, _lib.AFQ_SR_LOCAL, "restricted")
        return self.__class__(outs[0]), w

    def stochastic_reconfiguration_global(self, weights, zeta, comm=None):
        """walkers.py:147-153 -> sr.py:52-92.  ``comm``: a torch.distributed
        process group (one rank per GPU; the same zeta on every rank) for the
        reconfiguration across ranks (sr_ranks.py), None for one rank."""
        if _multi_rank(comm):
            from .sr_ranks import reconfigure_across_ranks

            outs, w = reconfigure_across_ranks([self.data], to_dev(weights), float(zeta), comm)
            return self.__class__(outs[0]), w
        outs, w, _ = self._sr([self.data], weights, zeta, _lib.AFQ_SR_GLOBAL, "restricted")
        return self.__class__(outs[0]), w

    def orthonormalize(self) -> "RHFWalkers":
        """walkers.py:155-157 -> linalg_utils.qr_vmap_restricted."""
        out, _ = self._qr([self.data], "restricted", False)
        return self.__class__(out[0])

    def orthogonalize(self) -> Tuple["RHFWalkers", torch.Tensor]:
        """walkers.py:159-162: QR and norms**2."""
        out, norms = self._qr([self.data], "restricted", True)
        return self.__class__(out[0]), norms**2

    def multiply_constants(self, constants) -> "RHFWalkers":
        """walkers.py:164-167."""
        c = to_dev(constants, torch.complex128).reshape(-1, 1, 1)
        return self.__class__(self.data * c)


@dataclass
class UHFWalkers(walker_batch):
    """Unrestricted walkers, data [(W, N, Na), (W, N, Nb)] complex128 (walkers.py:180-284)."""

    data: List[Any]

    def __post_init__(self):
        self.data = [to_dev(self.data[0], torch.complex128), to_dev(self.data[1], torch.complex128)]

    @property
    def n_walkers(self) -> int:
        return self.data[0].shape[0]

    def stochastic_reconfiguration_local(self, weights, zeta):
        """walkers.py:244-250 -> sr.py:37-48."""
        outs, w, _ = self._sr(self.data, weights, zeta, _lib.AFQ_SR_LOCAL, "unrestricted")
        return self.__class__(outs), w

    def stochastic_reconfiguration_global(self, weights, zeta, comm=None):
        """walkers.py:252-258 -> sr.py:95-153; ``comm`` as for RHFWalkers."""
        if _multi_rank(comm):
            from .sr_ranks import reconfigure_across_ranks

            outs, w = reconfigure_across_ranks(list(self.data), to_dev(weights), float(zeta), comm)
            return self.__class__(outs), w
        outs, w, _ = self._sr(self.data, weights, zeta, _lib.AFQ_SR_GLOBAL, "unrestricted")
        return self.__class__(outs), w

    def orthonormalize(self) -> "UHFWalkers":
        """walkers.py:260-262 -> linalg_utils.qr_vmap_unrestricted (sign-fixed column 0)."""
        out, _ = self._qr(self.data, "unrestricted", False)
        return self.__class__(out)

    def orthogonalize(self):
        """walkers.py:264-267: QR and |prod diag R_up| |prod diag R_dn|."""
        out, norms = self._qr(self.data, "unrestricted", True)
        return self.__class__(out), norms

    def multiply_constants(self, constants) -> "UHFWalkers":
        """walkers.py:269-275."""
        c0 = to_dev(constants[0], torch.complex128).reshape(-1, 1, 1)
        c1 = to_dev(constants[1], torch.complex128).reshape(-1, 1, 1)
        return self.__class__([self.data[0] * c0, self.data[1] * c1])


def walker_tensors(walkers) -> List[torch.Tensor]:
    if isinstance(walkers, UHFWalkers):
        return walkers.data
    if isinstance(walkers, RHFWalkers):
        return [walkers.data]
    raise TypeError(f"unsupported walker type {type(walkers)}")
