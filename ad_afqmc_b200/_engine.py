"""Device buffers behind the reference-facing classes.

An ``Engine`` owns the prepared Hamiltonian layout and the workspace for one
(shape, walker type, precision) combination; it is cached inside the
``ham_data`` dict under a private key, next to the tensors it was built
from.  Rebuilding intermediates (``hamiltonian.build_*``) drops the cache.
"""

from __future__ import annotations

import ctypes as C
import warnings
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import AfqError

CACHE_KEY = "_afq_engines"

# precision switch of the walker path (see include/afqmc_b200.h)
PRECISIONS = {"fp64": 0, "mixed": 1, "mixed_hi": 2}

_small_work: Dict[Tuple, torch.Tensor] = {}


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise AfqError("no CUDA device: the walker path runs only on the GPU")
    return torch.device("cuda", torch.cuda.current_device())


def to_dev(x, dtype=torch.float64) -> torch.Tensor:
    """Contiguous CUDA tensor of `dtype` (copies host arrays once)."""
    if isinstance(x, torch.Tensor):
        t = x
        if t.dtype != dtype:
            t = t.to(dtype)
        if not t.is_cuda:
            t = t.to(device())
        return t.contiguous()
    if isinstance(x, np.ndarray) and not x.flags.writeable:
        # a shared read-only host array: wrap without copying, then one host-to-device copy
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", UserWarning)
            t = torch.from_numpy(np.ascontiguousarray(x))
        # asynchronous from page-locked memory (the owner keeps it alive and unchanged)
        return t.to(device=device(), dtype=dtype, non_blocking=t.is_pinned()).contiguous()
    return torch.as_tensor(x, dtype=dtype, device=device()).contiguous()


def small_work(W: int) -> torch.Tensor:
    dev = device()
    key = (dev.index, W)
    t = _small_work.get(key)
    if t is None:
        t = torch.empty(W * 16, dtype=torch.float64, device=dev)
        _small_work[key] = t
    return t


def dims_for(trial, walker_type: str, nwalkers: int, nchol: int = 1, precision: str = "fp64",
             dt: float = 0.01, n_exp_terms: int = 6) -> _lib.afq_dims:
    from .wavefunctions import uhf

    wt = _lib.AFQ_RESTRICTED if walker_type == "restricted" else _lib.AFQ_UNRESTRICTED
    tt = _lib.AFQ_TRIAL_UHF if isinstance(trial, uhf) else _lib.AFQ_TRIAL_RHF
    pr = PRECISIONS[precision]
    return _lib.make_dims(trial.norb, trial.nelec, nchol, nwalkers, wt, tt, n_exp_terms, pr, dt)


class Engine:
    """Prepared Hamiltonian + workspace for one problem shape."""

    def __init__(self, dims: _lib.afq_dims, ham_data: dict, trial, wave_data: dict):
        self.dims = dims
        pbytes, wbytes = _lib.sizes(dims)
        dev = device()
        self.prepared = torch.empty(pbytes // 8, dtype=torch.float64, device=dev)
        # zero-filled once: holds the device error flag of the tensor-core kernels
        self.work = torch.zeros(wbytes // 8, dtype=torch.float64, device=dev)
        self.work_bytes = wbytes
        self.block_out = torch.zeros(2, dtype=torch.float64, device=dev)
        self._keep = []
        self._prepare(ham_data, trial, wave_data)

    def _prepare(self, ham_data: dict, trial, wave_data: dict):
        from .wavefunctions import uhf

        h = _lib.afq_ham()
        keep = self._keep
        mos = trial._mo_list(wave_data)
        if "rot_chol" not in ham_data or "rot_h1" not in ham_data:
            raise AfqError("measurement intermediates missing: call build_measurement_intermediates")
        rh1 = ham_data["rot_h1"]
        rc = ham_data["rot_chol"]
        if isinstance(trial, uhf):
            rh1 = [to_dev(rh1[0]), to_dev(rh1[1])]
            rc = [to_dev(rc[0]), to_dev(rc[1])]
        else:
            rh1 = [to_dev(rh1)]
            rc = [to_dev(rc)]
        keep += mos + rh1 + rc
        for s in range(len(rc)):
            h.mo[s] = mos[s].data_ptr()
            h.rot_h1[s] = rh1[s].data_ptr()
            h.rot_chol[s] = rc[s].data_ptr()
        chol = to_dev(ham_data["chol"])
        keep.append(chol)
        h.chol = chol.data_ptr()
        if "exp_h1" in ham_data:
            e = to_dev(ham_data["exp_h1"])
            if e.dim() == 2:
                e = e.unsqueeze(0)
            keep.append(e)
            for s in range(e.shape[0]):
                h.exp_h1[s] = e[s].data_ptr()
        if "mf_shifts" in ham_data:
            mf = to_dev(ham_data["mf_shifts"], torch.complex128)
            keep.append(mf)
            h.mf_shifts = mf.data_ptr()
        h.h0 = float(ham_data["h0"])
        if "h0_prop" in ham_data:
            hp = complex(torch.as_tensor(ham_data["h0_prop"]).item()) if isinstance(
                ham_data["h0_prop"], torch.Tensor) else complex(ham_data["h0_prop"])
            h.h0_prop[0] = hp.real
            h.h0_prop[1] = hp.imag
        self.has_prop = "exp_h1" in ham_data and "mf_shifts" in ham_data
        _lib.check(
            _lib.lib().afq_prepare(C.byref(self.dims), C.byref(h), self.prepared.data_ptr(),
                                   self.prepared.numel() * 8, _lib.stream_handle()),
            "afq_prepare",
        )
        # the prepared buffer holds copies; the sources can be released after the stream drains
        torch.cuda.current_stream().synchronize()
        self._keep = []

    def ensure_workspace(self) -> None:
        """Grow the workspace if the shape's tuning record now needs more (the
        buffers that persist across calls keep their offsets, so a grown
        workspace only needs the zeroed error flag, which a fresh buffer has).
        Call it before capturing graphs that use this engine."""
        _, wbytes = _lib.sizes(self.dims)
        if wbytes > self.work.numel() * 8:
            new = torch.zeros(wbytes // 8, dtype=torch.float64, device=self.work.device)
            new[: self.work.numel()].copy_(self.work)
            self.work = new
        self.work_bytes = self.work.numel() * 8

    def check_status(self) -> None:
        """Raise AfqError if a bounded device-side wait of the tensor-core
        kernels ran out on this workspace since the last check (the flag is
        read and cleared by afq_check_status, which synchronizes the stream)."""
        _lib.check(_lib.lib().afq_check_status(C.byref(self.dims), self.work.data_ptr(), self.work_bytes,
                                               _lib.stream_handle()), "device status")

    def status_flag(self) -> torch.Tensor:
        """(1,) int32 view of this workspace's device error flag (0 = clear),
        for code that copies it out inside a CUDA graph (afq_status_flag).
        The view follows the current workspace: take it again after
        ensure_workspace."""
        p = C.c_void_p()
        _lib.check(_lib.lib().afq_status_flag(C.byref(self.dims), self.work.data_ptr(), self.work_bytes,
                                              C.byref(p)), "afq_status_flag")
        off = (int(p.value) - self.work.data_ptr()) // 4
        return self.work.view(torch.int32)[off:off + 1]

    @property
    def handle(self) -> Tuple[int, int, int]:
        return self.prepared.data_ptr(), self.work.data_ptr(), self.work_bytes


def get_engine(ham_data: dict, trial, wave_data: dict, walker_type: str, nwalkers: int,
               precision: str = "fp64", dt: float = 0.01, n_exp_terms: int = 6) -> Engine:
    cache = ham_data.setdefault(CACHE_KEY, {})
    nchol = int(ham_data["chol"].shape[0])
    key = (walker_type, int(nwalkers), precision, float(dt), int(n_exp_terms), "exp_h1" in ham_data,
           id(wave_data))
    eng = cache.get(key)
    if eng is None:
        d = dims_for(trial, walker_type, nwalkers, nchol, precision, dt, n_exp_terms)
        eng = Engine(d, ham_data, trial, wave_data)
        cache[key] = eng
    return eng


def drop_engines(ham_data: dict) -> None:
    ham_data.pop(CACHE_KEY, None)
