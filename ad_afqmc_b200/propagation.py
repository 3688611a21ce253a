"""Phaseless propagator on the device (mirror of ad_afqmc/propagation.py).

``propagator_afqmc`` keeps the reference's fields (propagation.py:111-121),
``prop_data`` keys and method signatures: ``init_prop_data`` (:123-152),
``propagate_constrained`` (:274-336) and
``_build_propagation_intermediates`` (:378-438).  One call of
``propagate_constrained`` is one C-ABI call (``afq_propagate_constrained``)
that runs force bias, VHS, the Taylor propagator, overlaps and the weight
update on the GPU.  Device-resident scalars (``e_estimate``,
``pop_control_ene_shift``, the killed-walker count) live in
``prop_data["_scalars"]`` so the step needs no host round trip.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np
import torch

from . import _lib
from ._engine import device, drop_engines, get_engine, to_dev
from .walkers import RHFWalkers, UHFWalkers


class PRNGKey:
    """Counter-based key replacing ``jax.random.PRNGKey`` (propagation.py:134).

    ``seed`` selects the Philox stream; ``counter`` advances with every draw,
    which plays the role of ``random.split``."""

    def __init__(self, seed: int, counter: int = 0):
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.counter = int(counter)

    def take(self, n_pairs: int) -> int:
        c = self.counter
        self.counter += int(n_pairs)
        return c

    def uniform(self) -> float:
        """One U(0,1) draw for reconfiguration (replaces random.uniform(subkey))."""
        c = self.take(1)
        return float(np.random.default_rng([self.seed, c, 0x5A5A]).random())

    def __repr__(self):
        return f"PRNGKey(seed={self.seed}, counter={self.counter})"


def normal_fields(key: PRNGKey, shape, dev=None) -> torch.Tensor:
    """Standard-normal float64 fields drawn on the device (afq_normal_fields)."""
    n = int(np.prod(shape))
    out = torch.empty(n, dtype=torch.float64, device=dev or device())
    off = key.take((n + 1) // 2)
    _lib.check(_lib.lib().afq_normal_fields(out.data_ptr(), n, key.seed, off, _lib.stream_handle()),
               "afq_normal_fields")
    return out.reshape(shape)


def _scalar(v) -> torch.Tensor:
    return to_dev(torch.as_tensor(v, dtype=torch.float64).reshape(()))


def sync_scalars(prop_data: dict) -> torch.Tensor:
    """Bind e_estimate / pop_control_ene_shift / n_killed_walkers to the device scalars."""
    sc = prop_data.get("_scalars")
    if sc is None:
        sc = torch.zeros(8, dtype=torch.float64, device=device())
        prop_data["_scalars"] = sc
    for i, k in enumerate(("e_estimate", "pop_control_ene_shift", "n_killed_walkers")):
        if k not in prop_data:
            continue
        v = prop_data[k]
        view = sc[i]
        if isinstance(v, torch.Tensor) and v.is_cuda and v.data_ptr() == view.data_ptr():
            continue
        view.copy_(_scalar(v))
        prop_data[k] = view
    for i, k in enumerate(("e_estimate", "pop_control_ene_shift", "n_killed_walkers")):
        prop_data[k] = sc[i]
    return sc


def _walker_key(prop_data: dict, eng) -> tuple:
    w = prop_data["walkers"]
    ptrs = tuple(t.data_ptr() for t in (w.data if isinstance(w, UHFWalkers) else [w.data]))
    return (id(eng), id(w)) + ptrs


def make_state(prop_data: dict, eng=None) -> _lib.afq_state:
    """C-ABI state of prop_data.  The GREEN_CURRENT flag is set only when the
    engine's workspace holds the Green's function of exactly these walker
    tensors (left by the previous step); any new walker object clears it."""
    st = _lib.afq_state()
    w = prop_data["walkers"]
    if isinstance(w, UHFWalkers):
        st.walkers[0] = w.data[0].data_ptr()
        st.walkers[1] = w.data[1].data_ptr()
    else:
        st.walkers[0] = w.data.data_ptr()
        st.walkers[1] = None
    st.weights = prop_data["weights"].data_ptr()
    st.overlaps = prop_data["overlaps"].data_ptr()
    st.scalars = prop_data["_scalars"].data_ptr()
    st.flags = 0
    if eng is not None and prop_data.get("_afq_green_of") == _walker_key(prop_data, eng):
        st.flags = _lib.AFQ_STATE_GREEN_CURRENT
    return st


def note_state(prop_data: dict, st: _lib.afq_state, eng) -> None:
    """Record, after a C call, whether the workspace holds these walkers' G."""
    if st.flags & _lib.AFQ_STATE_GREEN_CURRENT:
        prop_data["_afq_green_of"] = _walker_key(prop_data, eng)
    else:
        prop_data.pop("_afq_green_of", None)


@dataclass
class propagator:
    dt: float = 0.01
    n_walkers: int = 50


@dataclass
class propagator_afqmc(propagator):
    """Propagator for phaseless AFQMC (propagation.py:111-441)."""

    dt: float = 0.01
    n_walkers: int = 50
    n_exp_terms: int = 6
    n_chunks: int = 1
    vhs_real_dtype: Any = None
    vhs_complex_dtype: Any = None
    walker_type: str = "restricted"
    precision: str = "fp64"

    def engine(self, ham_data: dict, trial, wave_data: dict):
        return get_engine(ham_data, trial, wave_data, self.walker_type, self.n_walkers, self.precision,
                          self.dt, self.n_exp_terms)

    def init_prop_data(self, trial, wave_data: dict, ham_data: dict, seed: int,
                       init_walkers=None) -> dict:
        """propagation.py:123-152."""
        dev = device()
        pd = {}
        pd["weights"] = torch.ones(self.n_walkers, dtype=torch.float64, device=dev)
        pd["key"] = PRNGKey(seed)
        if init_walkers is not None:
            if isinstance(init_walkers, (RHFWalkers, UHFWalkers)):
                pd["walkers"] = init_walkers
            elif isinstance(init_walkers, (list, tuple)):
                pd["walkers"] = UHFWalkers(list(init_walkers))
            else:
                pd["walkers"] = RHFWalkers(init_walkers)
        else:
            pd["walkers"] = trial.get_init_walkers(wave_data, self.n_walkers, self.walker_type)
        if "e_estimate" in ham_data:
            pd["e_estimate"] = _scalar(ham_data["e_estimate"])
        else:
            if self.precision != "fp64" and "exp_h1" in ham_data:
                # the propagator's own engine: no FP64 layout built for one energy evaluation
                e = torch.real(trial.calc_energy(pd["walkers"], ham_data, wave_data,
                                                 engine=self.engine(ham_data, trial, wave_data)))
            else:
                e = torch.real(trial.calc_energy(pd["walkers"], ham_data, wave_data))
            pd["e_estimate"] = torch.sum(e) / self.n_walkers
        pd["pop_control_ene_shift"] = pd["e_estimate"].clone()
        pd["n_killed_walkers"] = 0.0
        sync_scalars(pd)
        pd["overlaps"] = trial.calc_overlap(pd["walkers"], wave_data)
        pd["normed_overlaps"] = pd["overlaps"]
        pd["norms"] = torch.ones(self.n_walkers, dtype=torch.complex128, device=dev)
        return pd

    def propagate_constrained(self, trial, ham_data: dict, prop_data: dict, fields,
                              wave_data: dict) -> dict:
        """One phaseless step (propagation.py:274-336), in place on the device."""
        eng = self.engine(ham_data, trial, wave_data)
        if not eng.has_prop:
            raise _lib.AfqError("propagation intermediates missing: call build_propagation_intermediates")
        sync_scalars(prop_data)
        f = to_dev(fields, torch.float64)
        if f.shape != (self.n_walkers, int(ham_data["chol"].shape[0])):
            raise ValueError(f"fields must be (n_walkers, nchol), got {tuple(f.shape)}")
        st = make_state(prop_data, eng)
        p, w, wb = eng.handle
        _lib.check(
            _lib.lib().afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st), f.data_ptr(), w, wb,
                                                 _lib.stream_handle()),
            "afq_propagate_constrained",
        )
        note_state(prop_data, st, eng)
        return prop_data

    def propagate_free(self, trial, ham_data: dict, prop_data: dict, fields, wave_data: dict) -> dict:
        """Free propagation, propagation.py:338-376: the Trotterized propagator
        with the raw fields (afq_apply_trotprop), the mean-field constants
        exp(-sqrt(dt) x.mf_shifts_fp) exp(dt h0_prop_fp), orthogonalization
        with the norms into the weights, a local comb and the new overlaps."""
        if self.walker_type not in ("restricted", "unrestricted"):
            raise AssertionError("Free propagation is only implemented for restricted and unrestricted walkers.")
        eng = self.engine(ham_data, trial, wave_data)
        if not eng.has_prop:
            raise _lib.AfqError("propagation intermediates missing: call build_propagation_intermediates")
        f = to_dev(fields, torch.float64)
        if f.shape != (self.n_walkers, int(ham_data["chol"].shape[0])):
            raise ValueError(f"fields must be (n_walkers, nchol), got {tuple(f.shape)}")
        sdt = self.dt ** 0.5
        mf = to_dev(ham_data["mf_shifts_fp"], torch.complex128)
        h0p = to_dev(torch.as_tensor(ham_data["h0_prop_fp"]), torch.complex128)
        fc = f.to(torch.complex128)
        if self.walker_type == "unrestricted":
            constants = torch.exp(-sdt * (mf @ fc.T)) * torch.exp(self.dt * h0p).reshape(-1, 1)
        else:
            constants = torch.exp(-sdt * (fc @ mf)) * torch.exp(self.dt * h0p)
        walkers = prop_data["walkers"]
        data = [t.clone() for t in (walkers.data if isinstance(walkers, UHFWalkers) else [walkers.data])]
        ptrs = _lib.pair(data[0].data_ptr(), data[-1].data_ptr() if len(data) > 1 else None)
        p, w, wb = eng.handle
        _lib.check(_lib.lib().afq_apply_trotprop(C.byref(eng.dims), p, ptrs, f.data_ptr(), w, wb,
                                                 _lib.stream_handle()), "afq_apply_trotprop")
        walkers = UHFWalkers(data) if isinstance(walkers, UHFWalkers) else RHFWalkers(data[0])
        walkers = walkers.multiply_constants(constants)
        walkers, norms = walkers.orthogonalize()
        prop_data["weights"] = prop_data["weights"] * torch.real(norms)
        zeta = prop_data["key"].uniform() if getattr(self, "_zeta_source", None) is None else \
            float(self._zeta_source.uniform())
        prop_data["walkers"], prop_data["weights"] = walkers.stochastic_reconfiguration_local(
            prop_data["weights"], zeta)
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        prop_data.pop("_afq_green_of", None)
        return prop_data

    def _build_propagation_intermediates(self, ham_data: dict, trial, wave_data: dict) -> dict:
        """mf_shifts, h0_prop, *_fp, exp_h1 (propagation.py:378-438), by
        afq_propagation_intermediates (v0 and the exponentials on the FP64
        tensor cores)."""
        from . import intermediates

        ham_data["chol"] = to_dev(ham_data["chol"])
        ham_data["h1"] = to_dev(ham_data["h1"])
        unrestricted = self.walker_type == "unrestricted"
        mf, h0_prop, exp_h1 = intermediates.propagation(trial.norb, ham_data["h1"], wave_data["rdm1"],
                                                        ham_data["chol"], float(ham_data["h0"]), self.dt,
                                                        unrestricted)
        ham_data["mf_shifts"] = mf
        ham_data["h0_prop"] = h0_prop
        na, nb = trial.nelec
        ene0 = float(ham_data.get("ene0", 0.0))
        if unrestricted:
            ham_data["mf_shifts_fp"] = torch.stack((mf / na / 2.0, mf / nb / 2.0))
            ham_data["h0_prop_fp"] = torch.stack(((h0_prop + ene0) / na / 2.0, (h0_prop + ene0) / nb / 2.0))
        else:
            ham_data["mf_shifts_fp"] = mf / 2.0 / na
            ham_data["h0_prop_fp"] = (h0_prop + ene0) / na / 2.0
        ham_data["exp_h1"] = exp_h1
        drop_engines(ham_data)
        return ham_data

    def __hash__(self) -> int:
        return hash(tuple(str(v) for v in self.__dict__.values()))
