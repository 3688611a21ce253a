"""Block / reconfiguration loop on the device (mirror of ad_afqmc/sampling.py).

``sampler.propagate_phaseless`` follows sampling.py:343-365 with the scans of
``_sr_block_scan`` (:146-168), ``_block_scan`` (:52-94) and ``_step_scan``
(:22-36) unrolled into C-ABI calls: one ``afq_propagate_constrained`` per
step and one ``afq_block_end`` (QR, overlaps, energies, clamp, block energy,
population shift) per energy block.  All state stays on the device; the
returned energy is a 0-d CUDA tensor.

Randomness: fields are drawn on the device from the counter-based key in
``prop_data["key"]``.  A ``field_source`` object (with ``fields(S, W, G)``
and ``uniform()``) replaces the device draws, which is how parity tests feed
the same random numbers to this path and to the oracle.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Optional

import torch

from . import _lib
from ._engine import device, to_dev
from .propagation import make_state, normal_fields, note_state, sync_scalars


@dataclass
class sampler:
    n_prop_steps: int = 50
    n_ene_blocks: int = 50
    n_sr_blocks: int = 1
    n_blocks: int = 50
    field_source: Any = None

    def _fields(self, prop, prop_data, nchol):
        shape = (self.n_prop_steps, prop.n_walkers, nchol)
        if self.field_source is not None:
            return to_dev(self.field_source.fields(*shape), torch.float64)
        return normal_fields(prop_data["key"], shape)

    def _uniform(self, prop_data) -> float:
        if self.field_source is not None:
            return float(self.field_source.uniform())
        return prop_data["key"].uniform()

    def _block_scan(self, prop, trial, ham_data, prop_data, wave_data, out_row):
        """sampling.py:52-94."""
        eng = prop.engine(ham_data, trial, wave_data)
        nchol = int(ham_data["chol"].shape[0])
        fields = self._fields(prop, prop_data, nchol)
        p, w, wb = eng.handle
        lib = _lib.lib()
        stream = _lib.stream_handle()
        st = make_state(prop_data, eng)
        for s in range(self.n_prop_steps):
            _lib.check(lib.afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st),
                                                     fields[s].data_ptr(), w, wb, stream),
                       "afq_propagate_constrained")
        _lib.check(lib.afq_block_end(C.byref(eng.dims), p, C.byref(st), out_row.data_ptr(), w, wb,
                                     stream), "afq_block_end")
        st.flags = 0  # QR changed the walkers in place
        note_state(prop_data, st, eng)

    def propagate_phaseless(self, ham, ham_data: dict, prop, prop_data: dict, trial, wave_data: dict):
        """sampling.py:343-365.  Returns (E, prop_data) with E a 0-d device tensor."""
        eng = prop.engine(ham_data, trial, wave_data)
        if not eng.has_prop:
            raise _lib.AfqError("propagation intermediates missing: call build_propagation_intermediates")
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        prop_data["n_killed_walkers"] = 0.0
        prop_data["pop_control_ene_shift"] = prop_data["e_estimate"]
        if isinstance(prop_data["pop_control_ene_shift"], torch.Tensor):
            prop_data["pop_control_ene_shift"] = prop_data["pop_control_ene_shift"].clone()
        sync_scalars(prop_data)
        nb = self.n_sr_blocks * self.n_ene_blocks
        out = torch.zeros(nb, 2, dtype=torch.float64, device=device())
        i = 0
        for _ in range(self.n_sr_blocks):
            for _ in range(self.n_ene_blocks):
                self._block_scan(prop, trial, ham_data, prop_data, wave_data, out[i])
                i += 1
            zeta = self._uniform(prop_data)
            prop_data["walkers"], prop_data["weights"] = prop_data[
                "walkers"].stochastic_reconfiguration_local(prop_data["weights"], zeta)
            prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        sc = prop_data["_scalars"]
        sc[2].div_(nb * prop.n_walkers)
        be, bw = out[:, 0], out[:, 1]
        prop_data["block_energies"] = out
        eng.check_status()  # a timed-out device wait invalidates these blocks
        return torch.sum(be * bw) / torch.sum(bw), prop_data

    def propagate_free(self, ham, ham_data: dict, prop, prop_data: dict, trial, wave_data: dict):
        """Free projection, sampling.py:367-384 over _block_scan_free (:96-144):
        n_blocks blocks of n_prop_steps free steps.  Returns (ov, abs_ov,
        prop_data_tr, block_energy, block_weight, key): per block the sum of
        overlaps and of their moduli, a copy of the walker state, the
        overlap-weighted energy (clamped against ene0, complex) and its weight."""
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        nchol = int(ham_data["chol"].shape[0])
        ene0 = float(ham_data.get("ene0", 0.0))
        lim = (2.0 / prop.dt) ** 0.5
        prop._zeta_source = self.field_source
        ov, aov, be, bw, states = [], [], [], [], []
        try:
            for _ in range(self.n_blocks):
                fields = self._fields(prop, prop_data, nchol)
                for s in range(self.n_prop_steps):
                    prop_data = prop.propagate_free(trial, ham_data, prop_data, fields[s], wave_data)
                e = trial.calc_energy(prop_data["walkers"], ham_data, wave_data)
                e = torch.where(torch.abs(e - ene0) > lim, torch.full_like(e, ene0), e)
                o = prop_data["overlaps"]
                ow = o * prop_data["weights"]
                be.append(torch.sum(e * ow) / torch.sum(ow))
                bw.append(torch.sum(ow))
                ov.append(torch.sum(o))
                aov.append(torch.sum(torch.abs(o)))
                w = prop_data["walkers"]
                states.append({"walkers": [t.clone() for t in w.data] if isinstance(w.data, list) else w.data.clone(),
                               "weights": prop_data["weights"].clone(), "overlaps": o.clone()})
        finally:
            prop._zeta_source = None
        return (torch.stack(ov), torch.stack(aov), states, torch.stack(be), torch.stack(bw),
                prop_data["key"])

    def __hash__(self) -> int:
        return hash((self.n_prop_steps, self.n_ene_blocks, self.n_sr_blocks, self.n_blocks))


@dataclass
class sampler_lno(sampler):
    """sampling.sampler_lno (sampling.py:583-694): every energy block also
    averages the fragment's orbital energy (trial.calc_orbenergy, an rhf_lno
    trial).  Its block end clamps the local energies against
    pop_control_ene_shift (not e_estimate), and the orbital energies where the
    already clamped energies are still out of range, which never happens: both
    as the reference does.  propagate_phaseless returns (E, prop_data, orbE)."""

    def _block_scan(self, prop, trial, ham_data, prop_data, wave_data, out_row):
        """sampling.py:586-631."""
        eng = prop.engine(ham_data, trial, wave_data)
        nchol = int(ham_data["chol"].shape[0])
        fields = self._fields(prop, prop_data, nchol)
        p, w, wb = eng.handle
        lib = _lib.lib()
        stream = _lib.stream_handle()
        st = make_state(prop_data, eng)
        for s in range(self.n_prop_steps):
            _lib.check(lib.afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st),
                                                     fields[s].data_ptr(), w, wb, stream),
                       "afq_propagate_constrained")
        note_state(prop_data, st, eng)
        sc = prop_data["_scalars"]
        wts = prop_data["weights"]
        sc[2].add_(wts.numel() - torch.count_nonzero(wts).to(torch.float64))
        prop_data["walkers"] = prop_data["walkers"].orthonormalize()
        prop_data.pop("_afq_green_of", None)
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        lim = (2.0 / prop.dt) ** 0.5
        shift = sc[1].clone()
        e = torch.real(trial.calc_energy(prop_data["walkers"], ham_data, wave_data, engine=eng))
        e = torch.where(torch.abs(e - shift) > lim, shift, e)
        o = torch.real(trial.calc_orbenergy(prop_data["walkers"], ham_data, wave_data, engine=eng))
        o = torch.where(torch.abs(e - shift) > lim, shift, o)
        bw = torch.sum(wts)
        out_row[0] = torch.sum(e * wts) / bw
        out_row[1] = bw
        out_row[2] = torch.sum(o * wts) / bw
        sc[1].copy_(0.9 * shift + 0.1 * out_row[0])

    def propagate_phaseless(self, ham, ham_data: dict, prop, prop_data: dict, trial, wave_data: dict):
        """sampling.py:663-689."""
        eng = prop.engine(ham_data, trial, wave_data)
        if not eng.has_prop:
            raise _lib.AfqError("propagation intermediates missing: call build_propagation_intermediates")
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        prop_data["n_killed_walkers"] = 0.0
        prop_data["pop_control_ene_shift"] = prop_data["e_estimate"]
        if isinstance(prop_data["pop_control_ene_shift"], torch.Tensor):
            prop_data["pop_control_ene_shift"] = prop_data["pop_control_ene_shift"].clone()
        sync_scalars(prop_data)
        nb = self.n_sr_blocks * self.n_ene_blocks
        out = torch.zeros(nb, 3, dtype=torch.float64, device=device())
        i = 0
        for _ in range(self.n_sr_blocks):
            for _ in range(self.n_ene_blocks):
                self._block_scan(prop, trial, ham_data, prop_data, wave_data, out[i])
                i += 1
            zeta = self._uniform(prop_data)
            prop_data["walkers"], prop_data["weights"] = prop_data[
                "walkers"].stochastic_reconfiguration_local(prop_data["weights"], zeta)
            prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        sc = prop_data["_scalars"]
        sc[2].div_(nb * prop.n_walkers)
        be, bw, bo = out[:, 0], out[:, 1], out[:, 2]
        prop_data["block_energies"] = out
        eng.check_status()
        return torch.sum(be * bw) / torch.sum(bw), prop_data, torch.sum(bo * bw) / torch.sum(bw)
