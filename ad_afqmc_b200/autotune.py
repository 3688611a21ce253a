"""Autotuner of the tile and schedule choices of one problem shape.

The C library picks tiles by fixed rules (layout.cuh); ``afq_set_tuning``
overrides them per shape (see include/afqmc_b200.h).  ``Autotuner`` times the
candidates of every knob on the real calls of an energy block, S steps of
``afq_propagate_constrained`` plus one ``afq_calc_energy``, from a fixed
walker state, with CUDA events on the current stream.  It keeps a value only
when it beats the best so far by more than ``min_gain``, searching one knob at
a time.  Records are cached in a JSON file keyed by the shape, so a shape is
timed once per machine:

    $AFQ_TUNING_CACHE, else ~/.cache/ad_afqmc_b200/tuning.json

Knobs (0 = the built-in rule):
  vhs_bn, fb_bn     tensor-core column tile of the VHS / force-bias GEMMs
  fb_splitk         split-K of the force-bias GEMM
  exch_bn           tensor-core exchange column tile (walkers per tile)
  f64_exch_bn       FP64 exchange tile (FP64 path, or spins whose tensor-core
                    tile does not fit shared memory)
  max_stages        cap on the tcgen05 pipeline depth
  prop_order        tile order of the tensor-core propagator launches: 0
                    alternates the direction over the walkers from one launch
                    to the next (each starts where the previous one ended, on
                    data still in L2), 1 always runs forward
  prop_chunk        2: the propagator sums its K in FP32 round-to-nearest
                    chunks of four 64-wide blocks (shared-memory staging, two
                    operand stages) instead of the built-in single TMEM chain
                    (four stages: 87 -> 79 us per launch at N=200, W=512).  Not
                    searched: it changes results beyond the last bits
  vhs_chunk         2: the VHS GEMM sums its K (= Nchol) in FP32 chunks of
                    four 64-wide blocks instead of the built-in single TMEM
                    chain per accumulator group (364 vs 276 us per launch at
                    N=200, G=1000, W=512).  Not searched: it changes results
                    beyond the last bits
  prop_bn           column tile of the tensor-core propagator (several tiles
                    per walker when narrower than 2 No; bit-identical results,
                    slower at every measured shape, so not searched)
  grid_cap          CTAs of the persistent kernels (a batch-level knob: a
                    solve alone never gains from fewer CTAs, but overlapping
                    fragments can; ``tune_batch`` sweeps it for a whole batch)

Tuning changes the order of some partial sums (split-K, exchange tiles), so
results move in the last bits, within the path's tolerance; a given record
always gives the same bits.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import threading
from typing import Dict, List, Optional

import torch

from . import _lib
from .walkers import UHFWalkers

_KNOB_ORDER = ("vhs_bn", "fb_bn", "fb_splitk", "exch_bn", "f64_exch_bn", "max_stages", "prop_order")


def shape_key(d: _lib.afq_dims) -> str:
    nb = d.nocc[0] if d.walker_type == _lib.AFQ_RESTRICTED else d.nocc[1]
    return f"N{d.norb}_na{d.nocc[0]}_nb{nb}_G{d.nchol}_W{d.nwalkers}_wt{d.walker_type}_tt{d.trial_type}_p{d.precision}"


def candidates(d: _lib.afq_dims) -> Dict[str, List[int]]:
    mixed = d.precision != 0
    out: Dict[str, List[int]] = {"fb_splitk": [1, 2, 4, 8], "f64_exch_bn": [80, 120, 160]}
    if mixed:
        out.update({"vhs_bn": [64, 128], "fb_bn": [64, 128], "exch_bn": [32, 64, 80, 96, 128],
                    "max_stages": [2, 3, 4], "prop_order": [1]})
    return out


def default_cache_path() -> str:
    p = os.environ.get("AFQ_TUNING_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "ad_afqmc_b200", "tuning.json")


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, reps: int = 3, min_gain: float = 0.02,
                 n_prop_steps: int = 10):
        self.path = cache_path if cache_path is not None else default_cache_path()
        self.reps = reps
        self.min_gain = min_gain
        self.S = n_prop_steps
        self._lock = threading.Lock()
        self.cache: Dict[str, Dict] = {}
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                self.cache = json.load(f)

    # -- cache -----------------------------------------------------------------
    def save(self) -> None:
        if not self.path:
            return
        with self._lock:
            os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)

    def apply_cached(self, eng) -> bool:
        """Register the cached record of this engine's shape, if any."""
        rec = self.cache.get(shape_key(eng.dims))
        if rec is None:
            return False
        _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec["tuning"]))
        eng.ensure_workspace()
        return True

    # -- timing ----------------------------------------------------------------
    def _objective(self, eng, snap: List[torch.Tensor], work: List[torch.Tensor], weights, overlaps,
                   scalars, fields, energy_out) -> float:
        """Median time (ms) of S steps + one energy evaluation from the snapshot."""
        lib, stream = _lib.lib(), _lib.stream_handle()
        p, w, wb = eng.handle
        st = _lib.afq_state()
        st.walkers[0] = work[0].data_ptr()
        st.walkers[1] = work[1].data_ptr() if len(work) > 1 else None
        st.weights, st.overlaps, st.scalars = weights.data_ptr(), overlaps.data_ptr(), scalars.data_ptr()
        wk = _lib.pair(*[t.data_ptr() for t in work] + [None] * (2 - len(work)))
        times = []
        for rep in range(self.reps + 1):
            for t, s in zip(work, snap):
                t.copy_(s)
            st.flags = 0
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for s in range(self.S):
                _lib.check(lib.afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st),
                                                         fields[s % len(fields)].data_ptr(), w, wb, stream),
                           "afq_propagate_constrained")
            _lib.check(lib.afq_calc_energy(C.byref(eng.dims), p, wk, energy_out.data_ptr(), w, wb, stream),
                       "afq_calc_energy")
            b.record()
            b.synchronize()
            if rep > 0:
                times.append(a.elapsed_time(b))
        times.sort()
        return times[len(times) // 2]

    def tune(self, eng, prop_data: dict, force: bool = False) -> Dict:
        """Tune the shape of `eng` (a propagation engine) from the walkers of
        `prop_data`; returns the record {"tuning", "ms", "ms_default"}."""
        key = shape_key(eng.dims)
        if not force and key in self.cache:
            self.apply_cached(eng)
            return self.cache[key]
        if not eng.has_prop:
            raise _lib.AfqError("tuning needs a propagation engine (build_propagation_intermediates)")
        d = eng.dims
        dev = eng.prepared.device
        wl = prop_data["walkers"]
        snap = [t.clone() for t in (wl.data if isinstance(wl, UHFWalkers) else [wl.data])]
        work = [t.clone() for t in snap]
        weights = prop_data["weights"].clone()
        overlaps = prop_data["overlaps"].clone()
        scalars = prop_data["_scalars"].clone()
        gen = torch.Generator(device="cpu").manual_seed(1234)
        fields = [torch.randn(d.nwalkers, d.nchol, generator=gen, dtype=torch.float64).to(dev)
                  for _ in range(2)]
        energy = torch.empty(d.nwalkers, dtype=torch.complex128, device=dev)

        def measure(rec: Dict[str, int]) -> Optional[float]:
            try:
                _lib.set_tuning(d, _lib.afq_tuning.from_dict(rec))
            except _lib.AfqError:
                return None  # not usable at this shape
            eng.ensure_workspace()
            return self._objective(eng, snap, work, weights, overlaps, scalars, fields, energy)

        best: Dict[str, int] = {}
        t_default = measure(best)
        t_best = t_default
        for knob in _KNOB_ORDER:
            for v in candidates(d).get(knob, []):
                rec = dict(best, **{knob: v})
                t = measure(rec)
                if t is not None and t < t_best * (1.0 - self.min_gain):
                    best, t_best = rec, t
        _lib.set_tuning(d, _lib.afq_tuning.from_dict(best))
        eng.ensure_workspace()
        out = {"tuning": best, "ms": t_best, "ms_default": t_default, "steps": self.S}
        with self._lock:
            self.cache[key] = out
        return out


def tune_batch(batch_factory, tuner: Optional[Autotuner] = None, grid_caps=(0, 74, 37),
               n_streams=(8, 16, 32), reps: int = 3) -> Dict:
    """Schedule knobs of a fragment batch: the persistent-kernel grid cap (one
    value for every fragment, on top of each shape's cached record) and the
    number of forked streams of the batch graph.  ``batch_factory(n_streams)``
    returns an uncaptured FragmentBatch; returns the fastest combination and
    leaves it registered."""
    def records(engines, cap):
        for eng in engines:
            rec = dict(tuner.cache.get(shape_key(eng.dims), {"tuning": {}})["tuning"]) if tuner else {}
            rec["grid_cap"] = cap
            _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec))
            eng.ensure_workspace()

    results = []
    for ns in n_streams:
        fb = batch_factory(ns)
        engines = [b.eng for b in fb.blocks]
        for cap in grid_caps:
            records(engines, cap)
            fb.capture()
            fb.step()
            torch.cuda.synchronize()
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                fb.step()
            e.record()
            e.synchronize()
            results.append({"n_streams": ns, "grid_cap": cap, "ms": a.elapsed_time(e) / reps})
        del fb
    best = min(results, key=lambda r: r["ms"])
    for eng in engines:  # the same shapes in every batch: leave the winner registered
        rec = dict(tuner.cache.get(shape_key(eng.dims), {"tuning": {}})["tuning"]) if tuner else {}
        rec["grid_cap"] = best["grid_cap"]
        _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec))
    return dict(best, sweep=results)
