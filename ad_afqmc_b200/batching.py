"""Uneven fragment batches: many independent AFQMC solves advanced together.

A fragment is one seeded synthetic system (``synthetic.make_fragment_batch``:
N ~ U[30,160], No = round(N/4), G ~ U[4N, 6N], W ~ U[64, 256]) with its own
engine (prepared Hamiltonian + workspace) and its own ``BlockGraph``.
``FragmentBatch`` records one energy block of every fragment into a single
CUDA graph, each fragment on one of ``n_streams`` forked streams, so one
replay advances all fragments and their kernels overlap on the device.

    python -m ad_afqmc_b200.batching --precision mixed --fragments 64
"""

from __future__ import annotations

import argparse
import json
import time
from typing import Dict, List, Optional

import torch

from . import hamiltonian, propagation, wavefunctions
from .graphs import BatchGraph, BlockGraph, GroupedBatchGraph
from .synthetic import make_fragment_batch, make_system


def make_fragment_block(spec: Dict, precision: str = "mixed", n_prop_steps: int = 10,
                        dt: float = 0.005, chol_scale: float = 0.25) -> BlockGraph:
    """Engine, walkers and block graph (not yet captured) of one fragment."""
    sys_ = make_system(spec["norb"], tuple(spec["nelec"]), spec["nchol"], spec["seed"], "rhf",
                       chol_scale=chol_scale)
    trial = wavefunctions.rhf(sys_.norb, sys_.nelec)
    ham = hamiltonian.hamiltonian(sys_.norb)
    prop = propagation.propagator_afqmc(dt=dt, n_walkers=spec["n_walkers"], precision=precision)
    hd, wd = sys_.ham_data(), sys_.wave_data()
    hd = ham.build_measurement_intermediates(hd, trial, wd)
    hd = ham.build_propagation_intermediates(hd, prop, trial, wd)
    pd = prop.init_prop_data(trial, wd, hd, seed=spec["seed"])
    return BlockGraph(ham, hd, prop, trial, wd, pd, n_prop_steps=n_prop_steps)


class FragmentBatch:
    def __init__(self, specs: List[Dict], precision: str = "mixed", n_prop_steps: int = 10,
                 n_streams: int = 16, chol_scale: float = 0.25, tuner=None):
        self.specs = specs
        self.blocks = [make_fragment_block(s, precision, n_prop_steps, chol_scale=chol_scale)
                       for s in specs]
        self.tuning: List[Optional[Dict]] = [None] * len(self.blocks)
        if tuner is not None:
            # per-shape tile records, timed (or read from the cache) before any capture
            for i, b in enumerate(self.blocks):
                self.tuning[i] = tuner.tune(b.eng, b.pd)
            tuner.save()
        self.walker_steps_per_block = sum(s["n_walkers"] for s in specs) * n_prop_steps
        self.batch = BatchGraph(self.blocks, n_streams=n_streams)

    def capture(self) -> "FragmentBatch":
        self.batch.capture(warmup=1)
        return self

    def step(self) -> None:
        self.batch.replay()

    def energies(self) -> torch.Tensor:
        return torch.stack([b.block_out[0] for b in self.blocks])


def _time(fn, reps: int) -> float:
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def bench(n_fragments: int = 64, precision: str = "mixed", n_prop_steps: int = 10,
          n_streams: int = 16, reps: int = 3, seed: int = 1004, tune: bool = False,
          tuning_cache: Optional[str] = None) -> Dict:
    specs = make_fragment_batch(n_fragments, seed=seed)
    t0 = time.perf_counter()
    fb = FragmentBatch(specs, precision, n_prop_steps, n_streams)
    setup_s = time.perf_counter() - t0
    ws = fb.walker_steps_per_block
    # one by one: every fragment's block launched eagerly, fragment after fragment
    for b in fb.blocks:
        b.body()
    ms_seq = _time(lambda: [b.body() for b in fb.blocks], 1)
    # one by one from per-fragment graphs (launch overhead removed, no overlap)
    for b in fb.blocks:
        b.capture(warmup=0)
    ms_seq_graph = _time(lambda: [b.replay() for b in fb.blocks], reps)
    # all fragments in one graph on forked streams
    fb.capture()
    ms_batch = _time(fb.step, reps)
    extra: Dict = {}
    if precision != "fp64":
        # all fragments in one graph with the steps in grouped launches (persistent grouped
        # tcgen05 GEMMs over (fragment, tile) work lists), from the same state onward
        gb = GroupedBatchGraph(fb.blocks, n_streams=n_streams).capture(warmup=1)
        ms_grouped = _time(gb.replay, reps)
        gb.check_status()
        extra.update({"grouped_graph_ms": ms_grouped,
                      "walker_steps_per_s_grouped": ws / (ms_grouped / 1e3),
                      "launches_per_block_grouped": gb.launches_per_block,
                      "speedup_grouped_vs_forked_streams": ms_batch / ms_grouped})
        del gb
    if tune:
        from .autotune import Autotuner, tune_batch

        tuner = Autotuner(cache_path=tuning_cache)
        t0 = time.perf_counter()
        recs = [tuner.tune(b.eng, b.pd) for b in fb.blocks]
        tuner.save()
        extra["tune_s"] = time.perf_counter() - t0
        extra["tuned_shapes_changed"] = sum(1 for r in recs if r["tuning"])
        extra["tuned_fragment_gain"] = sum(r["ms_default"] for r in recs) / sum(r["ms"] for r in recs)
        fb.capture()
        extra["batched_graph_tuned_ms"] = _time(fb.step, reps)
        sched = tune_batch(lambda ns: FragmentBatch(specs, precision, n_prop_steps, ns), tuner,
                           n_streams=(n_streams, 2 * n_streams), reps=reps)
        extra["schedule"] = {k: sched[k] for k in ("n_streams", "grid_cap", "ms")}
        extra["schedule_sweep"] = sched["sweep"]
        best = min(ms_batch, extra["batched_graph_tuned_ms"], sched["ms"])
        extra["walker_steps_per_s_tuned"] = ws / (best / 1e3)
    return extra | {
        "workload": f"{n_fragments} fragments N~U[30,160], No=round(N/4), G~U[4N,6N], W~U[64,256]",
        "precision": precision, "n_streams": n_streams, "walker_steps_per_block": ws,
        "setup_s": setup_s,
        "one_by_one_eager_ms": ms_seq, "one_by_one_graph_ms": ms_seq_graph, "batched_graph_ms": ms_batch,
        "walker_steps_per_s_batched": ws / (ms_batch / 1e3),
        "walker_steps_per_s_one_by_one": ws / (ms_seq / 1e3),
        "speedup_batched_vs_one_by_one": ms_seq / ms_batch,
        "launches_per_block": fb.batch.launches_per_block,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--fragments", type=int, default=64)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_hi"])
    ap.add_argument("--streams", type=int, default=16)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--tune", action="store_true", help="autotune tiles per shape and the batch schedule")
    ap.add_argument("--tuning-cache", default=None)
    a = ap.parse_args()
    torch.cuda.set_device(0)
    print(json.dumps(bench(a.fragments, a.precision, n_streams=a.streams, reps=a.reps, tune=a.tune,
                           tuning_cache=a.tuning_cache)))


if __name__ == "__main__":
    main()
