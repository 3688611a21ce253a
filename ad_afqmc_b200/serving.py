"""Continuous-batching server for independent fragment solves.

Requests (fragment Hamiltonians of different sizes, as produced by an LNO
driver — lnoutils.py:8-203 solves them one at a time, each in a fresh
process) arrive over time.  The server keeps every admitted solve resident on
the GPU — Hamiltonian layout, walkers, weights and scalars — and advances all
active solves one energy block at a time, each replaying its own captured
block graph on its own stream, so their kernels overlap on the device.

* Admission: a request is admitted when a slot is free and its device
  footprint (prepared Hamiltonian + workspace + walker state, computed from
  the C ABI sizes before anything is allocated) fits in the HBM budget.
* Completion: after every block the block energy is copied to pinned host
  memory without blocking; the solve stops when the blocking-analysis error of
  its block energies (stat_utils.blocking_analysis, the rule of
  driver.afqmc_LNOenergy, driver.py:376-389) drops below ``target_error`` after
  ``min_blocks``, or at ``max_blocks``.
* A solve's arithmetic depends only on its own inputs and seed (its own RNG
  counter, workspace and stream), so its result is the same alone and in any
  mix (tests/test_gpu_serving.py checks this bit for bit).

    python -m ad_afqmc_b200.serving --rate 20 --duration 10
"""

from __future__ import annotations

import argparse
import json
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib, hamiltonian, propagation, stat_utils, wavefunctions
from ._engine import dims_for
from .graphs import BlockGraph
from .synthetic import SyntheticSystem, make_fragment_batch, make_system


@dataclass
class Request:
    rid: int
    system: SyntheticSystem       # host-side integrals of the fragment
    n_walkers: int
    seed: int
    arrival: float = 0.0          # seconds from the start of the run


@dataclass
class Result:
    rid: int
    energy: float
    error: Optional[float]
    n_blocks: int
    converged: bool
    arrival: float
    admitted: float
    finished: float
    block_energies: List[float] = field(default_factory=list)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def footprint_bytes(req: Request, precision: str) -> int:
    """Device bytes of one solve: prepared layout + workspace + walkers/state."""
    trial = wavefunctions.rhf(req.system.norb, req.system.nelec)
    d = dims_for(trial, "restricted", req.n_walkers, req.system.nchol,
                 precision if precision != "fp64" else "fp64")
    pbytes, wbytes = _lib.sizes(d)
    # FP64 engine for the initial energy shares the layout sizes of the fp64 dims
    d64 = dims_for(trial, "restricted", req.n_walkers, req.system.nchol, "fp64")
    p64, w64 = _lib.sizes(d64)
    n, no, g, w = req.system.norb, req.system.nelec[0], req.system.nchol, req.n_walkers
    state = 3 * w * n * no * 16 + 12 * g * n * n + 8 * g * no * n * 2
    return int(pbytes + wbytes + p64 + w64 + state)


class Solve:
    """One admitted request: engine, walkers and its captured block graph."""

    def __init__(self, req: Request, precision: str, n_prop_steps: int, t_admit: float):
        self.req = req
        self.t_admit = t_admit
        self.stream = torch.cuda.Stream()
        sys_ = req.system
        with torch.cuda.stream(self.stream):
            trial = wavefunctions.rhf(sys_.norb, sys_.nelec)
            ham = hamiltonian.hamiltonian(sys_.norb)
            prop = propagation.propagator_afqmc(dt=0.005, n_walkers=req.n_walkers, precision=precision)
            hd, wd = sys_.ham_data(), sys_.wave_data()
            hd = ham.build_measurement_intermediates(hd, trial, wd)
            hd = ham.build_propagation_intermediates(hd, prop, trial, wd)
            pd = prop.init_prop_data(trial, wd, hd, seed=req.seed)
            self.block = BlockGraph(ham, hd, prop, trial, wd, pd, n_prop_steps=n_prop_steps)
            self.block.capture(warmup=0, device_sync=False)
        self.host = torch.empty(2, dtype=torch.float64).pin_memory()
        self.event = torch.cuda.Event()
        self.energies: List[float] = []
        self.weights: List[float] = []
        self.in_flight = False

    def launch(self) -> None:
        with torch.cuda.stream(self.stream):
            out = self.block.replay()
            self.host.copy_(out, non_blocking=True)
            self.event.record(self.stream)
        self.in_flight = True

    def poll(self) -> bool:
        """True once the block in flight has finished (result read)."""
        if not self.in_flight or not self.event.query():
            return False
        self.in_flight = False
        self.energies.append(float(self.host[0]))
        self.weights.append(float(self.host[1]))
        return True

    def error(self) -> Optional[float]:
        e = np.array(self.energies)
        w = np.array(self.weights)
        ok = np.isfinite(e) & np.isfinite(w) & (w > 0)
        if ok.sum() < 4:
            return None
        _, err = stat_utils.blocking_analysis(w[ok], e[ok])
        return err


class Server:
    def __init__(self, precision: str = "mixed", hbm_budget_gb: float = 170.0, max_slots: int = 64,
                 n_prop_steps: int = 10, target_error: float = 5e-4, min_blocks: int = 8,
                 max_blocks: int = 20):
        self.precision = precision
        self.budget = int(hbm_budget_gb * 1e9)
        self.max_slots = max_slots
        self.S = n_prop_steps
        self.target_error = target_error
        self.min_blocks = min_blocks
        self.max_blocks = max_blocks

    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        pending = sorted(requests, key=lambda r: r.arrival)
        active: List[Solve] = []
        used = 0
        sizes: Dict[int, int] = {}
        results: List[Result] = []
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        while pending or active:
            now = clock()
            # admit arrived requests while memory and slots allow
            while pending and (pending[0].arrival <= now or not realtime) and len(active) < self.max_slots:
                fp = footprint_bytes(pending[0], self.precision)
                if used + fp > self.budget and active:
                    break
                req = pending.pop(0)
                sizes[req.rid] = fp
                used += fp
                active.append(Solve(req, self.precision, self.S, clock()))
                active[-1].launch()
            progressed = False
            for s in list(active):
                if not s.poll():
                    continue
                progressed = True
                n = len(s.energies)
                err = s.error() if n >= self.min_blocks else None
                done = n >= self.max_blocks or (err is not None and err < self.target_error)
                if done:
                    e = np.array(s.energies)
                    w = np.array(s.weights)
                    ok = np.isfinite(e) & (w > 0)
                    en = float(np.sum(e[ok] * w[ok]) / np.sum(w[ok])) if ok.any() else float("nan")
                    results.append(Result(s.req.rid, en, err, n, err is not None and err < self.target_error,
                                          s.req.arrival, s.t_admit, clock(), list(s.energies)))
                    active.remove(s)
                    used -= sizes.pop(s.req.rid)
                    del s
                else:
                    s.launch()
            if not progressed:
                if not active and pending and realtime:
                    time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.01)))
                else:
                    time.sleep(0.0002)
        torch.cuda.synchronize()
        return results


def make_requests(rate: float, duration: float, seed: int = 1005, large_frac: float = 0.10,
                  chol_scale: float = 0.25) -> List[Request]:
    """Poisson arrivals at `rate`/s for `duration` s; sizes as the uneven fragment
    batch plus `large_frac` of them at N=250, G=1250."""
    rng = np.random.default_rng(seed)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        arrivals.append(t)
    specs = make_fragment_batch(len(arrivals), seed=seed, large_frac=large_frac)
    out = []
    for i, (a, sp) in enumerate(zip(arrivals, specs)):
        sys_ = make_system(sp["norb"], tuple(sp["nelec"]), sp["nchol"], sp["seed"], "rhf",
                           chol_scale=chol_scale)
        out.append(Request(i, sys_, sp["n_walkers"], sp["seed"], a))
    return out


def one_by_one(requests: List[Request], precision: str, server: Server) -> List[Result]:
    """Baseline: the same requests solved one at a time in arrival order."""
    one = Server(precision, max_slots=1, n_prop_steps=server.S, target_error=server.target_error,
                 min_blocks=server.min_blocks, max_blocks=server.max_blocks)
    return one.run(requests, realtime=True)


def summarize(results: List[Result], wall: float) -> Dict:
    lat = np.array([r.latency for r in results])
    return {"n": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
            "fragments_per_s": len(results) / wall,
            "converged_fraction": float(np.mean([r.converged for r in results])),
            "mean_blocks": float(np.mean([r.n_blocks for r in results]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_hi"])
    ap.add_argument("--max-blocks", type=int, default=20)
    ap.add_argument("--no-baseline", action="store_true")
    a = ap.parse_args()
    torch.cuda.set_device(0)
    reqs = make_requests(a.rate, a.duration)
    srv = Server(a.precision, max_blocks=a.max_blocks)
    # warm the CUDA context and kernels with one throw-away request
    srv.run([make_requests(1.0, 1.0, seed=7)[0]], realtime=False)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    out = {"workload": f"Poisson {a.rate}/s for {a.duration} s, config-4 sizes + 10% N=250/G=1250",
           "precision": a.precision, "serving": summarize(res, wall)}
    if not a.no_baseline:
        t0 = time.perf_counter()
        base = one_by_one(reqs, a.precision, srv)
        out["one_by_one"] = summarize(base, time.perf_counter() - t0)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
