"""Continuous-batching server for independent fragment solves.

Requests arrive over time: fragment Hamiltonians of different sizes, as an LNO
driver produces them. The reference solves these one at a time, each in a
fresh process: lnoutils.py:8-203 runs ``os.system("mpirun ... launch_script.py")``
once per fragment, and driver.afqmc_LNOenergy is driver.py:195-402.

The server keeps every admitted solve resident on the GPU: its prepared
Hamiltonian, workspace, walkers, weights and scalars. It advances the active
solves one energy block at a time. Each solve replays its own captured block
graph on its own stream, so kernels from different solves overlap on the device.

* Admission. A request is admitted when a slot is free and its device
  footprint fits in the HBM budget. The footprint is the prepared Hamiltonian,
  the workspace and the walker state, computed from the C ABI sizes before
  anything is allocated. Slots are capped (``max_slots``) at what keeps the
  GPU busy. Admitted requests then finish in about arrival order, instead of
  every queued request sharing the device and all finishing late.
* Setup off the launch path. A worker thread builds each admitted solve on its
  own stream: host-to-device copy of the integrals, intermediates, initial
  walkers and energy, and graph capture in thread-local capture mode. Blocks
  of the other solves keep launching meanwhile.
* Completion. ``n_eql`` equilibration blocks come first and are discarded.
  After every sampling block the (energy, weight) pair goes to pinned host
  memory without blocking. The stop rule defaults to the reference LNO
  driver's (driver.py:376-389): every ``max(max_blocks // 5, 1)`` blocks with
  n > 4, stop when std(E[:n+1]) / sqrt(n+1) < ``target_error``. The
  alternative is ``stop_rule="blocking"``, the plateau error of
  stat_utils.blocking_analysis (stat_utils.py:8-64). A solve always stops at
  ``max_blocks``.
* Determinism. A solve's arithmetic depends only on its own inputs and seed:
  its own RNG counter, workspace and stream. Its result is therefore the same
  alone and in any mix; tests/test_gpu_serving.py checks this bit for bit.

    python -m ad_afqmc_b200.serving --rate 20 --duration 10
"""

from __future__ import annotations

import argparse
import json
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib, hamiltonian, propagation, stat_utils, wavefunctions
from ._engine import dims_for
from .graphs import BlockGraph
from .synthetic import SyntheticSystem, fragment_chol_scale, make_fragment_batch, make_system


@dataclass
class Request:
    rid: int
    system: SyntheticSystem       # host-side integrals of the fragment
    n_walkers: int
    seed: int
    arrival: float = 0.0          # seconds from the start of the run
    prjlo: Optional[np.ndarray] = None  # (n_lo, nocc): an LNO fragment (orbital energy, rhf_lno)


@dataclass
class Result:
    rid: int
    energy: float
    error: Optional[float]
    n_blocks: int                 # sampling blocks (equilibration not counted)
    converged: bool
    arrival: float
    admitted: float
    started: float                # first block launched (setup done)
    finished: float
    block_energies: List[float] = field(default_factory=list)
    orbE: Optional[float] = None        # LNO fragments: orbital energy and its error
    orbE_err: Optional[float] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def footprint_bytes(req: Request, precision: str) -> int:
    """Device bytes of one solve: prepared layout + workspace + walkers/state."""
    trial = wavefunctions.rhf(req.system.norb, req.system.nelec)
    d = dims_for(trial, "restricted", req.n_walkers, req.system.nchol, precision)
    pbytes, wbytes = _lib.sizes(d)
    n, no, g, w = req.system.norb, req.system.nelec[0], req.system.nchol, req.n_walkers
    # walkers + SR copy + initial walkers; chol and its transposed/rotated copies on the torch side
    state = 3 * w * n * no * 16 + 12 * g * n * n + 8 * g * no * n * 2
    return int(pbytes + wbytes + state)


def sem_stop(energies: np.ndarray, max_blocks: int, target: float) -> Tuple[bool, Optional[float]]:
    """driver.py:376-389: after block n (0-based), when n % max(n_blocks // 5, 1)
    == 0 and n > 4, stop if std(E[:n+1]) / sqrt(n+1) < target."""
    n = len(energies) - 1
    if n <= 4 or n % max(max_blocks // 5, 1) != 0:
        return False, None
    sem = float(np.std(energies) / np.sqrt(n + 1))
    return sem < target, sem


class Solve:
    """One admitted request: engine, walkers and its captured block graph."""

    def __init__(self, req: Request, precision: str, n_prop_steps: int, t_admit: float,
                 device: Optional[int] = None, stream: Optional[torch.cuda.Stream] = None):
        if device is not None:
            torch.cuda.set_device(device)
        self.req = req
        self.t_admit = t_admit
        self.t_start = 0.0
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.lno = req.prjlo is not None
        self.host = torch.empty(3, dtype=torch.float64).pin_memory()
        self.host_status = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.event = torch.cuda.Event()
        sys_ = req.system
        with torch.cuda.stream(self.stream):
            trial = (wavefunctions.rhf_lno if self.lno else wavefunctions.rhf)(sys_.norb, sys_.nelec)
            ham = hamiltonian.hamiltonian(sys_.norb)
            prop = propagation.propagator_afqmc(dt=0.005, n_walkers=req.n_walkers, precision=precision)
            hd, wd = sys_.ham_data(), sys_.wave_data()
            if self.lno:
                wd["prjlo"] = np.asarray(req.prjlo, dtype=np.float64)
            hd = ham.build_measurement_intermediates(hd, trial, wd)
            hd = ham.build_propagation_intermediates(hd, prop, trial, wd)
            pd = prop.init_prop_data(trial, wd, hd, seed=req.seed)
            self.block = BlockGraph(ham, hd, prop, trial, wd, pd, n_prop_steps=n_prop_steps, lno=self.lno)
            self.block.capture(warmup=0, device_sync=False)
        self.energies: List[float] = []
        self.weights: List[float] = []
        self.orbes: List[float] = []
        self.n_done = 0
        self.in_flight = False

    def launch(self, n_eql: int = 0) -> None:
        """Queue the next block; the equilibration blocks ride along with the
        first sampling block (their results are not read)."""
        with torch.cuda.stream(self.stream):
            for _ in range(n_eql):
                self.block.replay()
            out = self.block.replay()
            self.host[: out.numel()].copy_(out, non_blocking=True)
            self.host_status.copy_(self.block.status, non_blocking=True)
            self.event.record(self.stream)
        self.in_flight = True

    def poll(self) -> bool:
        """True once the block in flight has finished (result read)."""
        if not self.in_flight or not self.event.query():
            return False
        self.in_flight = False
        if int(self.host_status[0]) != 0:
            raise _lib.AfqError(f"request {self.req.rid}: a device-side wait timed out; its blocks are invalid")
        self.energies.append(float(self.host[0]))
        self.weights.append(float(self.host[1]))
        if self.lno:
            self.orbes.append(float(self.host[2]))
        return True

    def blocking_error(self) -> Optional[float]:
        e, w = np.array(self.energies), np.array(self.weights)
        ok = np.isfinite(e) & np.isfinite(w) & (w > 0)
        if ok.sum() < 4:
            return None
        return stat_utils.blocking_analysis(w[ok], e[ok])[1]


class Server:
    def __init__(self, precision: str = "mixed", hbm_budget_gb: float = 180.0, max_slots: int = 16,
                 n_prop_steps: int = 10, n_eql: int = 5, target_error: float = 5e-4,
                 max_blocks: int = 40, stop_rule: str = "sem", min_blocks: int = 5,
                 setup_thread: bool = True, reserve_gb_per_slot: float = 4.0):
        if stop_rule not in ("sem", "blocking"):
            raise ValueError(f"stop_rule must be 'sem' or 'blocking', not {stop_rule!r}")
        self.precision = precision
        # the requested budget, capped by what the device has free now (less 2 GB of headroom
        # for the CUDA context, cuBLAS workspaces and allocator rounding)
        free = torch.cuda.mem_get_info()[0] if torch.cuda.is_available() else int(hbm_budget_gb * 1e9)
        self.budget = int(min(hbm_budget_gb * 1e9, free - 2e9))
        self.max_slots = max_slots
        self.S = n_prop_steps
        self.n_eql = n_eql
        self.target_error = target_error
        self.max_blocks = max_blocks
        self.stop_rule = stop_rule
        self.min_blocks = min_blocks
        self.setup_thread = setup_thread
        self.reserve = int(min(reserve_gb_per_slot * 1e9, self.budget / max(max_slots, 1)))
        self._streams: List[torch.cuda.Stream] = []

    def _stream_pool(self) -> List[torch.cuda.Stream]:
        """One stream per slot, kept across runs.  The caching allocator keeps
        freed blocks per stream, so a solve set up on a slot's stream reuses
        the memory of the solve that held the slot before; a block of
        ``reserve`` bytes allocated and freed once on every stream lets first
        solves of new sizes split cached memory instead of calling cudaMalloc."""
        while len(self._streams) < self.max_slots:
            st = torch.cuda.Stream()
            if self.reserve > 0:
                with torch.cuda.stream(st):
                    x = torch.empty(self.reserve, dtype=torch.uint8)
                    del x
            self._streams.append(st)
        return self._streams

    def _done(self, s: Solve) -> Tuple[bool, Optional[float], bool]:
        """(stop, error, converged) after the block just read.  LNO fragments
        stop on their orbital energies (driver.py:376-389), others on the
        block energies."""
        n = len(s.energies)
        if self.stop_rule == "sem":
            series = s.orbes if s.lno else s.energies
            conv, err = sem_stop(np.array(series), self.max_blocks, self.target_error)
        else:
            err = s.blocking_error() if n >= self.min_blocks else None
            conv = err is not None and err < self.target_error
        return conv or n >= self.max_blocks, err, conv

    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        pending = sorted(requests, key=lambda r: r.arrival)
        active: List[Solve] = []
        setting_up: List[Tuple[Future, int]] = []
        used = 0
        sizes: Dict[int, int] = {}
        results: List[Result] = []
        dev = torch.cuda.current_device()
        free_streams = list(self._stream_pool())
        slot_of: Dict[int, torch.cuda.Stream] = {}
        pool = ThreadPoolExecutor(max_workers=1) if self.setup_thread else None
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        try:
            while pending or active or setting_up:
                now = clock()
                # admit arrived requests while memory and slots allow
                while (pending and (pending[0].arrival <= now or not realtime)
                       and len(active) + len(setting_up) < self.max_slots):
                    fp = footprint_bytes(pending[0], self.precision)
                    if used + fp > self.budget and (active or setting_up):
                        break
                    req = pending.pop(0)
                    sizes[req.rid] = fp
                    used += fp
                    st = free_streams.pop()
                    slot_of[req.rid] = st
                    if pool is not None:
                        setting_up.append((pool.submit(Solve, req, self.precision, self.S, clock(), dev, st),
                                           req.rid))
                    else:
                        s = Solve(req, self.precision, self.S, clock(), stream=st)
                        s.t_start = clock()
                        s.launch(self.n_eql)
                        active.append(s)
                progressed = False
                for item in list(setting_up):
                    fut, _ = item
                    if fut.done():
                        s = fut.result()  # re-raises a setup error here
                        s.t_start = clock()
                        s.launch(self.n_eql)
                        active.append(s)
                        setting_up.remove(item)
                        progressed = True
                for s in list(active):
                    if not s.poll():
                        continue
                    progressed = True
                    stop, err, conv = self._done(s)
                    if stop:
                        e, w = np.array(s.energies), np.array(s.weights)
                        ok = np.isfinite(e) & (w > 0)
                        en = float(np.sum(e[ok] * w[ok]) / np.sum(w[ok])) if ok.any() else float("nan")
                        if err is None:
                            err = float(np.std(e) / np.sqrt(len(e))) if len(e) > 1 else None
                        res = Result(s.req.rid, en, err, len(e), conv, s.req.arrival, s.t_admit,
                                     s.t_start, clock(), list(s.energies))
                        if s.lno:
                            o = np.array(s.orbes)
                            res.orbE = float(np.sum(o[ok] * w[ok]) / np.sum(w[ok])) if ok.any() else float("nan")
                            res.orbE_err = float(np.std(o) / np.sqrt(len(o))) if len(o) > 1 else None
                        results.append(res)
                        active.remove(s)
                        used -= sizes.pop(s.req.rid)
                        free_streams.append(slot_of.pop(s.req.rid))
                    else:
                        s.launch()
                if not progressed:
                    if not active and not setting_up and pending and realtime:
                        time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.01)))
                    else:
                        time.sleep(0.0002)
        finally:
            if pool is not None:
                pool.shutdown(wait=True)
        torch.cuda.synchronize()
        return results


def make_requests(rate: float, duration: float, seed: int = 1005, large_frac: float = 0.10,
                  chol_scale: Optional[float] = None, pinned: bool = True,
                  lno: bool = False) -> List[Request]:
    """Poisson arrivals at ``rate``/s for ``duration`` s. Sizes follow the uneven
    fragment batch, plus ``large_frac`` of them at N=250, G=1250. The two-body
    scale is ``fragment_chol_scale(N)`` unless ``chol_scale`` is given. With
    ``pinned`` the client hands over its Cholesky vectors in page-locked memory."""
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
        cs = chol_scale if chol_scale is not None else fragment_chol_scale(sp["norb"])
        sys_ = make_system(sp["norb"], tuple(sp["nelec"]), sp["nchol"], sp["seed"], "rhf", chol_scale=cs)
        if pinned:
            sys_.pin()
        prj = None
        if lno:  # one localized orbital per fragment, a normalized row (lnoafqmc.py:147)
            prj = rng.standard_normal((1, sp["nelec"][0]))
            prj /= np.linalg.norm(prj)
        out.append(Request(i, sys_, sp["n_walkers"], sp["seed"], a, prj))
    return out


def one_by_one(requests: List[Request], server: Server) -> List[Result]:
    """Baseline: the same requests solved one at a time in arrival order, each
    set up when the previous one finished (what the per-fragment driver does,
    minus its process start-up)."""
    one = Server(server.precision, max_slots=1, n_prop_steps=server.S, n_eql=server.n_eql,
                 target_error=server.target_error, max_blocks=server.max_blocks,
                 stop_rule=server.stop_rule, min_blocks=server.min_blocks, setup_thread=False)
    return one.run(requests, realtime=True)


def summarize(results: List[Result], wall: float) -> Dict:
    lat = np.array([r.latency for r in results])
    queue = np.array([r.started - r.arrival for r in results])
    return {"n": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
            "mean_wait_to_first_block_s": float(queue.mean()),
            "fragments_per_s": len(results) / wall,
            "converged_fraction": float(np.mean([r.converged for r in results])),
            "mean_blocks": float(np.mean([r.n_blocks for r in results]))}


def setup_latency(precision: str = "mixed", norb: int = 250, nchol: int = 1250, n_walkers: int = 256,
                  reps: int = 5) -> Dict:
    """Per-request set-up time of the largest served fragment (N = 250, G =
    1250): integrals from the client's pinned buffer to the device,
    measurement and propagation intermediates, initial walkers and energy,
    and the capture of the block graph, on one stream (median of ``reps``)."""
    no = int(round(norb / 4))
    sys_ = make_system(norb, (no, no), nchol, 4242, "rhf", chol_scale=fragment_chol_scale(norb)).pin()
    times = []
    for k in range(reps + 1):
        req = Request(k, sys_, n_walkers, 100 + k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sv = Solve(req, precision, 10, 0.0)
        sv.stream.synchronize()
        if k > 0:  # the first one also loads kernels
            times.append(time.perf_counter() - t0)
        del sv
    return {"norb": norb, "nchol": nchol, "nocc": no, "n_walkers": n_walkers,
            "setup_ms_median": 1e3 * float(np.median(times)), "setup_ms_min": 1e3 * float(np.min(times)),
            "setup_ms": [1e3 * t for t in times]}


def bench(rate: float = 20.0, duration: float = 10.0, precision: str = "mixed", slots: int = 16,
          max_blocks: int = 40, stop_rule: str = "sem", lno: bool = False, baseline: bool = True) -> Dict:
    """The serving workload: Poisson arrivals at ``rate``/s for ``duration``
    s, served with continuous batching, then (``baseline``) the same requests
    solved one by one in arrival order.  Returns latency percentiles and
    fragments/s of both."""
    reqs = make_requests(rate, duration, lno=lno)
    srv = Server(precision, max_slots=slots, max_blocks=max_blocks, stop_rule=stop_rule)
    # warm the CUDA context and kernels with throw-away requests of every path
    warm = make_requests(4.0, 1.0, seed=7, lno=lno)[:3]
    srv.run(warm, realtime=False)
    one_by_one(warm[:1], srv)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    wall = time.perf_counter() - t0
    out = {"workload": (f"Poisson {rate}/s for {duration} s: N~U[30,160], No=round(N/4), G~U[4N,6N], "
                        f"W~U[64,256], 10% N=250/G=1250; stop std err < 0.5 mHa ({stop_rule}) "
                        f"or {max_blocks} blocks after 5 equilibration blocks"),
           "construction": ("synthetic recipe with the Cholesky vectors scaled by 0.035*sqrt(100/N) "
                            "(the unscaled recipe's block-energy noise keeps most fragments from "
                            "reaching 0.5 mHa); the work per block does not depend on the scale"),
           "precision": precision, "slots": slots, "lno": lno, "hbm_budget_gb": srv.budget / 1e9,
           "serving": summarize(res, wall)}
    if baseline:
        t0 = time.perf_counter()
        base = one_by_one(reqs, srv)
        out["one_by_one"] = summarize(base, time.perf_counter() - t0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_hi"])
    ap.add_argument("--max-blocks", type=int, default=40)
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--stop-rule", default="sem", choices=["sem", "blocking"])
    ap.add_argument("--no-baseline", action="store_true")
    ap.add_argument("--lno", action="store_true",
                    help="LNO fragments: orbital energies (rhf_lno), stop on their standard error")
    a = ap.parse_args()
    torch.cuda.set_device(0)
    print(json.dumps(bench(a.rate, a.duration, a.precision, a.slots, a.max_blocks, a.stop_rule, a.lno,
                           baseline=not a.no_baseline)))


if __name__ == "__main__":
    main()
