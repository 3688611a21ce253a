#!/usr/bin/env python
"""Throughput benchmark of the phaseless AFQMC walker path (walker-steps/s).

Workload (default): synthetic RHF Hamiltonian Norb=200, Na=Nb=40, Nchol=1000,
512 walkers, dt=0.005 (see ad_afqmc_b200/synthetic.py for the recipe).  One
bench step is one energy block of ``sampler.propagate_phaseless``: 10
phaseless steps (device-drawn fields, force bias, VHS, Taylor propagator,
overlaps, weights) followed by the block end (QR, overlaps, local energies,
clamp, block energy, population shift) and one reconfiguration.  The metric
counts walker-steps: 512 x 10 per bench step, with the per-block QR, energy
and reconfiguration amortised inside the time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # the CPU oracle (NumPy port) arm

Multi-GPU runs (torchrun, one process per GPU) are replicas: each rank runs
its own walker population (weak scaling); the block energy and weight are
combined with one NCCL all-reduce per block, the driver's only exchange.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "walker-steps/s @Norb200/Nchol1000 (mixed vs FP64 GPU, <=0.1 mHa); p99 solve latency"
UNIT = "walker-steps/s"
CONFIG = "rhf_n200_g1000"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_hi"])
    ap.add_argument("--eager", action="store_true",
                    help="launch every kernel from Python instead of replaying the block's CUDA graph")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the FP64 comparison leg and the block-energy error check")
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--walkers", type=int, default=0, help="override walker count")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other two workloads (N=10 RHF and N=300 UHF, FP64 and mixed)")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the fragment batch (64 uneven fragments) and the serving run")
    ap.add_argument("--serving-duration", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-walkers", type=int, default=32)
    ap.add_argument("--chol-scale", type=float, default=1.0,
                    help="Cholesky scale of the synthetic system (1.0 = prescribed recipe)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU oracle timing (reported baseline; also the --impl reference arm)
# ---------------------------------------------------------------------------
def cpu_oracle_sample(sys_, n_walkers, n_steps, dt, seed=5):
    """Time the NumPy oracle on a bounded sample: n_walkers walkers, n_steps
    phaseless steps and one block end (QR + energies).  Returns walker-steps/s."""
    from oracle import afqmc_oracle as orc

    trial = orc.RHFTrial(sys_.norb, sys_.nelec) if sys_.trial == "rhf" else orc.UHFTrial(sys_.norb, sys_.nelec)
    wt = "restricted" if sys_.trial == "rhf" else "unrestricted"
    ham = sys_.ham_data()
    wave = sys_.wave_data()
    prop = orc.Propagator(dt=dt, n_walkers=n_walkers, walker_type=wt)
    ham = trial.build_measurement_intermediates(ham, wave)
    ham = prop.build_propagation_intermediates(ham, trial, wave)
    rng = np.random.default_rng(seed)
    pd = prop.init_prop_data(trial, wave, ham)
    pd["n_killed_walkers"] = 0
    fields = rng.standard_normal((n_steps, n_walkers, sys_.nchol))
    t0 = time.perf_counter()
    for s in range(n_steps):
        pd = prop.propagate_constrained(trial, ham, pd, fields[s], wave)
    pd["walkers"] = orc.orthonormalize(pd["walkers"])
    pd["overlaps"] = trial.calc_overlap(pd["walkers"], wave)
    e = np.real(trial.calc_energy(pd["walkers"], ham, wave))
    idx, w = orc.sr_indices(pd["weights"], 0.5)
    t = time.perf_counter() - t0
    return n_walkers * n_steps / t, t


def clocks_start(path):
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def clocks_stop(proc, path, gpu_index):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9 or f[0] != str(gpu_index):
            continue
        try:
            sm.append(float(f[1]))
            mx = float(f[2])
        except ValueError:
            continue
        for n, v in zip(names, f[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def measure_fp64_peak(n: int = 8192, reps: int = 5) -> float:
    """FP64 dense peak of this GPU in TFLOP/s: cuBLAS DGEMM n^3 through
    torch.matmul, best of `reps` after warm-up, timed with CUDA events (the
    peaks file carries no FP64 figure, so every run measures its own)."""
    import torch

    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def path_flops_per_walker_step(sys_, S: int, K: int = 6) -> float:
    """Algorithmic real flops of one walker-step, the per-block QR and energy
    amortised over S steps (complex FMA = 8 flops, real x complex = 4):
    per spin sector s with n_s occupied orbitals, force bias 4 G N n_s,
    Taylor terms 8 (K-1) N^2 n_s, one-body half-steps 8 N^2 n_s, overlap and
    Green's function 16 N n_s^2 + 16 n_s^3, plus the VHS build 4 G N^2; per
    block the energy 4 G n_s^2 N + 8 G n_s^2 and the QR 8 (2 N n_s^2 - 2/3 n_s^3).
    Restricted walkers count one sector.  N=200, n=40, G=1000, S=10: 4.05e8."""
    N, G = sys_.norb, sys_.nchol
    secs = [sys_.nelec[0]] if sys_.trial == "rhf" else list(sys_.nelec)
    step = 4.0 * G * N * N
    block = 0.0
    for n in secs:
        step += 4.0 * G * N * n + 8.0 * (K - 1) * N * N * n + 8.0 * N * N * n + 16.0 * N * n * n + 16.0 * n ** 3
        block += 4.0 * G * n * n * N + 8.0 * G * n * n + 8.0 * (2.0 * N * n * n - 2.0 / 3.0 * n ** 3)
    return step + block / S


def blas_threads() -> int:
    try:
        from threadpoolctl import threadpool_info

        n = [i.get("num_threads", 0) for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(n) if n else 1
    except Exception:
        return os.cpu_count() or 1


# Cholesky scales of the same-shape systems on which the mixed-precision
# block-energy error is measured: the largest of 1, 1/2, 1/4, 1/10, 1/20 at
# which at most 1 % of the local energies lie further than sqrt(2/dt) from
# e_estimate over the first blocks (the NumPy oracle, 8 walkers, 3 blocks).
# With the prescribed recipe (scale 1) the N = 200 and N = 300 systems sit in
# the regime where the clamp of sampling.py:84-88 replaces almost every local
# energy, and the block energies then agree across precisions by construction.
ACCURACY_CHOL_SCALE = {"h10_sto6g_synthetic": 0.5, "rhf_n200_g1000": 0.1, "uhf_n300_g1500": 0.1}


class Solver:
    """One walker population of a synthetic system on the device, built
    through the reference-facing API (intermediates, initial walkers and
    energy) for one precision."""

    def __init__(self, sys_, precision, n_walkers, dt, seed):
        from ad_afqmc_b200 import hamiltonian, propagation, wavefunctions

        self.sys = sys_
        self.trial = (wavefunctions.rhf(sys_.norb, sys_.nelec) if sys_.trial == "rhf"
                      else wavefunctions.uhf(sys_.norb, sys_.nelec))
        self.wt = "restricted" if sys_.trial == "rhf" else "unrestricted"
        self.ham = hamiltonian.hamiltonian(sys_.norb)
        self.hd, self.wv = sys_.ham_data(), sys_.wave_data()
        self.prop = propagation.propagator_afqmc(dt=dt, n_walkers=n_walkers, walker_type=self.wt,
                                                 precision=precision)
        self.hd = self.ham.build_measurement_intermediates(self.hd, self.trial, self.wv)
        self.hd = self.ham.build_propagation_intermediates(self.hd, self.prop, self.trial, self.wv)
        self.pd = self.prop.init_prop_data(self.trial, self.wv, self.hd, seed=seed)


def time_graph_blocks(sv, S, steps, warmup):
    """Blocks (S steps, block end, comb, e_estimate update) replayed from one
    CUDA graph; returns (ms per block, killed-walker fraction of the last
    block, graph launches per block)."""
    import torch

    from ad_afqmc_b200.graphs import BlockGraph

    bg = BlockGraph(sv.ham, sv.hd, sv.prop, sv.trial, sv.wv, sv.pd, n_prop_steps=S).capture(warmup=1)
    for _ in range(warmup):
        bg.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        bg.replay()
    b.record()
    torch.cuda.synchronize()
    bg.check_status()
    killed = float(sv.pd["_scalars"][2])
    n = bg.launches_per_block
    del bg
    return a.elapsed_time(b) / steps, killed, n


def accuracy_check(sys_, precision, W, dt, S, nb, seed=4242):
    """Block energies of `precision` and of the FP64 path from the same
    initial walkers and the same device-drawn fields (identical Philox
    streams), nb blocks of S steps.  Returns the largest block-energy
    difference, the difference of the unclamped weighted local energies of
    the final walkers (both evaluated in FP64), the largest fraction of local
    energies clamped by the sqrt(2/dt) rule of sampling.py:84-88 (FP64 run;
    walkers after each block's comb, against the e_estimate of that block) and
    the killed-walker fraction."""
    import torch

    from ad_afqmc_b200 import sampling

    lim = (2.0 / dt) ** 0.5
    res = {}
    for prec in (precision, "fp64"):
        sv = Solver(sys_, prec, W, dt, seed)
        smp = sampling.sampler(n_prop_steps=S, n_ene_blocks=1, n_sr_blocks=1)
        es, clamped, killed = [], 0.0, 0.0
        for _ in range(nb):
            e_est = sv.pd["e_estimate"].clone()
            e, sv.pd = smp.propagate_phaseless(sv.ham, sv.hd, sv.prop, sv.pd, sv.trial, sv.wv)
            es.append(float(e))
            killed = max(killed, float(sv.pd["n_killed_walkers"]))
            el = torch.real(sv.trial.calc_energy(sv.pd["walkers"], sv.hd, sv.wv))
            clamped = max(clamped, float(torch.mean((torch.abs(el - e_est) > lim).double())))
            sv.pd["e_estimate"] = 0.9 * sv.pd["e_estimate"] + 0.1 * e
        el = torch.real(sv.trial.calc_energy(sv.pd["walkers"], sv.hd, sv.wv))
        wsum = torch.sum(sv.pd["weights"])
        e_unc = float(torch.sum(el * sv.pd["weights"]) / wsum) if float(wsum) > 0 else float("nan")
        res[prec] = (es, e_unc, clamped, killed)
        del sv, smp
        torch.cuda.empty_cache()
    err = max(abs(a - b) for a, b in zip(res[precision][0], res["fp64"][0]))
    return {"block_energy_error_ha": err,
            "unclamped_local_energy_error_ha": abs(res[precision][1] - res["fp64"][1]),
            "clamped_fraction": res["fp64"][2], "clamped_fraction_mixed": res[precision][2],
            "killed_fraction": res[precision][3], "killed_fraction_fp64": res["fp64"][3],
            "block_energies_fp64": res["fp64"][0], "blocks": nb, "steps_per_block": S,
            "n_walkers": W, "chol_scale": None}


def measure_config(name, precision, steps, warmup, nb_acc):
    """FP64 and `precision` walker-steps/s of one named workload (graph
    replays, prescribed recipe) and its block-energy error in the unclamped
    regime (same shape, Cholesky vectors scaled by ACCURACY_CHOL_SCALE)."""
    import torch

    from ad_afqmc_b200.synthetic import make_config

    sys_, cfg = make_config(name)
    W, S, dt = cfg["n_walkers"], cfg["n_prop_steps"], cfg["dt"]
    out = {"workload": name, "norb": sys_.norb, "nelec": list(sys_.nelec), "nchol": sys_.nchol,
           "n_walkers": W, "n_prop_steps": S, "dt": dt, "trial": sys_.trial}
    for prec in (precision, "fp64"):
        sv = Solver(sys_, prec, W, dt, 1000)
        ms, killed, n = time_graph_blocks(sv, S, steps if prec != "fp64" else max(2, steps // 2),
                                          warmup)
        out[prec] = {"walker_steps_per_s": W * S / (ms / 1e3), "ms_per_block": ms,
                     "killed_walker_fraction": killed, "launches_per_block": n}
        del sv
        torch.cuda.empty_cache()
    out["speedup_vs_fp64"] = out[precision]["walker_steps_per_s"] / out["fp64"]["walker_steps_per_s"]
    scale = ACCURACY_CHOL_SCALE[name]
    sys_a, _ = make_config(name, chol_scale=scale)
    acc = accuracy_check(sys_a, precision, W, dt, S, nb_acc)
    acc["chol_scale"] = scale
    out["accuracy"] = acc
    return out

# DRAM bytes (read + written) per propagator launch, mean over the 7 launches
# of one step, from ncu (dram__bytes_read.sum + dram__bytes_write.sum, caches
# flushed before each launch) on the bench workload (N=200, No=40, G=1000,
# 512 walkers, mixed, Taylor terms in Horner form).
PROP_DRAM_BYTES_PER_LAUNCH = 243791506


def main():
    args = parse()
    from ad_afqmc_b200.synthetic import make_config

    sys_, cfg = make_config(args.config, chol_scale=args.chol_scale)
    W = args.walkers or cfg["n_walkers"]
    S = cfg["n_prop_steps"]
    dt = cfg["dt"]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        nw = max(8, args.cpu_walkers // 2)
        vals = []
        for i in range(args.warmup + args.steps):
            v, t = cpu_oracle_sample(sys_, nw, S, dt, seed=i)
            if i >= args.warmup:
                vals.append(v)
        val = float(np.mean(vals))
        cores = os.cpu_count()
        out = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * nw * S / val,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic",
               "config": {"workload": args.config, "norb": sys_.norb, "nelec": list(sys_.nelec),
                          "nchol": sys_.nchol, "n_walkers": nw, "n_prop_steps": S, "dt": dt},
               "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"{nw} walkers x {S} steps + 1 block end (QR, energies, comb) "
                                          "per step, NumPy oracle (the JAX reference needs jax, absent)"},
               "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return 0

    import torch

    if world > 1:
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    from ad_afqmc_b200 import _lib, hamiltonian, propagation, sampling, wavefunctions
    from ad_afqmc_b200.driver import afqmc_blocks

    trial = wavefunctions.rhf(sys_.norb, sys_.nelec) if sys_.trial == "rhf" else wavefunctions.uhf(sys_.norb, sys_.nelec)
    wt = "restricted" if sys_.trial == "rhf" else "unrestricted"
    ham = hamiltonian.hamiltonian(sys_.norb)

    def setup(system, precision, seed):
        hd, wv = system.ham_data(), system.wave_data()
        pr = propagation.propagator_afqmc(dt=dt, n_walkers=W, walker_type=wt, precision=precision)
        hd = ham.build_measurement_intermediates(hd, trial, wv)
        hd = ham.build_propagation_intermediates(hd, pr, trial, wv)
        pd_ = pr.init_prop_data(trial, wv, hd, seed=seed)
        return hd, wv, pr, pd_

    def one_block(smp_, hd, wv, pr, pd_):
        e, pd_ = smp_.propagate_phaseless(ham, hd, pr, pd_, trial, wv)
        if world > 1:
            t = torch.stack([e * torch.sum(pd_["weights"]), torch.sum(pd_["weights"])])
            dist.all_reduce(t)
        pd_["e_estimate"] = 0.9 * pd_["e_estimate"] + 0.1 * e
        return pd_, e

    def timed_run(precision, steps, warmup, profile_kernel=None, graph=False):
        hd, wv, pr, pd_ = setup(sys_, precision, 1000 + rank)
        if graph:
            # the block (fields, 10 steps, block end, comb, e_estimate update) as one CUDA graph;
            # with several ranks the comb and the estimate update follow the reference driver
            # (driver.py:133-168): block energy all-reduced (weighted), walkers reconfigured
            # across ranks (sr_ranks.py), e_estimate from the global block energy
            from ad_afqmc_b200.graphs import BlockGraph
            multi = world > 1
            bg = BlockGraph(ham, hd, pr, trial, wv, pd_, n_prop_steps=S, reconfigure=not multi,
                            update_estimate=not multi).capture(warmup=1)
            zeta_rng = np.random.default_rng(97)  # identical stream on every rank

            def run_block():
                out = bg.replay()
                if multi:
                    wsum = torch.sum(pd_["weights"])
                    t = torch.stack([out[0] * wsum, wsum])
                    dist.all_reduce(t)
                    e_glob = t[0] / t[1]
                    new, w_new = pd_["walkers"].stochastic_reconfiguration_global(
                        pd_["weights"], float(zeta_rng.random()), dist.group.WORLD)
                    for dst, src in zip(bg.tensors, new.data if isinstance(new.data, list) else [new.data]):
                        dst.copy_(src)
                    pd_["weights"].copy_(w_new)
                    pd_["overlaps"].copy_(trial.calc_overlap(pd_["walkers"], wv))
                    sc = pd_["_scalars"]
                    sc[0].mul_(0.9).add_(0.1 * e_glob)
        else:
            smp_ = sampling.sampler(n_prop_steps=S, n_ene_blocks=1, n_sr_blocks=1)

            def run_block():
                nonlocal pd_
                pd_, _ = one_block(smp_, hd, wv, pr, pd_)
        for _ in range(warmup):
            run_block()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        n0 = _lib.launch_count()
        if profile_kernel and not graph:
            _lib.profile_begin(profile_kernel)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(steps):
            run_block()
        stop.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = start.elapsed_time(stop)
        kern = _lib.profile_end() if (profile_kernel and not graph) else (0.0, 0)
        launches = _lib.launch_count() - n0
        if graph:
            launches = bg.launches_per_block * steps + launches  # + eager launches (several ranks)
            if profile_kernel:
                # the dominant kernel timed with CUDA events in eager blocks of the same state
                smp_ = sampling.sampler(n_prop_steps=S, n_ene_blocks=1, n_sr_blocks=1)
                _lib.profile_begin(profile_kernel)
                for _ in range(max(1, steps // 2)):
                    pd_, _ = one_block(smp_, hd, wv, pr, pd_)
                torch.cuda.synchronize()
                kern = _lib.profile_end()
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, kern, launches, float(pd_["n_killed_walkers"]), (hd, wv, pr, pd_)

    clk_path = os.path.join(tempfile.gettempdir(), f"afq_clocks_{rank}.csv")
    clk = clocks_start(clk_path)
    ms_total, (kern_ms, kern_n), launches, killed, (ham_data, wave, prop, pd) = timed_run(
        args.precision, args.steps, args.warmup, "vhs" if args.precision == "fp64" else "prop",
        graph=not args.eager)
    clocks = clocks_stop(clk, clk_path, torch.cuda.current_device())
    value = world * W * S * args.steps / (ms_total / 1e3)

    # ---- FP64 GPU path on the same workload, and the block-energy error -------
    compare = None
    if not args.no_compare and args.precision != "fp64":
        ms64, _, _, _, _ = timed_run("fp64", max(2, args.steps // 2), 1, graph=not args.eager)
        v64 = world * W * S * max(2, args.steps // 2) / (ms64 / 1e3)
        compare = {"fp64_value": v64, "fp64_ms_per_step": ms64 / max(2, args.steps // 2),
                   "speedup_vs_fp64": value / v64}
        if world == 1:
            # accuracy on the same shape in the unclamped regime (Cholesky vectors scaled so
            # that <= 1 % of the local energies meet the sqrt(2/dt) clamp)
            from ad_afqmc_b200.synthetic import make_config as _mk
            scale = ACCURACY_CHOL_SCALE.get(args.config, 0.1)
            sys_h, _ = _mk(args.config, chol_scale=scale)
            acc = accuracy_check(sys_h, args.precision, W, dt, S, 3)
            acc["chol_scale"] = scale
            compare.update({k: acc[k] for k in ("block_energy_error_ha", "unclamped_local_energy_error_ha",
                                                "block_energies_fp64")})
            compare["clamped_fraction_check"] = acc["clamped_fraction"]
            compare["killed_fraction_check"] = acc["killed_fraction"]
            compare["block_energy_check"] = (f"3 blocks x {S} steps, {W} walkers, chol_scale {scale}, "
                                             "same walkers and device-drawn fields, vs the FP64 GPU path "
                                             "(which matches the NumPy oracle to 1e-8 Ha)")
            # the headline shape on that live population: same kernels, timed the same way
            sv = Solver(sys_h, args.precision, W, dt, 1000)
            ms_live, killed_live, _ = time_graph_blocks(sv, S, args.steps, 2)
            compare["live_population"] = {"value": W * S / (ms_live / 1e3), "ms_per_step": ms_live,
                                          "chol_scale": scale, "killed_walker_fraction": killed_live}
            del sv
            torch.cuda.empty_cache()
        compare["fp64_peak_tflops_measured"] = measure_fp64_peak()
        # whole-path FP64 rate (algorithmic flops per walker-step) against the measured DGEMM peak
        compare["fp64_path_tflops"] = v64 * path_flops_per_walker_step(sys_, S) / 1e12
        compare["fp64_path_frac_of_dgemm"] = compare["fp64_path_tflops"] / compare["fp64_peak_tflops_measured"]

    # ---- end to end through the public API with host buffers -------------
    e2e = None
    if not args.no_e2e:
        G = sys_.nchol
        host_fields = torch.empty((S, W, G), dtype=torch.float64).pin_memory()
        host_fields.normal_(generator=torch.Generator().manual_seed(7 + rank))

        class PinnedSource:
            def fields(self, s, w, g):
                return host_fields.to(dev, non_blocking=True)

            def uniform(self):
                return 0.5

        if world == 1:
            # the block as one CUDA graph fed from host memory (graphs.HostFieldBlocks):
            # every block uploads its fields from the pinned buffer (on a copy stream,
            # overlapping the previous block) and reads (energy, weight, weights) back
            from ad_afqmc_b200.graphs import BlockGraph, HostFieldBlocks

            bg = BlockGraph(ham, ham_data, prop, trial, wave, pd, n_prop_steps=S, external_fields=True)
            bg.fields.copy_(host_fields)
            bg.capture(warmup=1)
            runner = HostFieldBlocks(bg)
            runner.upload(host_fields)
            runner.run(host_fields)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                runner.run(host_fields)
            torch.cuda.synchronize()
            t_e2e = time.perf_counter() - t0
            out_numel = runner.out_host.numel()
        else:
            smp_e2e = sampling.sampler(n_prop_steps=S, n_ene_blocks=1, n_sr_blocks=1,
                                       field_source=PinnedSource())
            out_host = torch.empty(W + 1, dtype=torch.float64).pin_memory()

            def e2e_block(pd):
                e, pd = smp_e2e.propagate_phaseless(ham, ham_data, prop, pd, trial, wave)
                out_host[0].copy_(e, non_blocking=True)
                out_host[1:].copy_(pd["weights"], non_blocking=True)
                torch.cuda.current_stream().synchronize()
                pd["e_estimate"] = 0.9 * pd["e_estimate"] + 0.1 * e
                return pd

            pd = e2e_block(pd)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                pd = e2e_block(pd)
            torch.cuda.synchronize()
            t_e2e = time.perf_counter() - t0
            out_numel = out_host.numel()
        if world > 1:
            t = torch.tensor([t_e2e], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": world * W * S * args.steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": int(host_fields.numel() * 8),
               "d2h_bytes_per_step": int(out_numel * 8)}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    # ---- roofline of the dominant kernel ------------------------------------
    N, G = sys_.norb, sys_.nchol
    avg_ms = kern_ms / max(kern_n, 1)
    products = {"fp64": 1, "mixed": 3, "mixed_hi": 6}[args.precision]
    if args.precision == "fp64":
        fp64_peak = measure_fp64_peak()
        # the FP64 VHS GEMM, tensor-bound: C(2W x N^2) = Xt(2W x G) L(G x N^2)
        flops_per_launch = 4.0 * W * N * N * G
        achieved = flops_per_launch / (avg_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "kernel": "vhs_gemm_kernel (FP64 DMMA)", "achieved": achieved,
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                "peak_source": "measured in this run (cuBLAS DGEMM 8192^3)", "traffic": None,
                "launches": kern_n, "avg_launch_ms": avg_ms, "flops_per_launch": flops_per_launch}
    else:
        # the propagator GEMMs (7 launches per step, the largest share of a block), HBM-bound:
        # algorithmic bytes of one step per spin sector s (nc = 2 No_s, npc bf16 pieces):
        #   5 Taylor terms in Horner form: VHS pieces W N 2N, iterate pieces W nc 2N, FP32 y read
        #     from the accumulator (W nc N); next iterate pieces W nc 2N, except the last term,
        #     which writes the finished sum to the accumulator and its pieces (N columns)
        #   2 one-body half-steps: (e^{-dt h/2} - I) pieces N N, walker/sum pieces W nc N,
        #     accumulator read (+ written by the first), next pieces W nc 2N / walker W N nc
        #     doubles out (the second)
        npc = 2 if args.precision == "mixed" else 3
        nsec = 1 if sys_.trial == "rhf" else 2
        step_bytes = 0.0
        for s_ in range(nsec):
            nc = 2 * sys_.nelec[s_]
            bf = 2.0 * npc
            taylor = (W * N * 2 * N * bf + W * nc * 2 * N * bf + W * nc * N * 4.0)
            step_bytes += 5 * taylor + 4 * W * nc * 2 * N * bf + W * nc * N * (bf + 4.0)
            step_bytes += 2 * (N * N * bf + W * nc * N * bf)           # the two half-steps' operands
            step_bytes += 2 * W * nc * N * 4.0 + W * nc * 2 * N * bf   # first half-step: acc r/w, pieces
            step_bytes += W * nc * N * 4.0 + W * N * nc * 8.0          # second: acc read, walker out
        bytes_per_launch = step_bytes / 7.0
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
        pk, src = measured_peaks()
        roof = {"bound": "hbm", "kernel": f"umma_gemm_kernel<PropEpiU> (tcgen05 BF16x{products}, "
                                           "Taylor terms and one-body half-steps)",
                "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": src + " HBM copy",
                "traffic": PROP_DRAM_BYTES_PER_LAUNCH if W == 512 and args.config == CONFIG else None,
                "launches": kern_n, "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                "note": "average over the 7 launches of a step; traffic = ncu dram bytes read+written "
                        "per launch on this workload (the VHS pieces, 164 MB, are read by each of the "
                        "5 Taylor launches)"}

    cpu = None
    if not args.no_cpu:
        v, t = cpu_oracle_sample(sys_, args.cpu_walkers, S, dt)
        cpu = {"value": v, "unit": UNIT, "cores": blas_threads(), "kind": "port",
               "sample": f"{args.cpu_walkers} walkers x {S} steps + 1 block end, NumPy oracle "
                         f"(BLAS on all host threads), {t:.1f} s"}
        # one thread, as the reference runs one thread per MPI rank (config.py:102-104)
        try:
            from threadpoolctl import threadpool_limits

            with threadpool_limits(limits=1):
                nw1 = max(4, args.cpu_walkers // 4)
                v1, t1 = cpu_oracle_sample(sys_, nw1, S, dt)
            cpu["single_thread"] = {"value": v1, "unit": UNIT, "cores": 1,
                                    "sample": f"{nw1} walkers x {S} steps + 1 block end, {t1:.1f} s"}
        except Exception as exc:  # threadpoolctl missing: report why
            cpu["single_thread"] = {"unavailable": str(exc)}

    # ---- the other workloads: N=10 RHF and N=300 UHF, FP64 and mixed ------------
    configs = None
    if not args.no_configs and world == 1 and args.precision != "fp64":
        configs = {}
        for name, steps, nb in (("h10_sto6g_synthetic", max(3, args.steps), 5),
                                ("uhf_n300_g1500", max(2, args.steps // 5), 3)):
            try:
                configs[name] = measure_config(name, args.precision, steps, 2, nb)
            except Exception as exc:  # keep the headline line even if one leg fails
                configs[name] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()

    # ---- fragments: the uneven batch and the serving loop ----------------------
    fragments = None
    if not args.no_serving and world == 1 and args.precision != "fp64":
        fragments = {}
        try:
            from ad_afqmc_b200 import batching

            fragments["batch"] = batching.bench(64, args.precision, reps=2)
        except Exception as exc:
            fragments["batch"] = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()
        try:
            from ad_afqmc_b200 import serving

            fragments["serving"] = serving.bench(rate=20.0, duration=args.serving_duration,
                                                 precision=args.precision)
            fragments["setup"] = serving.setup_latency(args.precision)
        except Exception as exc:
            fragments["serving"] = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": {"fp64": "f64", "mixed": "bf16x3+f32acc/f64", "mixed_hi": "bf16x6+f32acc/f64"}[args.precision],
           "data": "synthetic",
           "config": {"workload": args.config, "norb": N, "nelec": list(sys_.nelec), "nchol": G,
                      "n_walkers_per_gpu": W, "n_prop_steps_per_bench_step": S, "dt": dt,
                      "precision": args.precision,
                      "parallelism": (f"dp{world}: walkers sharded by rank, block energy all-reduced, "
                                      "reconfiguration across ranks every block") if world > 1 else "1 GPU",
                      "l2": "working set (VHS 328 MB, chol 320 MB) exceeds the 126 MB L2",
                      "chol_scale": args.chol_scale, "killed_walker_fraction": killed,
                      "launch": "eager" if args.eager else "cuda_graph_per_block"},
           "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
           "clocks": clocks, "compare": compare, "configs": configs, "fragments": fragments}
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
