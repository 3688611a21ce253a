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


# FP64 dense peak of this pool's B200 (cuBLAS DGEMM 8192^3, measured with
# CUDA events; the driver's peaks file carries no FP64 figure).
FP64_PEAK_TFLOPS = 35.47

# DRAM bytes (read + written) per propagator launch, mean over the 7 launches
# of one step, from ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the
# bench workload (N=200, No=40, G=1000, 512 walkers, mixed).
PROP_DRAM_BYTES_PER_LAUNCH = 257510875


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
        # same-shape system with a surviving population (Cholesky vectors x0.25):
        # identical walkers and device-drawn fields for both precisions
        from ad_afqmc_b200.synthetic import make_config as _mk
        sys_h, _ = _mk(args.config, chol_scale=0.25)
        nb = 3
        energies = {}
        for precision in (args.precision, "fp64"):
            hd, wv = sys_h.ham_data(), sys_h.wave_data()
            pr = propagation.propagator_afqmc(dt=dt, n_walkers=W, walker_type=wt, precision=precision)
            hd = ham.build_measurement_intermediates(hd, trial, wv)
            hd = ham.build_propagation_intermediates(hd, pr, trial, wv)
            pd_ = pr.init_prop_data(trial, wv, hd, seed=4242)
            smp_ = sampling.sampler(n_prop_steps=S, n_ene_blocks=1, n_sr_blocks=1)
            es = []
            for _ in range(nb):
                pd_, e = one_block(smp_, hd, wv, pr, pd_)
                es.append(float(e))
            # unclamped weighted local energy of the final walkers (stays meaningful
            # when the sqrt(2/dt) clamp pins the block energies to e_estimate)
            el = torch.real(trial.calc_energy(pd_["walkers"], hd, wv))
            wsum = torch.sum(pd_["weights"])
            e_unclamped = float(torch.sum(el * pd_["weights"]) / wsum) if float(wsum) > 0 else float("nan")
            clamped = float(torch.mean((torch.abs(el - pd_["e_estimate"]) > (2.0 / dt) ** 0.5).double()))
            energies[precision] = (es, float(pd_["n_killed_walkers"]), e_unclamped, clamped)
            del hd, pr, pd_
        err = max(abs(a - b) for a, b in zip(energies[args.precision][0], energies["fp64"][0]))
        compare = {"fp64_value": v64, "fp64_ms_per_step": ms64 / max(2, args.steps // 2),
                   "speedup_vs_fp64": value / v64,
                   "block_energy_error_ha": err,
                   "block_energy_check": f"{nb} blocks x {S} steps, {W} walkers, chol_scale 0.25, "
                                         "same walkers and fields, vs the FP64 GPU path (which "
                                         "matches the NumPy oracle to 1e-8 Ha)",
                   "block_energies_fp64": energies["fp64"][0],
                   "killed_fraction_check": energies[args.precision][1],
                   "unclamped_local_energy_error_ha": abs(energies[args.precision][2] - energies["fp64"][2]),
                   "clamped_fraction_check": energies["fp64"][3]}

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
        # the FP64 VHS GEMM, tensor-bound: C(2W x N^2) = Xt(2W x G) L(G x N^2)
        flops_per_launch = 4.0 * W * N * N * G
        achieved = flops_per_launch / (avg_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "kernel": "vhs_gemm_kernel (FP64 DMMA)", "achieved": achieved,
                "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": achieved / FP64_PEAK_TFLOPS,
                "peak_source": "measured (cuBLAS DGEMM on this pool)", "traffic": None,
                "launches": kern_n, "avg_launch_ms": avg_ms, "flops_per_launch": flops_per_launch}
    else:
        # the propagator GEMMs (7 launches per step, the largest share of a block), HBM-bound:
        # algorithmic bytes of one step per spin sector s (nc = 2 No_s, npc bf16 pieces):
        #   5 Taylor terms: VHS pieces W N 2N, iterate pieces W nc 2N, FP32 accumulator read and
        #     written (W nc N), next iterate pieces W nc 2N (the last term: N columns)
        #   2 one-body half-steps: (e^{-dt h/2} - I) pieces N N, walker/sum pieces W nc N,
        #     accumulator read (+ written by the first), next pieces W nc 2N / walker W N nc
        #     doubles out (the second)
        npc = 2 if args.precision == "mixed" else 3
        nsec = 1 if sys_.trial == "rhf" else 2
        step_bytes = 0.0
        for s_ in range(nsec):
            nc = 2 * sys_.nelec[s_]
            bf = 2.0 * npc
            taylor = (W * N * 2 * N * bf + W * nc * 2 * N * bf + 2 * W * nc * N * 4.0)
            step_bytes += 5 * taylor + 4 * W * nc * 2 * N * bf + W * nc * N * bf
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
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"{args.cpu_walkers} walkers x {S} steps + 1 block end, NumPy oracle, "
                         f"{t:.1f} s"}

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
           "clocks": clocks, "compare": compare}
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
