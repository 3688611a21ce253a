"""Energy driver loop (mirror of ad_afqmc/driver.py:24-192 and :653-715, one rank).

The control flow of ``afqmc_energy`` is kept: intermediates, initial
propagation data, equilibration with a 50-step sampler, then ``n_blocks``
calls of ``sampler.propagate_phaseless`` each followed by QR, the driver's
(global-formula) reconfiguration and the e_estimate update.  Block energies
stay FP64 (the reference casts to float32 for MPI at driver.py:138-139).
The statistics (outlier rejection + blocking analysis) are host NumPy on the
per-block scalars, as in stat_utils.py.
"""

from __future__ import annotations

import json
import pickle
import time
import warnings
from typing import Optional, Tuple

import numpy as np
import torch

from . import stat_utils
from .sampling import sampler as sampler_cls


def _run_equilibration(ham, ham_data, prop, prop_data, trial, wave_data, sampler_eq,
                       field_source=None):
    """driver.py:653-715 (single rank)."""
    for _ in range(sampler_eq.n_blocks):
        e, prop_data = sampler_eq.propagate_phaseless(ham, ham_data, prop, prop_data, trial, wave_data)
        prop_data["walkers"] = prop_data["walkers"].orthonormalize()
        zeta = field_source.uniform() if field_source is not None else prop_data["key"].uniform()
        prop_data["walkers"], prop_data["weights"] = prop_data["walkers"].stochastic_reconfiguration_global(
            prop_data["weights"], zeta)
        prop_data["e_estimate"] = 0.9 * prop_data["e_estimate"] + 0.1 * e
    return prop_data


def _host_prop_data(prop_data: dict) -> dict:
    """A host copy of prop_data (walkers, weights, overlaps, scalars as NumPy,
    the counter-based key as (seed, counter)) for pickling."""
    out = {}
    for k, v in prop_data.items():
        if k.startswith("_"):
            continue
        if k == "walkers":
            d = v.data
            out[k] = [t.cpu().numpy() for t in d] if isinstance(d, list) else d.cpu().numpy()
        elif isinstance(v, torch.Tensor):
            out[k] = v.detach().cpu().numpy()
        elif k == "key":
            out[k] = (v.seed, v.counter)
        else:
            out[k] = v
    return out


def save_walkers(prop_data: dict, n: int, tmpdir: str, rank: int = 0) -> None:
    """driver._save_walkers (driver.py:985-992): the walker state after block
    n pickled to ``tmpdir/prop_data_<rank>.bin`` (appended after block 0),
    copied from the device once per block."""
    mode = "ab" if n > 0 else "wb"
    with open(f"{tmpdir}/prop_data_{rank}.bin", mode) as f:
        pickle.dump(_host_prop_data(prop_data), f)


def write_metrics(path: str, energies: np.ndarray, weights: np.ndarray, seconds: float, **extra) -> None:
    """One JSON line per block (energy, weight) and a closing summary line."""
    with open(path, "w") as f:
        for n, (e, w) in enumerate(zip(energies, weights)):
            f.write(json.dumps({"block": n, "energy": float(e), "weight": float(w)}) + "\n")
        f.write(json.dumps({"blocks": int(len(energies)), "seconds": float(seconds), **extra}) + "\n")


def _warn_nonfinite(e: np.ndarray, w: np.ndarray) -> None:
    """Block energies or weights that are not finite (a population whose
    weights all went to zero gives 0/0) pass through the analysis as in the
    reference; say so instead of failing silently."""
    bad = ~(np.isfinite(e) & np.isfinite(w))
    if bad.any():
        warnings.warn(f"{int(bad.sum())} of {len(e)} blocks have non-finite energy or weight "
                      f"(first at block {int(np.argmax(bad))}); the population may have collapsed",
                      RuntimeWarning, stacklevel=3)


def afqmc_blocks(ham, ham_data, prop, prop_data, trial, wave_data, smp, n_blocks,
                 field_source=None, save: bool = False, tmpdir: str = "."):
    """Sampling loop of driver.py:133-168 on one rank; returns (energies, weights, prop_data).
    ``save``: the reference's ``save_walkers`` option (driver.py:160-161)."""
    energies = torch.zeros(n_blocks, dtype=torch.float64, device=prop_data["weights"].device)
    weights = torch.zeros_like(energies)
    for n in range(n_blocks):
        e, prop_data = smp.propagate_phaseless(ham, ham_data, prop, prop_data, trial, wave_data)
        energies[n] = e
        weights[n] = torch.sum(prop_data["weights"])
        prop_data["walkers"] = prop_data["walkers"].orthonormalize()
        if save:
            save_walkers(prop_data, n, tmpdir)
        zeta = field_source.uniform() if field_source is not None else prop_data["key"].uniform()
        prop_data["walkers"], prop_data["weights"] = prop_data["walkers"].stochastic_reconfiguration_global(
            prop_data["weights"], zeta)
        prop_data["e_estimate"] = 0.9 * prop_data["e_estimate"] + 0.1 * e
    return energies, weights, prop_data


def afqmc_energy(ham_data: dict, ham, propagator, trial, wave_data: dict, sampler, options: dict,
                 MPI=None, init_walkers=None, tmpdir: str = ".") -> Tuple[float, float]:
    """driver.py:24-192 on one GPU (no MPI ranks)."""
    if "rdm1" not in wave_data:
        wave_data["rdm1"] = trial.get_rdm1(wave_data)
    ham_data = ham.build_measurement_intermediates(ham_data, trial, wave_data)
    ham_data = ham.build_propagation_intermediates(ham_data, propagator, trial, wave_data)
    prop_data = propagator.init_prop_data(trial, wave_data, ham_data, options.get("seed", 0),
                                          init_walkers)
    if float(torch.abs(torch.sum(prop_data["overlaps"]))) < 1.0e-6:
        raise ValueError("Initial overlaps are zero. Pass walkers with non-zero overlap.")
    sampler_eq = sampler_cls(n_prop_steps=50, n_ene_blocks=options.get("n_ene_blocks_eql", 1),
                             n_sr_blocks=options.get("n_sr_blocks_eql", 5),
                             n_blocks=options.get("n_eql", 1))
    prop_data = _run_equilibration(ham, ham_data, propagator, prop_data, trial, wave_data, sampler_eq)
    t0 = time.perf_counter()
    energies, weights, prop_data = afqmc_blocks(ham, ham_data, propagator, prop_data, trial, wave_data,
                                                sampler, sampler.n_blocks,
                                                save=bool(options.get("save_walkers", False)), tmpdir=tmpdir)
    e = energies.cpu().numpy()
    w = weights.cpu().numpy()
    _warn_nonfinite(e, w)
    np.savetxt(tmpdir + "/samples_raw.dat", np.stack((w, e)).T)
    if options.get("metrics_file"):
        write_metrics(options["metrics_file"], e, w, time.perf_counter() - t0,
                      walkers=int(propagator.n_walkers), steps_per_block=int(sampler.n_prop_steps))
    clean, _ = stat_utils.reject_outliers(np.stack((w, e)).T, 1)
    return stat_utils.blocking_analysis(clean[:, 0], clean[:, 1], neql=0)


def afqmc_LNOenergy(ham_data: dict, ham, propagator, trial, wave_data: dict, sampler, options: dict,
                    MPI=None, init_walkers=None, tmpdir: str = ".",
                    results: Optional[dict] = None) -> Tuple[float, float]:
    """driver.afqmc_LNOenergy, driver.py:195-402, on one GPU: equilibration,
    sampling blocks of a sampler_lno (energy and orbital energy per block),
    stop when the orbital energy's standard error of the mean drops below
    options["maxError"] (checked every max(n_blocks // 5, 1) blocks after the
    fifth, driver.py:376-389), then the analysis of driver.py:1338-1400.
    Returns (E, E_err) as the reference; ``results`` (optional dict) also
    receives the orbital energy, its error and the block data."""
    if "rdm1" not in wave_data:
        wave_data["rdm1"] = trial.get_rdm1(wave_data)
    ham_data = ham.build_measurement_intermediates(ham_data, trial, wave_data)
    ham_data = ham.build_propagation_intermediates(ham_data, propagator, trial, wave_data)
    prop_data = propagator.init_prop_data(trial, wave_data, ham_data, options.get("seed", 0),
                                          init_walkers)
    if float(torch.abs(torch.sum(prop_data["overlaps"]))) < 1.0e-6:
        raise ValueError("Initial overlaps are zero. Pass walkers with non-zero overlap.")
    sampler_eq = sampler_cls(n_prop_steps=50, n_ene_blocks=options.get("n_ene_blocks_eql", 1),
                             n_sr_blocks=options.get("n_sr_blocks_eql", 5),
                             n_blocks=options.get("n_eql", 1))
    prop_data = _run_equilibration(ham, ham_data, propagator, prop_data, trial, wave_data, sampler_eq)
    max_error = options["maxError"]
    nb = sampler.n_blocks
    energies, weights, orbes = [], [], []
    truncate_at = nb
    for n in range(nb):
        e, prop_data, o = sampler.propagate_phaseless(ham, ham_data, propagator, prop_data, trial, wave_data)
        energies.append(float(e))
        weights.append(float(torch.sum(prop_data["weights"])))
        orbes.append(float(o))
        prop_data["walkers"] = prop_data["walkers"].orthonormalize()
        if options.get("save_walkers", False):
            save_walkers(prop_data, n, tmpdir)
        zeta = prop_data["key"].uniform()
        prop_data["walkers"], prop_data["weights"] = prop_data["walkers"].stochastic_reconfiguration_global(
            prop_data["weights"], zeta)
        prop_data["e_estimate"] = 0.9 * prop_data["e_estimate"] + 0.1 * e
        if n % max(nb // 5, 1) == 0 and n > 4:
            sem = np.std(orbes[: n + 1]) / np.sqrt(n + 1)
            if sem < max_error:
                truncate_at = n
                break
    w = np.array(weights[: truncate_at + 1])
    e = np.array(energies[: truncate_at + 1])
    o = np.array(orbes[: truncate_at + 1])
    _warn_nonfinite(e, w)
    np.savetxt(tmpdir + "/samples_raw.dat", np.stack((w, e)).T)
    clean, _ = stat_utils.reject_outliers(np.stack((w, e)).T, 1)
    e_afqmc, e_err = stat_utils.blocking_analysis(clean[:, 0], clean[:, 1], neql=0)
    orbe, orbe_err = stat_utils.blocking_analysis(w, o, neql=0)
    if results is not None:
        results.update({"orbE": orbe, "orbE_err": orbe_err if orbe_err is not None else 0.0,
                        "block_energies": e, "block_weights": w, "block_orbEs": o,
                        "n_blocks": len(e)})
    return e_afqmc, e_err
