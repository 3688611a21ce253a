"""Run set-up from files on disk (launch_script.py:60-94, :100-200, :213-260,
:262-420, :644-711, :713-770 and run_afqmc.run_afqmc, run_afqmc.py:16-100).

A calculation directory holds ``FCIDUMP_chol`` (the Hamiltonian, written by
``pyscf_interface.write_dqmc`` or ``fcidump.write_fcidump``) and
``mo_coeff.npz`` (the trial orbitals in the same basis).  ``setup_afqmc``
reads both, fills in the option defaults and builds this package's
hamiltonian, trial, propagator and sampler objects; ``run_afqmc`` then runs
the energy driver on one GPU and returns (energy, error) like the
reference's ``run_afqmc`` (which runs the same steps under mpirun).

Options that select code outside the phaseless walker path (AD modes,
symmetry projectors, CISD/GHF/NOCI trials, generalized walkers) raise an
error instead of being ignored.
"""

from __future__ import annotations

import os
from typing import Dict, Optional, Tuple

import numpy as np

from . import driver, hamiltonian, propagation, sampling, wavefunctions
from .fcidump import read_fcidump, read_mo_coeff

_TRIALS = ("rhf", "uhf")


def read_options(options: Optional[Dict] = None, tmp_dir: Optional[str] = None) -> Dict:
    """Option defaults of launch_script.read_options (launch_script.py:100-200)
    for what the phaseless walker path uses.  ``precision`` ("fp64" or
    "mixed") selects this package's arithmetic; the reference's
    ``vhs_mixed_precision`` maps to "mixed".  With ``options`` None the
    pickled ``options.bin`` of the directory is read, as there."""
    if options is None:
        path = os.path.join(tmp_dir or ".", "options.bin")
        options = {}
        if os.path.isfile(path):
            import pickle

            with open(path, "rb") as f:
                options = pickle.load(f)
    options = dict(options)
    options["dt"] = options.get("dt", 0.01)
    options["n_walkers"] = options.get("n_walkers", 50)
    options["n_prop_steps"] = options.get("n_prop_steps", 50)
    options["n_ene_blocks"] = options.get("n_ene_blocks", 50)
    options["n_sr_blocks"] = options.get("n_sr_blocks", 1)
    options["n_blocks"] = options.get("n_blocks", 50)
    options["n_ene_blocks_eql"] = options.get("n_ene_blocks_eql", 5)
    options["n_sr_blocks_eql"] = options.get("n_sr_blocks_eql", 10)
    options["seed"] = options.get("seed", int(np.random.randint(1, int(1e6))))
    options["n_eql"] = options.get("n_eql", 1)
    if options.get("ad_mode") is not None:
        raise ValueError(f"ad_mode={options['ad_mode']!r} is not part of the phaseless walker path")
    options["ad_mode"] = None
    wt = options.get("walker_type", "restricted")
    wt = {"rhf": "restricted", "uhf": "unrestricted"}.get(wt, wt)
    if wt not in ("restricted", "unrestricted"):
        raise ValueError(f"walker_type={wt!r}: only restricted and unrestricted walkers are supported")
    options["walker_type"] = wt
    if options.get("symmetry_projector") is not None:
        raise ValueError("symmetry projectors are not supported")
    trial = options.get("trial", None)
    if trial is None:
        trial = "rhf" if wt == "restricted" else "uhf"
    if trial not in _TRIALS:
        raise ValueError(f"trial={trial!r}: supported trials are {_TRIALS}")
    options["trial"] = trial
    options["ene0"] = options.get("ene0", 0.0)
    options["free_projection"] = options.get("free_projection", False)
    options["n_chunks"] = options.get("n_chunks", options.get("n_batch", 1))
    mixed = options.get("vhs_mixed_precision", False)
    options["precision"] = options.get("precision", "mixed" if mixed else "fp64")
    if options["precision"] not in ("fp64", "mixed"):
        raise ValueError(f"precision={options['precision']!r}")
    options["prjlo"] = options.get("prjlo", None)
    options["save_walkers"] = options.get("save_walkers", False)
    options["metrics_file"] = options.get("metrics_file", None)
    options["maxError"] = options.get("maxError", 1e-3)
    return options


def set_ham(norb: int, h0, h1, chol, ene0: float = 0.0) -> Tuple[hamiltonian.hamiltonian, Dict]:
    """launch_script.set_ham (launch_script.py:213-260): h1 replicated per
    spin, chol flattened to (nchol, norb*norb)."""
    ham = hamiltonian.hamiltonian(norb)
    chol = np.asarray(chol, dtype=np.float64)
    h1 = np.asarray(h1, dtype=np.float64)
    ham_data = {"h0": float(np.asarray(h0)), "h1": np.array([h1, h1]),
                "chol": chol.reshape(chol.shape[0], -1), "ene0": float(ene0)}
    return ham, ham_data


def set_trial(options: Dict, mo_coeff, norb: int, nelec_sp: Tuple[int, int]):
    """launch_script.set_trial (launch_script.py:262-420, :636-640) for the
    rhf and uhf trials: the occupied columns of mo_coeff, rdm1 from them.
    With ``prjlo`` the trial is rhf_lno on the alpha orbitals, whatever
    ``trial`` says, as there."""
    mo_coeff = np.asarray(mo_coeff, dtype=np.float64)
    mos = [np.ascontiguousarray(mo_coeff[0][:, :nelec_sp[0]]),
           np.ascontiguousarray(mo_coeff[1][:, :nelec_sp[1]])]
    wave_data = {"rdm1": np.array([m @ m.T for m in mos])}
    if options.get("prjlo") is not None:
        trial = wavefunctions.rhf_lno(norb, nelec_sp, n_chunks=options["n_chunks"])
        wave_data["mo_coeff"] = mos[0]
        wave_data["prjlo"] = np.asarray(options["prjlo"], dtype=np.float64)
    elif options["trial"] == "rhf":
        trial = wavefunctions.rhf(norb, nelec_sp, n_chunks=options["n_chunks"],
                                  projector=options.get("symmetry_projector"))
        wave_data["mo_coeff"] = mos[0]
    else:
        trial = wavefunctions.uhf(norb, nelec_sp, n_chunks=options["n_chunks"],
                                  projector=options.get("symmetry_projector"))
        wave_data["mo_coeff"] = mos
    return trial, wave_data


def set_prop(options: Dict) -> propagation.propagator_afqmc:
    """launch_script.set_prop (launch_script.py:644-667): 10 Taylor terms for
    free projection, else ``n_exp_terms`` (6)."""
    n_exp_terms = 10 if options["free_projection"] else options.get("n_exp_terms", 6)
    return propagation.propagator_afqmc(options["dt"], options["n_walkers"], n_exp_terms=n_exp_terms,
                                        n_chunks=options["n_chunks"], walker_type=options["walker_type"],
                                        precision=options["precision"])


def set_sampler(options: Dict) -> sampling.sampler:
    """launch_script.set_sampler (launch_script.py:670-694)."""
    cls = sampling.sampler_lno if options.get("prjlo") is not None else sampling.sampler
    return cls(options["n_prop_steps"], options["n_ene_blocks"], options["n_sr_blocks"], options["n_blocks"])


def setup_afqmc(options: Optional[Dict] = None, tmp_dir: Optional[str] = None):
    """launch_script.setup_afqmc (launch_script.py:713-770): (ham_data, ham,
    prop, trial, wave_data, sampler, options)."""
    directory = tmp_dir if tmp_dir is not None else "."
    h0, h1, chol, norb, nelec_sp = read_fcidump(directory)
    options = read_options(options, directory)
    ham, ham_data = set_ham(norb, h0, h1, chol, options["ene0"])
    trial, wave_data = set_trial(options, read_mo_coeff(directory), norb, nelec_sp)
    return ham_data, ham, set_prop(options), trial, wave_data, set_sampler(options), options


def run_afqmc(options: Optional[Dict] = None, script=None, mpi_prefix=None, nproc: Optional[int] = None,
              tmpdir: Optional[str] = None) -> Tuple[float, float]:
    """run_afqmc.run_afqmc (run_afqmc.py:16-100) on one GPU in this process:
    reads the calculation directory and returns (energy, error) of the
    phaseless energy driver (the LNO driver when ``prjlo`` is given).
    ``script`` and ``mpi_prefix`` are accepted for signature compatibility;
    ``nproc`` other than 1 raises (several GPUs run one process each under
    torch.distributed)."""
    if nproc not in (None, 1):
        raise ValueError("run_afqmc runs one process; launch one process per GPU for several GPUs")
    directory = tmpdir if tmpdir is not None else "."
    ham_data, ham, prop, trial, wave_data, smp, options = setup_afqmc(options, directory)
    if options["free_projection"]:
        raise ValueError("free projection runs through sampler.propagate_free, not the energy driver")
    if options.get("prjlo") is not None:
        return driver.afqmc_LNOenergy(ham_data, ham, prop, trial, wave_data, smp, options, tmpdir=directory)
    return driver.afqmc_energy(ham_data, ham, prop, trial, wave_data, smp, options, tmpdir=directory)
