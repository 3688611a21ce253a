"""Shared set-up for the parity tests: one synthetic system, seen by both the
NumPy oracle and the device path, with identical random inputs."""

from __future__ import annotations

import copy

import numpy as np

from ad_afqmc_b200.synthetic import make_system
from oracle import afqmc_oracle as orc


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def random_walkers(rng, W, N, nocc, walker_type):
    def one(no):
        return rng.standard_normal((W, N, no)) + 1j * rng.standard_normal((W, N, no))
    if walker_type == "restricted":
        return one(nocc[0])
    return [one(nocc[0]), one(nocc[1])]


def near_trial_walkers(rng, mo, W, eps=0.2):
    """Walkers close to the trial (well-conditioned overlaps)."""
    N, no = mo.shape
    out = mo[None, :, :] + eps * (rng.standard_normal((W, N, no)) + 1j * rng.standard_normal((W, N, no)))
    return out.astype(np.complex128)


def oracle_system(sys_, walker_type, dt):
    trial = orc.RHFTrial(sys_.norb, sys_.nelec) if sys_.trial == "rhf" else orc.UHFTrial(sys_.norb, sys_.nelec)
    ham = sys_.ham_data()
    wave = sys_.wave_data()
    prop = orc.Propagator(dt=dt, walker_type=walker_type)
    ham = trial.build_measurement_intermediates(ham, wave)
    ham = prop.build_propagation_intermediates(ham, trial, wave)
    return trial, ham, wave, prop


def device_system(sys_, walker_type, dt, n_walkers, precision="fp64", n_exp_terms=6):
    from ad_afqmc_b200 import hamiltonian, propagation, wavefunctions

    trial = (wavefunctions.rhf(sys_.norb, sys_.nelec) if sys_.trial == "rhf"
             else wavefunctions.uhf(sys_.norb, sys_.nelec))
    ham_data = sys_.ham_data()
    wave = sys_.wave_data()
    ham = hamiltonian.hamiltonian(sys_.norb)
    prop = propagation.propagator_afqmc(dt=dt, n_walkers=n_walkers, walker_type=walker_type,
                                        precision=precision, n_exp_terms=n_exp_terms)
    ham_data = ham.build_measurement_intermediates(ham_data, trial, wave)
    ham_data = ham.build_propagation_intermediates(ham_data, prop, trial, wave)
    return trial, ham_data, wave, prop, ham


class ListSource:
    """Feeds pre-drawn fields and uniforms in order (to oracle and device alike)."""

    def __init__(self, fields_list, uniforms):
        self.fields_list = list(fields_list)
        self.uniforms = list(uniforms)
        self.i = 0
        self.j = 0

    def fields(self, S, W, G):
        f = self.fields_list[self.i]
        assert f.shape == (S, W, G)
        self.i += 1
        return f

    def uniform(self):
        u = self.uniforms[self.j]
        self.j += 1
        return u
