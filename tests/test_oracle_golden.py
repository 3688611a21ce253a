"""Pin the NumPy oracle against the reference's golden values.

The inputs reproduce the seeded fixture of the reference test-suite
(tests/test_wavefunctions.py:12-86); the expected numbers are the values that
suite asserts (tests/test_wavefunctions.py:128-184).  The reference's own
tolerance is ``np.allclose`` defaults (rtol 1e-5); the oracle is held to 1e-12.
"""

import json
import os

import numpy as np
import pytest

from oracle import afqmc_oracle as orc

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
G = np.load(os.path.join(HERE, "trial_golden.npz"))
REF = {k: v[0] for k, v in json.load(open(os.path.join(HERE, "trial_golden.json"))).items()}
RTOL = 1e-12


def _rhf():
    trial = orc.RHFTrial(10, (5, 5))
    wave = {"mo_coeff": G["mo_coeff"]}
    ham = {"h0": float(G["h0"]), "rot_h1": G["rot_h1"], "rot_chol": G["rot_chol"]}
    return trial, wave, ham


def _uhf():
    trial = orc.UHFTrial(10, (3, 2))
    wave = {"mo_coeff": [G["mo_u0"], G["mo_u1"]]}
    ham = {
        "h0": float(G["h0"]),
        "rot_h1": [G["rot_h1"][:3], G["rot_h1"][:2]],
        "rot_chol": [G["rot_chol"][:, :3], G["rot_chol"][:, :2]],
    }
    return trial, wave, ham


def test_rhf_golden():
    trial, wave, ham = _rhf()
    w = G["walker"]
    assert np.isclose(trial.overlap_restricted(w, wave).real, REF["rhf_overlap_real"], rtol=RTOL, atol=0)
    assert np.isclose(orc.green(w, wave["mo_coeff"]).sum().real, REF["rhf_green_sum_real"], rtol=RTOL, atol=0)
    assert np.isclose(trial.force_bias_restricted(w, ham, wave).sum().real, REF["rhf_force_bias_sum_real"], rtol=RTOL, atol=0)
    assert np.isclose(trial.energy_restricted(w, ham, wave).real, REF["rhf_energy_real"], rtol=RTOL, atol=0)


def test_uhf_golden():
    trial, wave, ham = _uhf()
    wu, wd = G["walker_up"], G["walker_dn"]
    assert np.isclose(trial.overlap_unrestricted(wu, wd, wave).real, REF["uhf_overlap_real"], rtol=RTOL, atol=0)
    gu, gd = trial.greens(wu, wd, wave)
    assert np.isclose((gu.sum() + gd.sum()).real, REF["uhf_green_sum_real"], rtol=RTOL, atol=0)
    assert np.isclose(trial.force_bias_unrestricted(wu, wd, ham, wave).sum().real, REF["uhf_force_bias_sum_real"], rtol=RTOL, atol=0)
    assert np.isclose(trial.energy_unrestricted(wu, wd, ham, wave).real, REF["uhf_energy_real"], rtol=RTOL, atol=0)


def test_oracle_planted_mistake_is_caught():
    """A planted error in the oracle (CPU side) must break the golden check."""
    trial, wave, ham = _rhf()
    bad = dict(ham)
    bad["rot_chol"] = ham["rot_chol"] * (1 + 1e-9)
    e = trial.energy_restricted(G["walker"], bad, wave).real
    assert not np.isclose(e, REF["rhf_energy_real"], rtol=RTOL, atol=0)
