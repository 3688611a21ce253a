"""Oracle parity at the benchmark workloads' full walker counts, so that the
tile schedules of the timed runs (512 walkers at N = 200, 1024 at N = 300) are
the ones compared: one phaseless step of every walker in FP64 and in mixed
precision (at N = 300 the oracle steps 128 walkers spread over the 1024), the
QR of the stepped walkers, and the local energies of the N = 200 population
(all 512 evaluated in one launch, a spread of 48 of them checked, the
oracle's energy being the slow part).  The Cholesky vectors are
scaled to 0.1 so that the phaseless clamps stay inactive: the arithmetic is
compared, not the clamp."""

import copy

import numpy as np
import pytest

from ad_afqmc_b200.synthetic import make_config
from oracle import afqmc_oracle as orc
from tests._helpers import device_system, near_trial_walkers, oracle_system, rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-4}


def _np(t):
    return t.detach().cpu().numpy()


def _dev(w):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    return UHFWalkers([w[0].copy(), w[1].copy()]) if isinstance(w, list) else RHFWalkers(w.copy())


def _case(name, n_oracle=None):
    """The device steps all W walkers; the oracle steps every walker, or
    n_oracle of them spread over the population (the walkers of a step are
    independent given the fields and the energy shift)."""
    sys_, cfg = make_config(name, chol_scale=0.1)
    W, dt = cfg["n_walkers"], cfg["dt"]
    wt = "restricted" if sys_.trial == "rhf" else "unrestricted"
    rng = np.random.default_rng(17)
    if wt == "restricted":
        walkers = near_trial_walkers(rng, sys_.mo_coeff, W, eps=0.05)
    else:
        walkers = [near_trial_walkers(rng, sys_.mo_coeff[s], W, eps=0.05) for s in range(2)]
    fields = rng.standard_normal((W, sys_.nchol))
    # the population's mean local energy from the device (the oracle's energy of
    # 1024 walkers at N = 300 takes many minutes); both sides start from it
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, wt, dt, W, precision="fp64")
    e0 = float(d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(walkers))["e_estimate"])
    pick = np.arange(W) if n_oracle is None else np.linspace(0, W - 1, n_oracle).astype(int)
    sub = walkers[pick] if wt == "restricted" else [w[pick] for w in walkers]
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, dt)
    o_ham["e_estimate"] = e0
    o_prop.n_walkers = len(pick)
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(sub))
    o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields[pick], o_wave)
    return dict(sys=sys_, W=W, dt=dt, wt=wt, walkers=walkers, fields=fields, o_pd=o_pd, e0=e0,
                pick=pick, o_trial=o_trial, o_ham=o_ham, o_wave=o_wave)


@pytest.fixture(scope="module")
def rhf_case():
    return _case("rhf_n200_g1000")


@pytest.fixture(scope="module")
def uhf_case():
    return _case("uhf_n300_g1500", n_oracle=128)


def _device_step(c, precision):
    d_trial, d_ham, d_wave, d_prop, _ = device_system(c["sys"], c["wt"], c["dt"], c["W"], precision=precision)
    d_ham["e_estimate"] = c["e0"]
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(c["walkers"]))
    d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, c["fields"], d_wave)
    return d_trial, d_ham, d_wave, d_pd


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rhf_step_all_512_walkers(rhf_case, precision):
    c = rhf_case
    d_trial, d_ham, d_wave, d_pd = _device_step(c, precision)
    o_pd = c["o_pd"]
    assert rel_err(_np(d_pd["walkers"].data), o_pd["walkers"]) < TOL[precision]
    assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=10 * TOL[precision], atol=1e-8)
    assert rel_err(_np(d_pd["overlaps"]), o_pd["overlaps"]) < 10 * TOL[precision]
    # QR of all 512 stepped walkers against LAPACK on the oracle's walkers
    q_ref, _ = orc.qr_restricted(o_pd["walkers"])
    q = _np(d_pd["walkers"].orthonormalize().data)
    assert rel_err(q, q_ref) < (1e-10 if precision == "fp64" else 1e-4)
    if precision == "fp64":
        # local energies: all 512 in one launch, 48 of them against the oracle
        e = _np(d_trial.calc_energy(d_pd["walkers"], d_ham, d_wave))
        pick = np.linspace(0, c["W"] - 1, 48).astype(int)
        e_o = c["o_trial"].calc_energy(q_ref[pick], c["o_ham"], c["o_wave"])
        assert np.max(np.abs(e[pick] - e_o)) < 1e-9 * max(1.0, np.max(np.abs(e_o)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uhf_step_all_1024_walkers(uhf_case, precision):
    c = uhf_case
    d_trial, d_ham, d_wave, d_pd = _device_step(c, precision)
    o_pd = c["o_pd"]
    pick = c["pick"]
    for s in range(2):
        assert rel_err(_np(d_pd["walkers"].data[s])[pick], o_pd["walkers"][s]) < TOL[precision]
    assert np.allclose(_np(d_pd["weights"])[pick], o_pd["weights"], rtol=10 * TOL[precision], atol=1e-8)
