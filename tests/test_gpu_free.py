"""Free projection (propagator.propagate_free, propagation.py:338-376, and
sampler.propagate_free, sampling.py:96-144 / 367-384) against the oracle on
the same fields and uniforms."""

import copy

import numpy as np
import pytest
import torch

from ad_afqmc_b200.synthetic import make_system
from oracle import afqmc_oracle as orc
from tests._helpers import ListSource, device_system, near_trial_walkers, oracle_system, rel_err

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


CASES = [(24, (6, 6), 96, "rhf", "restricted", 8), (30, (8, 6), 120, "uhf", "unrestricted", 6)]


def _walkers(sys_, W, wt, seed):
    rng = np.random.default_rng(seed)
    if wt == "restricted":
        return near_trial_walkers(rng, sys_.mo_coeff, W, eps=0.1)
    mo = sys_.mo_coeff
    return [near_trial_walkers(rng, mo[0], W, eps=0.1), near_trial_walkers(rng, mo[1], W, eps=0.1)]


def _dev(w):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    return UHFWalkers([w[0].copy(), w[1].copy()]) if isinstance(w, list) else RHFWalkers(w.copy())


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
@pytest.mark.parametrize("case", CASES)
def test_free_step_matches_oracle(case, precision, tol):
    norb, nelec, nchol, tr, wt, W = case
    sys_ = make_system(norb, nelec, nchol, seed=21, trial=tr, chol_scale=0.25)
    walkers = _walkers(sys_, W, wt, 4)
    rng = np.random.default_rng(6)
    fields = [rng.standard_normal((W, nchol)) for _ in range(2)]
    zetas = [0.3, 0.8]
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, 0.005)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, wt, 0.005, W, precision=precision)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(walkers))
    d_prop._zeta_source = ListSource([], zetas)
    for f, z in zip(fields, zetas):
        o_pd = o_prop.propagate_free(o_trial, o_ham, o_pd, f, o_wave, z)
        d_pd = d_prop.propagate_free(d_trial, d_ham, d_pd, f, d_wave)
        if wt == "restricted":
            assert rel_err(_np(d_pd["walkers"].data), o_pd["walkers"]) < tol
        else:
            for s in range(2):
                assert rel_err(_np(d_pd["walkers"].data[s]), o_pd["walkers"][s]) < tol
        assert rel_err(_np(d_pd["weights"]), o_pd["weights"]) < tol
        assert rel_err(_np(d_pd["overlaps"]), o_pd["overlaps"]) < tol
    d_prop._zeta_source = None


@pytest.mark.parametrize("case", CASES)
def test_free_projection_blocks_match_oracle(case):
    from ad_afqmc_b200 import sampling

    norb, nelec, nchol, tr, wt, W = case
    sys_ = make_system(norb, nelec, nchol, seed=22, trial=tr, chol_scale=0.25)
    walkers = _walkers(sys_, W, wt, 5)
    S, nb = 3, 2
    rng = np.random.default_rng(8)
    fields = [rng.standard_normal((S, W, nchol)) for _ in range(nb)]
    uni = list(rng.random(S * nb))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, 0.005)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    ov_o, aov_o, be_o, bw_o = orc.sampler_propagate_free(orc.Sampler(S, 1, 1, nb), o_prop, o_trial, o_ham,
                                                         o_pd, o_wave, ListSource(fields, uni))
    d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, wt, 0.005, W)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(walkers))
    smp = sampling.sampler(S, 1, 1, nb, field_source=ListSource(fields, uni))
    ov, aov, states, be, bw, _ = smp.propagate_free(ham, d_ham, d_prop, d_pd, d_trial, d_wave)
    assert rel_err(_np(ov), ov_o) < 1e-10
    assert rel_err(_np(aov), aov_o) < 1e-10
    assert np.max(np.abs(_np(be) - be_o)) < 1e-8
    assert rel_err(_np(bw), bw_o) < 1e-10
    assert len(states) == nb
