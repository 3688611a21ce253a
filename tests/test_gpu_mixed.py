"""Mixed-precision (tcgen05, split-BF16) walker path against FP64.

Tolerances are the measured accuracy of the two-piece (BF16x3) and
three-piece (BF16x6) products with FP32 accumulation; every quantity that
decides walker survival (Green's functions, determinants, QR, weights) is
FP64 in both modes, so the differences come only from the contractions.
"""

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


def _walkers(sys_, W, seed, wt):
    rng = np.random.default_rng(seed)
    if wt == "restricted":
        mo = sys_.mo_coeff if sys_.trial == "rhf" else sys_.mo_coeff[0]
        return near_trial_walkers(rng, mo, W, eps=0.1)
    mo = sys_.mo_coeff if sys_.trial == "uhf" else [sys_.mo_coeff, sys_.mo_coeff]
    return [near_trial_walkers(rng, mo[0], W, eps=0.1), near_trial_walkers(rng, mo[1], W, eps=0.1)]


def _dev(w):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    return UHFWalkers([w[0].copy(), w[1].copy()]) if isinstance(w, list) else RHFWalkers(w.copy())


CASES = [
    (10, (5, 5), 50, "rhf", "restricted", 16),  # the N = 10 workload's shape
    (24, (6, 6), 96, "rhf", "restricted", 16),
    (64, (16, 16), 300, "rhf", "restricted", 40),
    (48, (13, 11), 200, "uhf", "unrestricted", 24),
    (200, (40, 40), 1000, "rhf", "restricted", 8),
    (80, (62, 62), 200, "rhf", "restricted", 4),
]
# BF16x6 is limited by FP32 accumulation over K (up to 8000 in the force bias)
TOL = {"mixed": 1e-4, "mixed_hi": 2e-5}


@pytest.mark.parametrize("precision", ["mixed", "mixed_hi"])
@pytest.mark.parametrize("case", CASES)
def test_mixed_measurements(case, precision):
    norb, nelec, nchol, tr, wt, W = case
    sys_ = make_system(norb, nelec, nchol, seed=11, trial=tr, chol_scale=0.25)
    walkers = _walkers(sys_, W, 3, wt)
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, wt, 0.005)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, wt, 0.005, W, precision=precision)
    eng = d_prop.engine(d_ham, d_trial, d_wave)
    # measurements through the engine of the requested precision
    import ctypes as C
    from ad_afqmc_b200 import _lib
    from ad_afqmc_b200.wavefunctions import _ptrs
    dw = _dev(walkers)
    fb = torch.empty(W, nchol, dtype=torch.complex128, device="cuda")
    p, w, wb = eng.handle
    _lib.check(_lib.lib().afq_calc_force_bias(C.byref(eng.dims), p, _ptrs(dw), fb.data_ptr(), w, wb,
                                              _lib.stream_handle()), "fb")
    e = torch.empty(W, dtype=torch.complex128, device="cuda")
    _lib.check(_lib.lib().afq_calc_energy(C.byref(eng.dims), p, _ptrs(dw), e.data_ptr(), w, wb,
                                          _lib.stream_handle()), "energy")
    fb_o = o_trial.calc_force_bias(walkers, o_ham, o_wave)
    e_o = o_trial.calc_energy(walkers, o_ham, o_wave)
    assert rel_err(_np(fb), fb_o) < TOL[precision]
    err_e = np.max(np.abs(_np(e) - e_o))
    scale = np.max(np.abs(e_o))
    assert err_e / scale < TOL[precision], (err_e, scale)


# two and three 128-row M tiles in the propagator (N = 200, N = 300 with UHF 60/58)
STEP_CASES = CASES[:4] + [(200, (40, 40), 1000, "rhf", "restricted", 4),
                          (300, (60, 58), 1500, "uhf", "unrestricted", 2)]


@pytest.mark.parametrize("precision", ["mixed", "mixed_hi"])
@pytest.mark.parametrize("case", STEP_CASES)
def test_mixed_step(case, precision):
    norb, nelec, nchol, tr, wt, W = case
    sys_ = make_system(norb, nelec, nchol, seed=12, trial=tr, chol_scale=0.25)
    walkers = _walkers(sys_, W, 4, wt)
    rng = np.random.default_rng(5)
    fields = rng.standard_normal((W, nchol))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, 0.005)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields, o_wave)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, wt, 0.005, W, precision=precision)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(walkers))
    d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, fields, d_wave)
    if wt == "restricted":
        pairs = [(_np(d_pd["walkers"].data), o_pd["walkers"])]
    else:
        pairs = [(_np(d_pd["walkers"].data[s]), o_pd["walkers"][s]) for s in range(2)]
    for d, o in pairs:
        assert rel_err(d, o) < TOL[precision]
    assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=10 * TOL[precision], atol=1e-6)


BLOCK_SHAPES = [
    # norb, nelec, nchol, trial, walkers, steps per block, blocks, Cholesky scale
    (64, (16, 16), 300, "rhf", 32, 5, 3, 0.25),
    (200, (40, 40), 1000, "rhf", 16, 3, 2, 0.1),
    # the N = 300 UHF workload's shape (Na/Nb = 60/58, G = 1500)
    (300, (60, 58), 1500, "uhf", 4, 2, 1, 0.1),
]


@pytest.mark.parametrize("precision", ["mixed", "mixed_hi"])
@pytest.mark.parametrize("shape", BLOCK_SHAPES)
def test_mixed_block_energy_error(precision, shape):
    """Block energies of the mixed path vs the FP64 oracle (same walkers,
    fields and uniforms), within 0.1 mHa, in the unclamped regime: at most 1 %
    of the final local energies lie further than sqrt(2/dt) from e_estimate
    (the clamp of sampling.py:84-88 would otherwise replace them by
    e_estimate and make the block energies agree by construction).  The
    unclamped weighted local energy of the final walkers (FP64 evaluation of
    the mixed-propagated walkers vs the oracle's) is bounded the same way."""
    from ad_afqmc_b200 import sampling

    norb, nelec, nchol, tr, W, S, nb, scale = shape
    wt = "restricted" if tr == "rhf" else "unrestricted"
    sys_ = make_system(norb, nelec, nchol, seed=13, trial=tr, chol_scale=scale)
    walkers = _walkers(sys_, W, 6, wt)
    rng = np.random.default_rng(7)
    fields = [rng.standard_normal((S, W, nchol)) for _ in range(nb)]
    uni = list(rng.random(nb))
    dt = 0.005
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, dt)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    e_o, o_pd = orc.Sampler(S, nb, 1).propagate_phaseless(o_prop, o_trial, o_ham, o_pd, o_wave,
                                                          ListSource(fields, uni))
    d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, wt, dt, W, precision=precision)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev(walkers))
    e_d, d_pd = sampling.sampler(S, nb, 1, field_source=ListSource(fields, uni)).propagate_phaseless(
        ham, d_ham, d_prop, d_pd, d_trial, d_wave)
    # regime: local energies of the final walkers against e_estimate
    el_o = np.real(o_trial.calc_energy(orc.orthonormalize(o_pd["walkers"]), o_ham, o_wave))
    clamped = float(np.mean(np.abs(el_o - o_pd["e_estimate"]) > (2.0 / dt) ** 0.5))
    assert clamped <= 0.01, clamped
    assert o_pd["n_killed_walkers"] == 0
    assert abs(float(e_d) - e_o) < 1e-4  # 0.1 mHa
    # unclamped weighted local energy of the final walkers, both evaluated in FP64
    el_d = _np(torch.real(d_trial.calc_energy(d_pd["walkers"].orthonormalize(), d_ham, d_wave)))
    w_d, w_o = _np(d_pd["weights"]), o_pd["weights"]
    e_unc_d = float(np.sum(el_d * w_d) / np.sum(w_d))
    e_unc_o = float(np.sum(el_o * w_o) / np.sum(w_o))
    assert abs(e_unc_d - e_unc_o) < 1e-4, (e_unc_d, e_unc_o)
