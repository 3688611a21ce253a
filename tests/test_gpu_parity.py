"""FP64 parity of the CUDA walker path against the NumPy oracle.

Tolerances (from the specification of this path): per-step walker matrices
1e-10 relative; block energies 1e-8 Ha absolute; reconfiguration indices
bit-exact.  Measurements (overlap, Green's function, force bias, energy) are
held to 1e-10 relative.  All calls go through the reference-facing classes,
which call libafqmc_b200 through its C ABI.
"""

import copy
import json
import os

import numpy as np
import pytest
import torch

from ad_afqmc_b200.synthetic import make_system
from oracle import afqmc_oracle as orc
from tests._helpers import (ListSource, device_system, near_trial_walkers, oracle_system, rel_err)

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _np(t):
    return t.detach().cpu().numpy()


# ---------------------------------------------------------------------------
# the reference's own golden values, through the device path
# ---------------------------------------------------------------------------
def test_golden_values_rhf_uhf_on_device():
    from ad_afqmc_b200 import wavefunctions
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    G = np.load(os.path.join(GOLD, "trial_golden.npz"))
    ref = {k: v[0] for k, v in json.load(open(os.path.join(GOLD, "trial_golden.json"))).items()}
    tol = 1e-10
    # RHF (tests/test_wavefunctions.py:128-147)
    trial = wavefunctions.rhf(10, (5, 5))
    wave = {"mo_coeff": G["mo_coeff"]}
    ham = {"h0": float(G["h0"]), "rot_h1": torch.tensor(G["rot_h1"]).cuda(),
           "rot_chol": torch.tensor(G["rot_chol"]).cuda(),
           "chol": torch.tensor(G["chol"].reshape(5, 100)).cuda()}
    w = RHFWalkers(G["walker"][None])
    assert abs(_np(trial.calc_overlap(w, wave))[0].real - ref["rhf_overlap_real"]) < tol * 1
    assert abs(_np(trial.calc_green(w, wave)).sum().real - ref["rhf_green_sum_real"]) < tol * 100
    assert abs(_np(trial.calc_force_bias(w, ham, wave)).sum().real - ref["rhf_force_bias_sum_real"]) < tol * 100
    assert abs(_np(trial.calc_energy(w, ham, wave))[0].real - ref["rhf_energy_real"]) < tol * 1000
    # UHF (tests/test_wavefunctions.py:157-186)
    trial = wavefunctions.uhf(10, (3, 2))
    wave = {"mo_coeff": [G["mo_u0"], G["mo_u1"]]}
    ham = {"h0": float(G["h0"]),
           "rot_h1": [torch.tensor(G["rot_h1"][:3]).cuda(), torch.tensor(G["rot_h1"][:2]).cuda()],
           "rot_chol": [torch.tensor(np.ascontiguousarray(G["rot_chol"][:, :3])).cuda(),
                        torch.tensor(np.ascontiguousarray(G["rot_chol"][:, :2])).cuda()],
           "chol": torch.tensor(G["chol"].reshape(5, 100)).cuda()}
    w = UHFWalkers([G["walker_up"][None], G["walker_dn"][None]])
    assert abs(_np(trial.calc_overlap(w, wave))[0].real - ref["uhf_overlap_real"]) < tol
    g = trial.calc_green(w, wave)
    assert abs((_np(g[0]).sum() + _np(g[1]).sum()).real - ref["uhf_green_sum_real"]) < tol * 100
    assert abs(_np(trial.calc_force_bias(w, ham, wave)).sum().real - ref["uhf_force_bias_sum_real"]) < tol * 100
    assert abs(_np(trial.calc_energy(w, ham, wave))[0].real - ref["uhf_energy_real"]) < tol * 100


# ---------------------------------------------------------------------------
# measurements vs oracle on synthetic systems
# ---------------------------------------------------------------------------
CASES = [
    # (norb, nelec, nchol, trial, walker_type, W)
    (10, (5, 5), 50, "rhf", "restricted", 12),
    (24, (6, 6), 96, "rhf", "restricted", 20),
    (24, (6, 6), 96, "rhf", "unrestricted", 8),
    (30, (7, 5), 130, "uhf", "unrestricted", 9),
    (41, (11, 9), 77, "uhf", "unrestricted", 5),     # odd N, odd G, ragged tiles
    (70, (62, 62), 90, "rhf", "restricted", 3),     # No > 60: 128 x 160 exchange tile
    (66, (64, 61), 80, "uhf", "unrestricted", 2),   # the largest occupied block
]


def _setup(case, seed=7):
    norb, nelec, nchol, tr, wt, W = case
    sys_ = make_system(norb, nelec, nchol, seed=seed, trial=tr)
    rng = np.random.default_rng(seed + 1)
    if tr == "rhf":
        mo = [sys_.mo_coeff, sys_.mo_coeff]
    else:
        mo = sys_.mo_coeff
    if wt == "restricted":
        walkers = near_trial_walkers(rng, mo[0], W)
    else:
        walkers = [near_trial_walkers(rng, mo[0], W), near_trial_walkers(rng, mo[1], W)]
    return sys_, walkers


def _dev_walkers(walkers):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    if isinstance(walkers, list):
        return UHFWalkers([walkers[0].copy(), walkers[1].copy()])
    return RHFWalkers(walkers.copy())


@pytest.mark.parametrize("case", CASES)
def test_measurements_match_oracle(case):
    sys_, walkers = _setup(case)
    wt = case[4]
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, wt, 0.005)
    d_trial, d_ham, d_wave, _, _ = device_system(sys_, wt, 0.005, case[5])
    dw = _dev_walkers(walkers)
    assert rel_err(_np(d_trial.calc_overlap(dw, d_wave)), o_trial.calc_overlap(walkers, o_wave)) < 1e-10
    assert rel_err(_np(d_trial.calc_force_bias(dw, d_ham, d_wave)),
                   o_trial.calc_force_bias(walkers, o_ham, o_wave)) < 1e-10
    assert rel_err(_np(d_trial.calc_energy(dw, d_ham, d_wave)),
                   o_trial.calc_energy(walkers, o_ham, o_wave)) < 1e-10


def test_green_matches_oracle():
    sys_, walkers = _setup(CASES[3])
    d_trial, _, d_wave, _, _ = device_system(sys_, "unrestricted", 0.005, CASES[3][5])
    g = d_trial.calc_green(_dev_walkers(walkers), d_wave)
    for s in range(2):
        ref = np.array([orc.green(w, sys_.mo_coeff[s]) for w in walkers[s]])
        assert rel_err(_np(g[s]), ref) < 1e-11


# ---------------------------------------------------------------------------
# one phaseless step vs oracle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", CASES)
def test_one_step_matches_oracle(case):
    sys_, walkers = _setup(case)
    wt, W = case[4], case[5]
    dt = 0.005
    rng = np.random.default_rng(11)
    fields = rng.standard_normal((W, sys_.nchol))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, dt)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, wt, dt, W)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev_walkers(walkers))
    assert abs(float(d_pd["e_estimate"]) - o_pd["e_estimate"]) < 1e-9
    for step in range(2):
        f = fields if step == 0 else rng.standard_normal((W, sys_.nchol))
        o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, f, o_wave)
        d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, f, d_wave)
        if wt == "restricted":
            pairs = [(_np(d_pd["walkers"].data), o_pd["walkers"])]
        else:
            pairs = [(_np(d_pd["walkers"].data[s]), o_pd["walkers"][s]) for s in range(2)]
        for d, o in pairs:
            for w in range(W):
                assert rel_err(d[w], o[w]) < 1e-10, (step, w)
        assert rel_err(_np(d_pd["overlaps"]), o_pd["overlaps"]) < 1e-10
        assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=1e-10, atol=1e-13)
        ds, os_ = float(d_pd["pop_control_ene_shift"]), float(o_pd["pop_control_ene_shift"])
        # every walker killed: log(0) makes both shifts +inf
        assert ds == os_ or abs(ds - os_) < 1e-8, (ds, os_)


# ---------------------------------------------------------------------------
# QR and reconfiguration
# ---------------------------------------------------------------------------
# N = 330 is above the register-resident variant's 320 rows: the loop form
@pytest.mark.parametrize("shape", [(10, 5), (40, 12), (61, 17), (200, 40), (330, 9)])
def test_qr_matches_lapack(shape):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    N, no = shape
    rng = np.random.default_rng(3)
    W = 6
    a = rng.standard_normal((W, N, no)) + 1j * rng.standard_normal((W, N, no))
    q_ref, n_ref = orc.qr_restricted(a)
    out, norms = RHFWalkers(a.copy()).orthogonalize()
    assert rel_err(_np(out.data), q_ref) < 1e-12
    assert rel_err(_np(norms), n_ref**2) < 1e-11
    b = rng.standard_normal((W, N, no - 1)) + 1j * rng.standard_normal((W, N, no - 1))
    qs, _ = orc.qr_unrestricted([a, b])
    u = UHFWalkers([a.copy(), b.copy()]).orthonormalize()
    assert rel_err(_np(u.data[0]), qs[0]) < 1e-12
    assert rel_err(_np(u.data[1]), qs[1]) < 1e-12


@pytest.mark.parametrize("qr_mode", [1, 2])
def test_qr_placement_knob(qr_mode):
    """The QR with the walker staged in shared memory (qr_mode 1) or factored
    in place in global memory (qr_mode 2, tuning record): both LAPACK's."""
    from ad_afqmc_b200 import _lib
    from ad_afqmc_b200.walkers import RHFWalkers, _dims

    rng = np.random.default_rng(8)
    W, N, no = 9, 200, 40
    a = rng.standard_normal((W, N, no)) + 1j * rng.standard_normal((W, N, no))
    q_ref, _ = orc.qr_restricted(a)
    d = _dims(N, (no, no), W, "restricted")
    t = _lib.afq_tuning()
    t.qr_mode = qr_mode
    _lib.set_tuning(d, t)
    try:
        out = RHFWalkers(a.copy()).orthonormalize()
        got = _np(out.data)
    finally:
        _lib.set_tuning(d, None)
    assert rel_err(got, q_ref) < 1e-12


def test_qr_large_walker_global_memory_path():
    """N=300, No=60 does not fit in shared memory: the in-place global path."""
    from ad_afqmc_b200.walkers import UHFWalkers

    rng = np.random.default_rng(5)
    a = rng.standard_normal((3, 300, 60)) + 1j * rng.standard_normal((3, 300, 60))
    b = rng.standard_normal((3, 300, 58)) + 1j * rng.standard_normal((3, 300, 58))
    qs, _ = orc.qr_unrestricted([a, b])
    u = UHFWalkers([a.copy(), b.copy()]).orthonormalize()
    assert rel_err(_np(u.data[0]), qs[0]) < 1e-12
    assert rel_err(_np(u.data[1]), qs[1]) < 1e-12


@pytest.mark.parametrize("W", [1, 7, 100, 512, 1024, 4099])
@pytest.mark.parametrize("mode", ["local", "global"])
def test_reconfiguration_bit_exact(W, mode):
    from ad_afqmc_b200.walkers import RHFWalkers

    rng = np.random.default_rng(W)
    weights = rng.random(W) * 2.0
    weights[rng.random(W) < 0.1] = 0.0  # killed walkers
    zeta = float(rng.random())
    walkers = rng.standard_normal((W, 4, 2)) + 1j * rng.standard_normal((W, 4, 2))
    if mode == "local":
        idx, wn = orc.sr_indices(weights, zeta)
        out, w = RHFWalkers(walkers.copy()).stochastic_reconfiguration_local(torch.tensor(weights).cuda(), zeta)
    else:
        idx, wn = orc.sr_indices_global(weights, zeta)
        out, w = RHFWalkers(walkers.copy()).stochastic_reconfiguration_global(torch.tensor(weights).cuda(), zeta)
    assert np.array_equal(_np(out.data), walkers[idx])  # bit-exact gather
    assert np.array_equal(_np(w), wn)


def test_reconfiguration_all_zero_weights():
    from ad_afqmc_b200.walkers import RHFWalkers

    W = 16
    walkers = np.arange(W * 4, dtype=np.complex128).reshape(W, 2, 2)
    idx, wn = orc.sr_indices(np.zeros(W), 0.3)
    out, w = RHFWalkers(walkers.copy()).stochastic_reconfiguration_local(torch.zeros(W, dtype=torch.float64).cuda(), 0.3)
    assert np.array_equal(_np(out.data), walkers[idx])
    assert np.array_equal(_np(w), wn)


# ---------------------------------------------------------------------------
# blocks (sampler.propagate_phaseless) vs oracle, injected randomness
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[3]])
def test_blocks_match_oracle(case):
    from ad_afqmc_b200 import sampling

    sys_, walkers = _setup(case)
    wt, W = case[4], case[5]
    dt = 0.005
    S, n_ene, n_sr = 4, 2, 2
    rng = np.random.default_rng(21)
    fields = [rng.standard_normal((S, W, sys_.nchol)) for _ in range(n_ene * n_sr)]
    uniforms = list(rng.random(n_sr))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, wt, dt)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    o_smp = orc.Sampler(n_prop_steps=S, n_ene_blocks=n_ene, n_sr_blocks=n_sr)
    e_o, o_pd = o_smp.propagate_phaseless(o_prop, o_trial, o_ham, o_pd, o_wave, ListSource(fields, uniforms))

    d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, wt, dt, W)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=_dev_walkers(walkers))
    d_smp = sampling.sampler(n_prop_steps=S, n_ene_blocks=n_ene, n_sr_blocks=n_sr,
                             field_source=ListSource(fields, uniforms))
    e_d, d_pd = d_smp.propagate_phaseless(ham, d_ham, d_prop, d_pd, d_trial, d_wave)
    assert abs(float(e_d) - e_o) < 1e-8
    assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=1e-9, atol=1e-12)
    assert abs(float(d_pd["n_killed_walkers"]) - o_pd["n_killed_walkers"]) < 1e-12


# ---------------------------------------------------------------------------
# full-size shapes: parity on a few walkers, properties on all of them
# ---------------------------------------------------------------------------
def test_config_rhf_n200_subset_parity_and_permutation():
    from ad_afqmc_b200.walkers import RHFWalkers

    sys_ = make_system(200, (40, 40), 1000, seed=1002, trial="rhf")
    rng = np.random.default_rng(2)
    W = 4
    walkers = near_trial_walkers(rng, sys_.mo_coeff, W, eps=0.05)
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, "restricted", 0.005)
    d_trial, d_ham, d_wave, _, _ = device_system(sys_, "restricted", 0.005, W)
    dw = RHFWalkers(walkers.copy())
    e_d = _np(d_trial.calc_energy(dw, d_ham, d_wave))
    e_o = o_trial.calc_energy(walkers, o_ham, o_wave)
    assert np.max(np.abs(e_d - e_o)) < 1e-8
    fb_d = _np(d_trial.calc_force_bias(dw, d_ham, d_wave))
    assert rel_err(fb_d, o_trial.calc_force_bias(walkers, o_ham, o_wave)) < 1e-10
    # permuting walkers permutes results exactly
    perm = np.array([2, 0, 3, 1])
    e_p = _np(d_trial.calc_energy(RHFWalkers(walkers[perm].copy()), d_ham, d_wave))
    assert np.array_equal(e_p, e_d[perm])


def test_config_uhf_n300_subset_parity():
    """Config-3 shapes (N=300, Na=60, Nb=58, G=1500): measurements and one step
    on a few walkers (QR and walkers take the in-place global-memory paths)."""
    from ad_afqmc_b200.walkers import UHFWalkers

    sys_ = make_system(300, (60, 58), 1500, seed=1003, trial="uhf", chol_scale=0.25)
    rng = np.random.default_rng(9)
    W = 3
    walkers = [near_trial_walkers(rng, sys_.mo_coeff[0], W, eps=0.05),
               near_trial_walkers(rng, sys_.mo_coeff[1], W, eps=0.05)]
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "unrestricted", 0.005)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "unrestricted", 0.005, W)
    dw = UHFWalkers([walkers[0].copy(), walkers[1].copy()])
    e_d = _np(d_trial.calc_energy(dw, d_ham, d_wave))
    assert np.max(np.abs(e_d - o_trial.calc_energy(walkers, o_ham, o_wave))) < 1e-8
    fields = rng.standard_normal((W, 1500))
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields, o_wave)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=dw)
    d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, fields, d_wave)
    for s in range(2):
        assert rel_err(_np(d_pd["walkers"].data[s]), o_pd["walkers"][s]) < 1e-10
    assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=1e-10, atol=1e-13)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config_rhf_n200_full_tile_step(precision):
    """A full tile of walkers at the N = 200 / G = 1000 headline shape (128
    walkers: whole 128-column tiles in the force-bias and VHS GEMMs and 16 row
    tiles of the exchange): one phaseless step and the local energies of every
    walker against the oracle, FP64 to 1e-10 and BF16x3 to 1e-4 relative."""
    from ad_afqmc_b200.walkers import RHFWalkers

    sys_ = make_system(200, (40, 40), 1000, seed=1002, trial="rhf", chol_scale=0.1)
    rng = np.random.default_rng(31)
    W = 128
    walkers = near_trial_walkers(rng, sys_.mo_coeff, W, eps=0.05)
    fields = rng.standard_normal((W, 1000))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "restricted", 0.005)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=walkers.copy())
    o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields, o_wave)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "restricted", 0.005, W, precision=precision)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=RHFWalkers(walkers.copy()))
    d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, fields, d_wave)
    tol = 1e-10 if precision == "fp64" else 1e-4
    dw = _np(d_pd["walkers"].data)
    for w in range(W):
        assert rel_err(dw[w], o_pd["walkers"][w]) < tol, w
    assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=10 * tol, atol=1e-12)
    e_o = np.real(o_trial.calc_energy(o_pd["walkers"], o_ham, o_wave))
    e_d = _np(torch.real(d_trial.calc_energy(d_pd["walkers"], d_ham, d_wave)))
    # mixed: the walkers differ at the 1e-5 level, which moves E_L (~ -290 Ha) by ~1e-3 Ha
    assert np.max(np.abs(e_d - e_o)) < (1e-8 if precision == "fp64" else 1e-2)
