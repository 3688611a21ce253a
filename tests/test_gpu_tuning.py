"""Tuning records change tiles, not results: the FP64 path stays at oracle
parity under every exchange tile and split-K, the mixed path within its
tolerance under every tensor-core tile/stage/grid choice, and the autotuner
produces a usable record."""

import ctypes as C

import numpy as np
import pytest
import torch

from ad_afqmc_b200 import _lib
from ad_afqmc_b200.synthetic import make_system
from ad_afqmc_b200.walkers import RHFWalkers
from ad_afqmc_b200.wavefunctions import _ptrs
from tests._helpers import device_system, near_trial_walkers, oracle_system, rel_err

pytestmark = pytest.mark.gpu


def _measure(eng, walkers, W, G):
    dw = RHFWalkers(walkers.copy())
    fb = torch.empty(W, G, dtype=torch.complex128, device="cuda")
    e = torch.empty(W, dtype=torch.complex128, device="cuda")
    p, w, wb = eng.handle
    _lib.check(_lib.lib().afq_calc_force_bias(C.byref(eng.dims), p, _ptrs(dw), fb.data_ptr(), w, wb,
                                              _lib.stream_handle()), "fb")
    _lib.check(_lib.lib().afq_calc_energy(C.byref(eng.dims), p, _ptrs(dw), e.data_ptr(), w, wb,
                                          _lib.stream_handle()), "energy")
    return fb.cpu().numpy(), e.cpu().numpy()


def _setup(precision, N=40, no=10, G=150, W=7, seed=21):
    sys_ = make_system(N, (no, no), G, seed=seed, trial="rhf", chol_scale=0.25)
    walkers = near_trial_walkers(np.random.default_rng(seed), sys_.mo_coeff, W, eps=0.1)
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, "restricted", 0.005)
    fb_o = o_trial.calc_force_bias(walkers, o_ham, o_wave)
    e_o = o_trial.calc_energy(walkers, o_ham, o_wave)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "restricted", 0.005, W, precision=precision)
    eng = d_prop.engine(d_ham, d_trial, d_wave)
    return eng, walkers, fb_o, e_o, W, G


@pytest.mark.parametrize("rec", [{"f64_exch_bn": 80}, {"f64_exch_bn": 120}, {"f64_exch_bn": 160},
                                 {"fb_splitk": 1}, {"fb_splitk": 3}, {"fb_splitk": 8}])
def test_fp64_parity_under_every_record(rec):
    eng, walkers, fb_o, e_o, W, G = _setup("fp64")
    try:
        _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec))
        eng.ensure_workspace()
        fb, e = _measure(eng, walkers, W, G)
    finally:
        _lib.set_tuning(eng.dims, None)
    assert rel_err(fb, fb_o) < 1e-10
    assert rel_err(e, e_o) < 1e-10


@pytest.mark.parametrize("rec", [{"vhs_bn": 64}, {"fb_bn": 64}, {"fb_splitk": 1}, {"exch_bn": 32},
                                 {"exch_bn": 64}, {"exch_bn": 128}, {"max_stages": 2},
                                 {"grid_cap": 3}, {"grid_cap": 1, "max_stages": 2, "fb_bn": 64}])
def test_mixed_within_tolerance_under_every_record(rec):
    eng, walkers, fb_o, e_o, W, G = _setup("mixed")
    try:
        _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec))
        eng.ensure_workspace()
        fb, e = _measure(eng, walkers, W, G)
    finally:
        _lib.set_tuning(eng.dims, None)
    assert rel_err(fb, fb_o) < 1e-4
    assert np.max(np.abs(e - e_o)) / np.max(np.abs(e_o)) < 1e-4


def test_autotuner_record_is_used_and_cached(tmp_path):
    from ad_afqmc_b200.autotune import Autotuner, shape_key

    sys_ = make_system(48, (12, 12), 200, seed=5, trial="rhf", chol_scale=0.25)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "restricted", 0.005, 64, precision="mixed")
    pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 3)
    eng = d_prop.engine(d_ham, d_trial, d_wave)
    tuner = Autotuner(cache_path=str(tmp_path / "tune.json"), reps=2, n_prop_steps=3)
    try:
        rec = tuner.tune(eng, pd)
        tuner.save()
        assert rec["ms"] <= rec["ms_default"]
        assert shape_key(eng.dims) in Autotuner(cache_path=str(tmp_path / "tune.json")).cache
        eff = _lib.get_tuning(eng.dims).as_dict()
        for k, v in rec["tuning"].items():
            assert eff[k] == v
        # the tuned engine still propagates
        f = torch.randn(64, 200, dtype=torch.float64, device="cuda")
        pd = d_prop.propagate_constrained(d_trial, d_ham, pd, f, d_wave)
        assert torch.isfinite(pd["weights"]).all()
    finally:
        _lib.set_tuning(eng.dims, None)


@pytest.mark.parametrize("rec", [{}, {"vhs_chunk": 2}, {"prop_chunk": 2}, {"vhs_chunk": 2, "prop_chunk": 2}])
@pytest.mark.parametrize("shape", [(48, (12, 12), 200, 8), (200, (40, 40), 1000, 4)])
def test_step_under_accumulation_choices(rec, shape):
    """The VHS GEMM and the propagator accumulate K in one TMEM chain by
    default, or in FP32 round-to-nearest chunks of four K blocks (knob value
    2): a step stays within the mixed path's 1e-4 of the oracle either way."""
    import copy

    N, nelec, G, W = shape
    sys_ = make_system(N, nelec, G, seed=12, trial="rhf", chol_scale=0.25)
    walkers = near_trial_walkers(np.random.default_rng(4), sys_.mo_coeff, W, eps=0.1)
    fields = np.random.default_rng(5).standard_normal((W, G))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "restricted", 0.005)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields, o_wave)
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "restricted", 0.005, W, precision="mixed")
    eng = d_prop.engine(d_ham, d_trial, d_wave)
    try:
        _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec) if rec else None)
        eng.ensure_workspace()
        d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=RHFWalkers(walkers.copy()))
        d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, fields, d_wave)
        got = d_pd["walkers"].data.cpu().numpy()
    finally:
        _lib.set_tuning(eng.dims, None)
    assert rel_err(got, o_pd["walkers"]) < 1e-4


@pytest.mark.parametrize("bn", [16, 32, 48])
def test_propagator_column_tiles_bit_identical(bn):
    """prop_bn splits a walker's 2 No = 80 propagator columns over several
    tensor-core tiles; every column's sum over K is the same chain in TMEM,
    so a step is bit-identical to the built-in single tile."""
    sys_ = make_system(200, (40, 40), 1000, seed=12, trial="rhf", chol_scale=0.25)
    W = 6
    walkers = near_trial_walkers(np.random.default_rng(4), sys_.mo_coeff, W, eps=0.1)
    fields = np.random.default_rng(5).standard_normal((W, 1000))
    d_trial, d_ham, d_wave, d_prop, _ = device_system(sys_, "restricted", 0.005, W, precision="mixed")
    eng = d_prop.engine(d_ham, d_trial, d_wave)
    out = []
    try:
        for rec in ({}, {"prop_bn": bn}):
            _lib.set_tuning(eng.dims, _lib.afq_tuning.from_dict(rec) if rec else None)
            eng.ensure_workspace()
            pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=RHFWalkers(walkers.copy()))
            pd = d_prop.propagate_constrained(d_trial, d_ham, pd, fields, d_wave)
            out.append((pd["walkers"].data.clone(), pd["weights"].clone()))
    finally:
        _lib.set_tuning(eng.dims, None)
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
