"""LNO fragment path: the orbital energy of rhf_lno (afq_calc_orbenergy) and
sampler_lno blocks against the oracle's restatement of
wavefunctions.py:6898-6923 and sampling.py:583-694.  The reference's own LNO
test (tests/test_lnoafqmc.py) needs pyscf and JAX random numbers, so the
orbital energy is checked against the oracle only."""

import copy

import numpy as np
import pytest
import torch

from ad_afqmc_b200.synthetic import make_system
from oracle import afqmc_oracle as orc
from tests._helpers import ListSource, device_system, near_trial_walkers, oracle_system, rel_err

pytestmark = pytest.mark.gpu


def _lno_system(n_lo, seed, N=30, no=8, G=110):
    sys_ = make_system(N, (no, no), G, seed=seed, trial="rhf", chol_scale=0.25)
    rng = np.random.default_rng(seed)
    prj = rng.standard_normal((n_lo, no))
    prj /= np.linalg.norm(prj, axis=1, keepdims=True)
    return sys_, prj


def _device_lno(sys_, W, precision, prj):
    from ad_afqmc_b200 import hamiltonian, propagation, wavefunctions

    trial = wavefunctions.rhf_lno(sys_.norb, sys_.nelec)
    ham = hamiltonian.hamiltonian(sys_.norb)
    prop = propagation.propagator_afqmc(dt=0.005, n_walkers=W, precision=precision)
    hd, wd = sys_.ham_data(), sys_.wave_data()
    wd["prjlo"] = prj
    hd = ham.build_measurement_intermediates(hd, trial, wd)
    hd = ham.build_propagation_intermediates(hd, prop, trial, wd)
    return trial, ham, prop, hd, wd


@pytest.mark.parametrize("n_lo", [1, 3, 8])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_orbital_energy_matches_oracle(n_lo, precision):
    from ad_afqmc_b200.walkers import RHFWalkers

    sys_, prj = _lno_system(n_lo, 31 + n_lo)
    W = 9
    walkers = near_trial_walkers(np.random.default_rng(5), sys_.mo_coeff, W, eps=0.3)
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, "restricted", 0.005)
    o_wave["prjlo"] = prj
    ref = o_trial.calc_orbenergy(walkers, o_ham, o_wave)
    trial, _, prop, hd, wd = _device_lno(sys_, W, precision, prj)
    dw = RHFWalkers(walkers.copy())
    got = trial.calc_orbenergy(dw, hd, wd).cpu().numpy()            # FP64 engine
    assert rel_err(got, ref) < 1e-10
    got = trial.calc_orbenergy(dw, hd, wd, engine=prop.engine(hd, trial, wd)).cpu().numpy()
    assert rel_err(got, ref) < 1e-10                                # FP64 whatever the precision
    # the ordinary energy still matches after the orbital energy overwrote Theta's occupied rows
    e = trial.calc_energy(dw, hd, wd).cpu().numpy()
    assert rel_err(e, o_trial.calc_energy(walkers, o_ham, o_wave)) < 1e-10


def test_orbital_energy_rejects_bad_inputs():
    from ad_afqmc_b200 import _lib
    from ad_afqmc_b200.walkers import UHFWalkers

    sys_, prj = _lno_system(1, 3)
    trial, _, _, hd, wd = _device_lno(sys_, 4, "fp64", prj)
    w = near_trial_walkers(np.random.default_rng(1), sys_.mo_coeff, 4)
    with pytest.raises(NotImplementedError):
        trial.calc_orbenergy(UHFWalkers([w, w]), hd, wd)
    from ad_afqmc_b200.walkers import RHFWalkers

    wd["prjlo"] = np.ones((9, sys_.nelec[0]))
    with pytest.raises(_lib.AfqError):
        trial.calc_orbenergy(RHFWalkers(w), hd, wd)


def test_sampler_lno_blocks_match_oracle():
    from ad_afqmc_b200 import sampling
    from ad_afqmc_b200.walkers import RHFWalkers

    sys_, prj = _lno_system(1, 7, N=24, no=6, G=90)
    W, S, nb = 12, 4, 2
    walkers = near_trial_walkers(np.random.default_rng(2), sys_.mo_coeff, W, eps=0.1)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal((S, W, sys_.nchol)) for _ in range(2 * nb)]
    uni = list(rng.random(2 * nb))
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "restricted", 0.005)
    o_wave["prjlo"] = prj
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    trial, ham, prop, hd, wd = _device_lno(sys_, W, "fp64", prj)
    d_pd = prop.init_prop_data(trial, wd, hd, 0, init_walkers=RHFWalkers(walkers.copy()))
    src_o, src_d = ListSource(fields, uni), ListSource(fields, uni)
    smp_o = orc.SamplerLNO(S, nb, 1)
    smp_d = sampling.sampler_lno(S, nb, 1, field_source=src_d)
    for _ in range(2):
        e_o, o_pd, orb_o = smp_o.propagate_phaseless(o_prop, o_trial, o_ham, o_pd, o_wave, src_o)
        e_d, d_pd, orb_d = smp_d.propagate_phaseless(ham, hd, prop, d_pd, trial, wd)
        assert abs(float(e_d) - e_o) < 1e-8
        assert abs(float(orb_d) - orb_o) < 1e-8
        assert abs(float(d_pd["pop_control_ene_shift"]) - o_pd["pop_control_ene_shift"]) < 1e-8


def _lno_graph(seed=9, W=16, precision="fp64"):
    from ad_afqmc_b200.graphs import BlockGraph

    sys_, prj = _lno_system(1, seed, N=24, no=6, G=90)
    trial, ham, prop, hd, wd = _device_lno(sys_, W, precision, prj)
    pd = prop.init_prop_data(trial, wd, hd, seed)
    return BlockGraph(ham, hd, prop, trial, wd, pd, n_prop_steps=4, lno=True), sys_, prj


def test_lno_graph_replay_equals_eager():
    a, _, _ = _lno_graph()
    b, _, _ = _lno_graph()
    ea = []
    for _ in range(3):
        a.body()
        ea.append(a.block_out.cpu().tolist())
    b.capture(warmup=0)
    eb = [b.replay().cpu().tolist() for _ in range(3)]
    assert ea == eb
    assert torch.equal(a.tensors[0], b.tensors[0])


def test_lno_graph_block_matches_oracle():
    """One recorded LNO block (device-drawn fields and zeta) vs SamplerLNO fed the same numbers."""
    bg, sys_, prj = _lno_graph(seed=12)
    w0 = bg.tensors[0].cpu().numpy().copy()
    bg.body()
    fields = bg.fields.cpu().numpy().copy()
    zeta = float(bg.zeta)
    o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "restricted", 0.005)
    o_wave["prjlo"] = prj
    o_prop.n_walkers = bg.prop.n_walkers
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=w0)
    e_o, o_pd, orb_o = orc.SamplerLNO(4, 1, 1).propagate_phaseless(o_prop, o_trial, o_ham, o_pd, o_wave,
                                                                   ListSource([fields], [zeta]))
    out = bg.block_out.cpu().numpy()
    assert abs(out[0] - e_o) < 1e-8 and abs(out[2] - orb_o) < 1e-8
    assert rel_err(bg.tensors[0].cpu().numpy(), o_pd["walkers"]) < 1e-10
