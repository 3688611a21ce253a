"""Per-solve intermediates on the library's kernels against the oracle.

afq_measurement_intermediates (symmetrized h1, rot_h1, rot_chol),
afq_propagation_intermediates (mf_shifts, h0_prop, v0 + v1 inside exp_h1),
afq_expm (Taylor scaling and squaring) and afq_eigh_desc (Jacobi) against
NumPy/SciPy FP64 (the oracle's restatement of wavefunctions.py:1215-1232,
1472-1496 and propagation.py:378-438), and the initial walkers of
get_init_walkers (wavefunctions.py:427-466)."""

import numpy as np
import pytest
import scipy.linalg
import torch

from ad_afqmc_b200.synthetic import make_system
from tests._helpers import device_system, oracle_system, rel_err

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


SHAPES = [(10, (5, 5), 50, "rhf"), (48, (13, 11), 200, "uhf"), (200, (40, 40), 1000, "rhf"),
          (131, (30, 27), 600, "uhf")]


@pytest.mark.parametrize("shape", SHAPES)
def test_intermediates_match_oracle(shape):
    n, nelec, g, tr = shape
    sys_ = make_system(n, nelec, g, seed=41, trial=tr, chol_scale=0.3)
    # an unsymmetric h1 exercises the symmetrization
    rng = np.random.default_rng(3)
    sys_.h1 = sys_.h1 + 0.01 * rng.standard_normal(sys_.h1.shape)
    wt = "restricted" if tr == "rhf" else "unrestricted"
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, wt, 0.005)
    d_trial, d_ham, d_wave, _, _ = device_system(sys_, wt, 0.005, 4)
    assert rel_err(_np(d_ham["h1"]), o_ham["h1"]) < 1e-14
    if tr == "rhf":
        assert rel_err(_np(d_ham["rot_h1"]), o_ham["rot_h1"]) < 1e-12
        assert rel_err(_np(d_ham["rot_chol"]), o_ham["rot_chol"]) < 1e-12
    else:
        for s in range(2):
            assert rel_err(_np(d_ham["rot_h1"][s]), o_ham["rot_h1"][s]) < 1e-12
            assert rel_err(_np(d_ham["rot_chol"][s]), o_ham["rot_chol"][s]) < 1e-12
    assert rel_err(_np(d_ham["mf_shifts"]), o_ham["mf_shifts"]) < 1e-12
    assert abs(complex(d_ham["h0_prop"].item()) - complex(o_ham["h0_prop"])) < 1e-10 * max(1.0, abs(o_ham["h0_prop"]))
    assert rel_err(_np(d_ham["exp_h1"]), o_ham["exp_h1"]) < 1e-12
    assert rel_err(_np(d_ham["mf_shifts_fp"]), o_ham["mf_shifts_fp"]) < 1e-12


@pytest.mark.parametrize("norm", [1e-3, 0.3, 7.0, 60.0])
def test_expm_matches_scipy(norm):
    from ad_afqmc_b200 import intermediates

    rng = np.random.default_rng(int(norm * 1000) % 97)
    n = 77
    a = rng.standard_normal((n, n))
    a *= norm / np.abs(a).sum(axis=0).max()
    ref = scipy.linalg.expm(-0.5 * a)
    got = _np(intermediates.expm(torch.as_tensor(a, device="cuda"), -0.5))
    # squaring amplifies the relative error of the scaled series by about 2^s
    assert rel_err(got, ref) < 1e-13 * max(1.0, norm)
    assert rel_err(_np(intermediates.expm(torch.zeros(5, 5, dtype=torch.float64, device="cuda"))),
                   np.eye(5)) == 0.0


@pytest.mark.parametrize("n", [1, 2, 9, 64, 200, 301])
def test_eigh_desc_matches_lapack(n):
    from ad_afqmc_b200 import intermediates

    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    a = (a + a.T) / 2
    w_ref, v_ref = np.linalg.eigh(a)
    w, v = intermediates.eigh_desc(torch.as_tensor(a, device="cuda"))
    w, v = _np(w), _np(v)
    scale = np.abs(w_ref).max()
    assert np.allclose(w, w_ref[::-1], rtol=0, atol=1e-12 * scale)
    assert np.allclose(v.T @ v, np.eye(n), atol=1e-12)
    assert np.linalg.norm(a @ v - v * w) < 1e-11 * scale * np.sqrt(n)
    # distinct eigenvalues: the same vectors as LAPACK up to sign
    dots = np.abs(np.sum(v * v_ref[:, ::-1], axis=0))
    assert np.allclose(dots, 1.0, atol=1e-9)


@pytest.mark.parametrize("tr", ["rhf", "uhf"])
def test_initial_walkers_are_natural_orbitals(tr):
    """Projector density matrices: the initial walkers span the trial's
    occupied space (|overlap| = 1) and their energy equals the oracle's."""
    from oracle import afqmc_oracle as orc

    nelec = (20, 20) if tr == "rhf" else (20, 17)
    sys_ = make_system(90, nelec, 300, seed=8, trial=tr, chol_scale=0.3)
    wt = "restricted" if tr == "rhf" else "unrestricted"
    o_trial, o_ham, o_wave, _ = oracle_system(sys_, wt, 0.005)
    d_trial, d_ham, d_wave, _, _ = device_system(sys_, wt, 0.005, 3)
    w = d_trial.get_init_walkers(d_wave, 3, wt)
    ov = _np(d_trial.calc_overlap(w, d_wave))
    assert np.allclose(np.abs(ov), 1.0, atol=1e-12)
    ow = orc.get_init_walkers(o_trial, o_wave, 3, wt)
    e_o = np.real(o_trial.calc_energy(ow, o_ham, o_wave))
    e_d = _np(torch.real(d_trial.calc_energy(w, d_ham, d_wave)))
    assert np.allclose(e_d, e_o, rtol=0, atol=1e-9)


def test_initial_walkers_correlated_density():
    """A density matrix with distinct occupations (not a projector): the
    natural orbitals match LAPACK's up to sign."""
    from ad_afqmc_b200 import wavefunctions

    n, no = 40, 8
    rng = np.random.default_rng(12)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    occ = np.sort(rng.random(n))[::-1]
    rdm = (q * occ) @ q.T
    trial = wavefunctions.rhf(n, (no, no))
    wave = {"mo_coeff": q[:, :no].copy(), "rdm1": np.array([rdm, rdm])}
    w = _np(trial.get_init_walkers(wave, 2, "restricted").data)[0].real
    ref = np.linalg.eigh(2 * rdm)[1][:, ::-1][:, :no]
    assert np.allclose(np.abs(np.sum(w * ref, axis=0)), 1.0, atol=1e-10)


@pytest.mark.parametrize("gap", [0.5, 1e-3])
def test_natural_orbitals_subspace_and_fallback(gap):
    """afq_natural_orbitals: a clear gap at the cut converges by subspace
    iteration; a gap of 1e-3 does not within its iteration limit and takes the
    full Jacobi eigensolver.  Either way the span of the k orbitals is LAPACK's
    (its projector to 1e-10) and the occupations match."""
    from ad_afqmc_b200 import intermediates

    n, k = 73, 17
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    occ = np.concatenate([1.0 + 0.9 * rng.random(k), (1.0 - gap) * rng.random(n - k)])
    occ[k - 1] = 1.0
    occ[k] = 1.0 - gap
    rdm = (q * occ) @ q.T
    orbs, o = intermediates.natural_orbitals(torch.as_tensor(rdm, device="cuda"), k, return_occ=True)
    orbs, o = _np(orbs), _np(o)
    ref = np.sort(occ)[::-1][:k]
    assert np.allclose(o, ref, atol=1e-12)
    w, v = np.linalg.eigh(rdm)
    vk = v[:, ::-1][:, :k]
    assert np.abs(orbs @ orbs.T - vk @ vk.T).max() < 1e-10
    assert np.allclose(orbs.T @ orbs, np.eye(k), atol=1e-12)
