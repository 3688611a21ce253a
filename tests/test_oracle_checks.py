"""Self-checks of the oracle (CPU) against independent mathematics, for the
rows the reference's own tests do not pin with golden values: QR
re-orthonormalisation, the reconfiguration comb and the Taylor propagator.
The GPU path is compared with the oracle elsewhere; these make sure the
oracle itself states the reference's arithmetic."""

import math

import numpy as np
import pytest
import scipy.linalg

from oracle import afqmc_oracle as orc


def _walkers(rng, W, N, no):
    return rng.standard_normal((W, N, no)) + 1j * rng.standard_normal((W, N, no))


def test_qr_restricted_is_householder_q_and_det_r():
    """Q orthonormal, Q R = W with R upper triangular (LAPACK), norms = prod diag R."""
    rng = np.random.default_rng(1)
    w = _walkers(rng, 5, 12, 4)
    q, norms = orc.qr_restricted(w)
    for k in range(w.shape[0]):
        assert np.allclose(q[k].conj().T @ q[k], np.eye(4), atol=1e-13)
        r = q[k].conj().T @ w[k]
        assert np.allclose(np.tril(r, -1), 0, atol=1e-12)
        assert np.allclose(q[k] @ r, w[k], atol=1e-12)
        assert np.isclose(norms[k], np.prod(np.diag(r)), rtol=1e-12)
    # orthogonalize: |det R|^2 weight factor for restricted walkers is norms**2
    _, n2 = orc.orthogonalize(w)
    assert np.allclose(n2, norms ** 2)


def test_qr_unrestricted_fixes_the_phase_of_column_zero():
    """linalg_utils.py:58-72: the first column carries sign(prod diag R), so
    Q R' = W still holds with R' = diag(conj phase) R and |norms| are returned."""
    rng = np.random.default_rng(2)
    w = [_walkers(rng, 3, 10, 3), _walkers(rng, 3, 10, 2)]
    qs, norms = orc.qr_unrestricted(w)
    for s in range(2):
        q0, n0 = orc.qr_restricted(w[s])
        ph = n0 / np.abs(n0)
        assert np.allclose(qs[s][:, :, 0], q0[:, :, 0] * ph[:, None])
        assert np.allclose(qs[s][:, :, 1:], q0[:, :, 1:])
        assert np.allclose(norms[s], np.abs(n0))


def _comb_direct(weights, zeta):
    """Comb written out element by element: slot i takes the first walker
    whose cumulative |weight| reaches total * (i + zeta) / W."""
    w = np.abs(weights)
    total = w.sum()
    W = len(w)
    out = []
    for i in range(W):
        z = total * (i + zeta) / W
        acc, j = 0.0, 0
        while j < W - 1 and acc + w[j] < z:
            acc += w[j]
            j += 1
        out.append(j)
    return np.array(out)


@pytest.mark.parametrize("zeta", [0.0, 0.37, 0.999])
def test_reconfiguration_comb_matches_direct_statement(zeta):
    rng = np.random.default_rng(3)
    weights = rng.random(40) * (rng.random(40) > 0.2)  # some killed walkers
    idx, new_w = orc.sr_indices(weights, zeta)
    # same up to ties at cumulative-sum boundaries (measure zero for these weights)
    assert np.array_equal(idx, _comb_direct(weights, zeta))
    assert np.allclose(new_w, np.abs(weights).sum() / len(weights))
    # killed walkers are never selected; the comb is non-decreasing
    assert np.all(weights[idx] > 0)
    assert np.all(np.diff(idx) >= 0)


def test_global_comb_on_one_rank_equals_local_comb():
    rng = np.random.default_rng(4)
    weights = rng.random(64)
    for zeta in (0.1, 0.6):
        a, wa = orc.sr_indices(weights, zeta)
        b, wb = orc.sr_indices_global(weights, zeta, n_ranks=1)
        assert np.array_equal(a, b) and np.allclose(wa, wb)
    # across two ranks: every rank's slot draws from the gathered weights
    b2, w2 = orc.sr_indices_global(np.concatenate([weights, weights[::-1]]), 0.3, n_ranks=2)
    assert b2.shape == (128,) and np.allclose(w2, np.abs(np.concatenate([weights, weights[::-1]])).mean())


def test_taylor_propagator_approximates_the_exponential():
    """propagation.py:154-176: e^{-dt h/2} (sum_{n<K} VHS^n / n!) e^{-dt h/2}
    equals the exact exponential up to the first omitted term |VHS|^K / K!."""
    rng = np.random.default_rng(5)
    N, no = 16, 4
    prop = orc.Propagator(dt=0.01, walker_type="restricted", n_exp_terms=6)
    a = rng.standard_normal((N, N))
    vhs = 0.05j * (a + a.T)
    h = rng.standard_normal((N, N))
    exp_h1 = scipy.linalg.expm(-0.01 * (h + h.T) / 4)
    w = rng.standard_normal((N, no)) + 1j * rng.standard_normal((N, no))
    got = prop.apply_trotprop_single_det_vhs(w, vhs, exp_h1)
    exact = exp_h1 @ scipy.linalg.expm(vhs) @ exp_h1 @ w
    bound = np.linalg.norm(vhs, 2) ** 6 / math.factorial(6) * 1.1
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < bound
    # and the truncation is really the sixth term: ten terms are closer still
    prop10 = orc.Propagator(dt=0.01, walker_type="restricted", n_exp_terms=10)
    got10 = prop10.apply_trotprop_single_det_vhs(w, vhs, exp_h1)
    assert np.linalg.norm(got10 - exact) < np.linalg.norm(got - exact)
