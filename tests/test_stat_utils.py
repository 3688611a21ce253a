"""Block statistics (stat_utils.py:8-78) against a plain-loop statement of
the same algorithm: weighted mean, blocked weighted errors for block sizes
1, 2, 5, 10, ... below half the sample count, the first plateau (an error
within 5 % of the previous one) or twice the unblocked error, and the
outlier mask from the median / IQR dispersion."""

import os

import numpy as np
import pytest

from ad_afqmc_b200 import stat_utils


def _blocking_loops(weights, energies, neql=0):
    weights, energies = weights[neql:], energies[neql:]
    n = len(weights)
    we = weights * energies
    mean_energy = we.sum() / weights.sum()
    prev, plateau, errors = 0.0, None, []
    for i in [1, 2, 5, 10, 20, 50, 100, 200, 300, 400, 500, 1000, 10000]:
        if not i < n / 2.0:
            continue
        nb = n // i
        bw = np.array([weights[j * i:(j + 1) * i].sum() for j in range(nb)])
        be = np.array([we[j * i:(j + 1) * i].sum() for j in range(nb)]) / bw
        v1, v2 = bw.sum(), (bw ** 2).sum()
        mean = (bw * be).sum() / v1
        err = ((bw * (be - mean) ** 2).sum() / (v1 - v2 / v1) / (nb - 1)) ** 0.5
        errors.append(err)
        if err < 1.05 * prev and plateau is None:
            plateau = max(err, prev)
        prev = err
    if plateau is None and errors:
        plateau = 2 * errors[0]
    return mean_energy, plateau


@pytest.mark.parametrize("n,neql,corr", [(3, 0, 0.0), (40, 0, 0.0), (250, 10, 0.9), (1200, 0, 0.5)])
def test_blocking_analysis_matches_loops(n, neql, corr):
    rng = np.random.default_rng(n)
    e = np.empty(n)
    x = 0.0
    for k in range(n):  # AR(1) series: correlated block energies
        x = corr * x + rng.standard_normal()
        e[k] = -3.2 + 0.01 * x
    w = rng.random(n) + 0.5
    got = stat_utils.blocking_analysis(w, e, neql=neql)
    ref = _blocking_loops(w, e, neql)
    assert np.isclose(got[0], ref[0], rtol=0, atol=1e-14)
    if ref[1] is None:
        assert got[1] is None
    else:
        assert np.isclose(got[1], ref[1], rtol=1e-12)


def test_blocking_writes_blocked_samples(tmp_path):
    rng = np.random.default_rng(0)
    w, e = rng.random(30) + 1, rng.standard_normal(30)
    cwd = os.getcwd()
    try:
        os.chdir(tmp_path)
        stat_utils.blocking_analysis(w, e, writeBlockedQ=True)
        assert sorted(os.listdir(tmp_path)) == ["samples_blocked_1.dat", "samples_blocked_10.dat",
                                                "samples_blocked_2.dat", "samples_blocked_5.dat"]
        blocked = np.loadtxt(tmp_path / "samples_blocked_5.dat")
        assert blocked.shape == (6, 2) and np.isclose(blocked[0, 0], w[:5].sum())
    finally:
        os.chdir(cwd)


def test_reject_outliers_mask():
    rng = np.random.default_rng(1)
    data = np.stack((rng.random(50) + 1, -3.2 + 0.01 * rng.standard_normal(50))).T
    data[7, 1] = 5.0   # a wild block energy
    data[21, 1] = -40.0
    clean, mask = stat_utils.reject_outliers(data, 1)
    target = data[:, 1]
    d = np.abs(target - np.median(target))
    q1, q3 = np.percentile(target, [25, 75])
    disp = max(np.median(d), (q3 - q1) / 1.349, 1e-5)
    assert np.array_equal(mask, d / disp < 10.0)
    assert not mask[7] and not mask[21] and mask.sum() == 48 and clean.shape == (48, 2)
