"""Host-side block statistics (mirror of ad_afqmc/stat_utils.py:8-78).

These act on a handful of per-block scalars after they leave the device; the
serving loop's stop rule (energy standard error below a target) uses them.
"""

from __future__ import annotations

import numpy as np


def blocking_analysis(weights, energies, neql=0, printQ=False, writeBlockedQ=False):
    """stat_utils.py:8-64: weighted mean and plateau error of the blocked means."""
    weights = np.asarray(weights, dtype=np.float64)[neql:]
    energies = np.asarray(energies, dtype=np.float64)[neql:]
    n = weights.shape[0]
    we = weights * energies
    mean_energy = we.sum() / weights.sum()
    block_sizes = np.array([1, 2, 5, 10, 20, 50, 100, 200, 300, 400, 500, 1000, 10000])
    prev, plateau, errors = 0.0, None, []
    for i in block_sizes[block_sizes < n / 2.0]:
        nb = int(n // i)
        bw = np.add.reduceat(weights[: nb * i], np.arange(0, nb * i, i))
        be = np.add.reduceat(we[: nb * i], np.arange(0, nb * i, i)) / bw
        v1, v2 = bw.sum(), (bw**2).sum()
        mean = (bw * be).sum() / v1
        err = ((bw * (be - mean) ** 2).sum() / (v1 - v2 / v1) / (nb - 1)) ** 0.5
        errors.append(err)
        if writeBlockedQ:
            np.savetxt(f"samples_blocked_{i}.dat", np.stack((bw, be)).T)
        if printQ:
            print(f"  {i:5d}           {nb:6d}       {mean:.8e}       {err:.6e}")
        if err < 1.05 * prev and plateau is None:
            plateau = max(err, prev)
        prev = err
    if plateau is None and errors:
        plateau = 2 * errors[0]
    return mean_energy, plateau


def reject_outliers(data, obs, m=10.0, min_threshold=1e-5):
    """stat_utils.py:67-78."""
    target = data[:, obs]
    med = np.median(target)
    d = np.abs(target - med)
    mdev = np.median(d)
    q1, q3 = np.percentile(target, [25, 75])
    disp = max(mdev, (q3 - q1) / 1.349, min_threshold)
    mask = d / disp < m
    return data[mask], mask
