"""Host-side serving logic: the reference LNO stop rule and the footprint sizes
(no GPU needed)."""

import numpy as np


def test_sem_stop_follows_reference_schedule():
    """driver.py:376-389: checked after block n when n % max(n_blocks // 5, 1) == 0
    and n > 4; SEM = std(E[:n+1]) / sqrt(n+1)."""
    from ad_afqmc_b200.serving import sem_stop

    rng = np.random.default_rng(0)
    e = -10.0 + 1e-3 * rng.standard_normal(40)
    checked = []
    for n in range(40):
        stop, sem = sem_stop(e[: n + 1], 40, 1e-12)
        if sem is not None:
            checked.append(n)
            assert np.isclose(sem, np.std(e[: n + 1]) / np.sqrt(n + 1))
            assert not stop
    assert checked == [8, 16, 24, 32]
    # a loose target stops at the first check
    assert sem_stop(e[:9], 40, 1.0)[0]
    assert not sem_stop(e[:8], 40, 1.0)[0]
    # fewer than 5 blocks per check interval: every block after the fourth
    assert [n for n in range(12) if sem_stop(e[: n + 1], 3, 1.0)[1] is not None] == list(range(5, 12))


def test_footprint_grows_with_size():
    from ad_afqmc_b200.serving import Request, footprint_bytes
    from ad_afqmc_b200.synthetic import make_system

    small = Request(0, make_system(30, (8, 8), 120, 1, "rhf"), 64, 1)
    large = Request(1, make_system(60, (15, 15), 300, 1, "rhf"), 128, 1)
    fs, fl = footprint_bytes(small, "mixed"), footprint_bytes(large, "mixed")
    assert 0 < fs < fl
    # the chol matrix alone (G x N^2 doubles) is a lower bound
    assert fl > 300 * 60 * 60 * 8


def test_fragment_chol_scale():
    from ad_afqmc_b200.synthetic import fragment_chol_scale

    assert np.isclose(fragment_chol_scale(100), 0.035)
    assert fragment_chol_scale(40) > fragment_chol_scale(250)
