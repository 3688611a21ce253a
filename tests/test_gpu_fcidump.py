"""The walker path on the reference's driver-test Hamiltonian, read back from
an FCIDUMP_chol directory written by this package (the decoded datasets are
committed in golden/fcidump_golden.npz; nothing here reads the reference).

* the trial determinant's energy on the device equals the HF energy
  computed from the datasets with plain NumPy (1e-10);
* two phaseless steps match the oracle (walker matrices 1e-10 relative);
* ``launch_script.run_afqmc`` with the options of the reference's driver
  test (tests/test_driver.py:74-86) gives an AFQMC energy that agrees with
  the reference's asserted value within the statistics of two independent
  runs (the reference's random stream cannot be reproduced), and lies below
  the HF energy.
"""

import copy
import json
import os

import numpy as np
import pytest

from ad_afqmc_b200 import fcidump, launch_script
from tests._helpers import device_system, near_trial_walkers, oracle_system, rel_err

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _np(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def calc_dir(tmp_path_factory):
    z = np.load(os.path.join(GOLD, "fcidump_golden.npz"))
    ds = {k[3:]: z[k] for k in z.files if k.startswith("ds_")}
    d = tmp_path_factory.mktemp("fcidump")
    n, g = int(ds["header"][1]), int(ds["header"][3])
    fcidump.write_fcidump(ds["hcore"].reshape(n, n), ds["hcore_mod"].reshape(n, n), ds["chol"].reshape(g, -1),
                          int(ds["header"][0]), n, float(ds["energy_core"]), int(ds["header"][2]),
                          filename=str(d / "FCIDUMP_chol"), mo_coeffs=[ds["mo_coeffs_up"], ds["mo_coeffs_dn"]])
    fcidump.write_mo_coeff(z["mo_coeff"], str(d))
    with open(os.path.join(GOLD, "fcidump_golden.json")) as f:
        meta = json.load(f)
    return str(d), float(z["e_uhf"]), meta


def test_trial_energy_on_device(calc_dir):
    from ad_afqmc_b200.walkers import UHFWalkers

    d, e_uhf, _ = calc_dir
    s = fcidump.system_from_fcidump(d, trial="uhf")
    trial, ham, wave, _, _ = device_system(s, "unrestricted", 0.01, 4)
    w = UHFWalkers([np.repeat(s.mo_coeff[k][None].astype(np.complex128), 4, axis=0) for k in range(2)])
    e = _np(trial.calc_energy(w, ham, wave))
    assert np.abs(e.real - e_uhf).max() < 1e-10
    assert np.allclose(_np(trial.calc_overlap(w, wave)), 1.0, atol=1e-12)


@pytest.mark.parametrize("tr,wt", [("uhf", "unrestricted"), ("rhf", "restricted"), ("rhf", "unrestricted")])
def test_two_steps_match_oracle(calc_dir, tr, wt):
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    d, _, _ = calc_dir
    s = fcidump.system_from_fcidump(d, trial=tr)
    W, dt = 16, 0.01
    rng = np.random.default_rng(5)
    mo = [s.mo_coeff, s.mo_coeff] if tr == "rhf" else s.mo_coeff
    if wt == "restricted":
        walkers = near_trial_walkers(rng, mo[0], W)
        dw = RHFWalkers(walkers.copy())
    else:
        walkers = [near_trial_walkers(rng, mo[0], W), near_trial_walkers(rng, mo[1], W)]
        dw = UHFWalkers([walkers[0].copy(), walkers[1].copy()])
    o_trial, o_ham, o_wave, o_prop = oracle_system(s, wt, dt)
    o_prop.n_walkers = W
    o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=copy.deepcopy(walkers))
    d_trial, d_ham, d_wave, d_prop, _ = device_system(s, wt, dt, W)
    d_pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 0, init_walkers=dw)
    assert abs(float(d_pd["e_estimate"]) - o_pd["e_estimate"]) < 1e-9
    for _ in range(2):
        f = rng.standard_normal((W, s.nchol))
        o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, f, o_wave)
        d_pd = d_prop.propagate_constrained(d_trial, d_ham, d_pd, f, d_wave)
        dd = d_pd["walkers"].data
        pairs = [(_np(dd), o_pd["walkers"])] if wt == "restricted" else \
            [(_np(dd[k]), o_pd["walkers"][k]) for k in range(2)]
        for a, b in pairs:
            for w in range(W):
                assert rel_err(a[w], b[w]) < 1e-10
        assert np.allclose(_np(d_pd["weights"]), o_pd["weights"], rtol=1e-10, atol=1e-13)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_run_afqmc_driver_options(calc_dir, precision):
    d, e_uhf, meta = calc_dir
    options = dict(meta["driver_options"], precision=precision)
    e, err = launch_script.run_afqmc(options, tmpdir=d)
    e_ref = meta["reference_values"]["afqmc_energy_1proc"][0]
    err = float(err) if err is not None and np.isfinite(err) else 0.0
    print(f"run_afqmc ({precision}): E = {e:.6f} +- {err:.6f} Ha; reference run {e_ref:.6f} Ha")
    # two independent stochastic runs of 50 walkers x 5000 steps: a few mHa apart at most
    assert abs(e - e_ref) < max(0.01, 5.0 * err), (e, err, e_ref)
    assert e < e_uhf - 0.05
    assert os.path.isfile(os.path.join(d, "samples_raw.dat"))


def test_run_afqmc_tight_statistics(calc_dir):
    """The energy of the reference's driver test at its own settings (50
    walkers, 10 blocks of 10 x 50 steps, UHF trial, seed 98 in the reference)
    averaged over 80 independent seeds, so that its standard error drops below
    0.3 mHa, compared at three combined standard errors with both energies the
    reference asserts (tests/test_driver.py:74-86, one rank, and :19-33, two
    ranks of 50 walkers).  Each reference value is a single run of its own
    random stream: its statistical error is the spread of single runs, which
    the 80 seeds measure directly (over sqrt(2) for the two-rank run, which
    has twice the walkers).  The walker count stays the reference's because
    the population-control bias depends on it."""
    d, e_uhf, meta = calc_dir
    base = dict(meta["driver_options"], precision="fp64")
    runs = np.array([launch_script.run_afqmc(dict(base, seed=1000 + k), tmpdir=d)[0] for k in range(80)])
    e_mean = float(runs.mean())
    s_single = float(runs.std(ddof=1))
    s_mean = s_single / np.sqrt(len(runs))
    print(f"80 runs at the reference settings: E = {e_mean:.6f} +- {s_mean:.6f} Ha "
          f"(single-run spread {s_single:.6f})")
    assert s_mean < 3e-4
    refs = [(meta["reference_values"]["afqmc_energy_1proc"][0], s_single),
            (meta["reference_values"]["afqmc_energy_2proc"][0], s_single / np.sqrt(2.0))]
    for e_ref, s_ref in refs:
        assert abs(e_mean - e_ref) < 3.0 * np.hypot(s_mean, s_ref), (e_mean, s_mean, e_ref, s_ref)


def test_save_walkers_and_metrics(calc_dir, tmp_path):
    """The reference's save_walkers option (driver.py:160-161, 985-992): one
    pickled host copy of the walker state per block, appended; and the JSON
    lines of per-block energies and weights."""
    import json
    import pickle

    d, _, meta = calc_dir
    metrics = str(tmp_path / "metrics.jsonl")
    options = dict(meta["driver_options"], precision="fp64", n_blocks=4, n_walkers=16,
                   save_walkers=True, metrics_file=metrics)
    launch_script.run_afqmc(options, tmpdir=d)
    states = []
    with open(os.path.join(d, "prop_data_0.bin"), "rb") as f:
        while True:
            try:
                states.append(pickle.load(f))
            except EOFError:
                break
    assert len(states) == 4
    for st in states:
        up, dn = st["walkers"]
        assert up.shape == (16, 6, 3) and dn.shape == (16, 6, 3)
        # orthonormalized walkers (QR) before the reconfiguration
        assert np.allclose(np.einsum("wpi,wpj->wij", up.conj(), up), np.eye(3)[None], atol=1e-10)
        assert st["weights"].shape == (16,)
    lines = [json.loads(x) for x in open(metrics)]
    assert [x["block"] for x in lines[:-1]] == [0, 1, 2, 3]
    assert lines[-1]["blocks"] == 4 and lines[-1]["walkers"] == 16
    assert all(np.isfinite(x["energy"]) for x in lines[:-1])
