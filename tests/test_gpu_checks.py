"""The debug build (python -m ad_afqmc_b200.build --checks, loaded with
AFQ_CHECKS=1): the same results as the release build on one phaseless step,
and a host pointer handed to an entry point is rejected (AFQ_ERR_ARG) before
anything reaches the device.  Runs in a child process, since the library is
chosen when it is first loaded."""

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes as C, copy, sys
import numpy as np, torch
sys.path.insert(0, ROOT)
from ad_afqmc_b200 import _lib
assert _lib.LIB_PATH.endswith("libafqmc_b200_checks.so"), _lib.LIB_PATH
from ad_afqmc_b200.synthetic import make_system
from ad_afqmc_b200.propagation import make_state
from tests._helpers import device_system, near_trial_walkers, oracle_system, rel_err
from ad_afqmc_b200.walkers import RHFWalkers
sys_ = make_system(24, (6, 6), 96, seed=3, trial="rhf", chol_scale=0.25)
W = 8
rng = np.random.default_rng(1)
walkers = near_trial_walkers(rng, sys_.mo_coeff, W, eps=0.1)
fields = rng.standard_normal((W, 96))
o_trial, o_ham, o_wave, o_prop = oracle_system(sys_, "restricted", 0.005)
o_prop.n_walkers = W
o_pd = o_prop.init_prop_data(o_trial, o_wave, o_ham, init_walkers=walkers.copy())
o_pd = o_prop.propagate_constrained(o_trial, o_ham, o_pd, fields, o_wave)
for precision, tol in (("fp64", 1e-10), ("mixed", 1e-4)):
    trial, ham, wave, prop, _ = device_system(sys_, "restricted", 0.005, W, precision=precision)
    pd = prop.init_prop_data(trial, wave, ham, 0, init_walkers=RHFWalkers(walkers.copy()))
    pd = prop.propagate_constrained(trial, ham, pd, fields, wave)
    assert rel_err(pd["walkers"].data.cpu().numpy(), o_pd["walkers"]) < tol, precision
    eng = prop.engine(ham, trial, wave)
    eng.check_status()
    # a host array as the fields: rejected on the host
    host = np.ascontiguousarray(fields)
    st = make_state(pd)
    p, w, wb = eng.handle
    rc = _lib.lib().afq_propagate_constrained(C.byref(eng.dims), p, C.byref(st), host.ctypes.data, w, wb,
                                              _lib.stream_handle())
    assert rc == 6, rc
torch.cuda.synchronize()
print("CHECKS_OK")
"""


def test_debug_build_matches_and_rejects_host_pointers():
    lib = os.path.join(ROOT, "ad_afqmc_b200", "lib", "libafqmc_b200_checks.so")
    if not os.path.exists(lib):
        pytest.fail("the debug build is missing: python -m ad_afqmc_b200.build --checks")
    env = dict(os.environ, AFQ_CHECKS="1")
    r = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + CHILD], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "CHECKS_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
