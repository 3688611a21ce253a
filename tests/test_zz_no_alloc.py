"""The allocation-free overlap entry point (afq_calc_overlap_static).

Callers that cannot allocate device memory (a host framework that owns the
GPU memory pool, such as an XLA custom call inside a JAX program, or code
recording into a CUDA graph under a capture mode that forbids allocation)
use afq_calc_overlap_static, whose scratch is a fixed array in the library's
device image.  This file runs last (pytest collects files in name order) so
that a failure here cannot hide other results; it also passes on its own in a
fresh process, where its first call performs the one-time device set-up.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from ad_afqmc_b200 import _lib
from ad_afqmc_b200.synthetic import make_system

pytestmark = pytest.mark.gpu

STATIC_MAX_WALKERS = 8192


def _static_overlap(trial, walkers, wave_data):
    from ad_afqmc_b200.wavefunctions import _ptrs

    mos = trial._mo_list(wave_data)
    d = trial._dims(walkers)
    out = torch.empty(walkers.n_walkers, dtype=torch.complex128, device="cuda")
    rc = _lib.lib().afq_calc_overlap_static(C.byref(d), _lib.pair(mos[0].data_ptr(), mos[-1].data_ptr()),
                                            _ptrs(walkers), out.data_ptr(), _lib.stream_handle())
    _lib.check(rc, "afq_calc_overlap_static")
    return out


@pytest.mark.parametrize("kind", ["rhf", "uhf"])
def test_static_overlap_matches_workspace_path_twice(kind):
    from ad_afqmc_b200 import wavefunctions
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers

    rng = np.random.default_rng(17)
    if kind == "rhf":
        sys_ = make_system(40, (10, 10), 60, seed=3, trial="rhf")
        trial = wavefunctions.rhf(40, (10, 10))
    else:
        sys_ = make_system(40, (11, 9), 60, seed=4, trial="uhf")
        trial = wavefunctions.uhf(40, (11, 9))
    wave = sys_.wave_data()
    for call in range(2):  # two calls in a row on the shared scratch
        W = 300 + 37 * call
        if kind == "rhf":
            w = RHFWalkers(sys_.mo_coeff[None] + 0.3 * (rng.standard_normal((W, 40, 10))
                                                         + 1j * rng.standard_normal((W, 40, 10))))
        else:
            w = UHFWalkers([m[None] + 0.3 * (rng.standard_normal((W, 40, m.shape[1]))
                                             + 1j * rng.standard_normal((W, 40, m.shape[1])))
                            for m in sys_.mo_coeff])
        ref = trial.calc_overlap(w, wave)
        got = _static_overlap(trial, w, wave)
        torch.cuda.synchronize()
        assert torch.allclose(got, ref, rtol=1e-12, atol=0), call


@pytest.mark.parametrize("kind", ["rhf", "uhf"])
def test_static_overlap_matches_oracle_at_capacity(kind):
    """Exactly the capacity (8192 walkers), against the NumPy oracle's
    determinants, not only against the workspace entry point."""
    from ad_afqmc_b200 import wavefunctions
    from ad_afqmc_b200.walkers import RHFWalkers, UHFWalkers
    from oracle import afqmc_oracle as orc

    rng = np.random.default_rng(23)
    W, N = STATIC_MAX_WALKERS, 12
    if kind == "rhf":
        sys_ = make_system(N, (4, 4), 20, seed=5, trial="rhf")
        trial, o_trial = wavefunctions.rhf(N, (4, 4)), orc.RHFTrial(N, (4, 4))
        host = sys_.mo_coeff[None] + 0.3 * (rng.standard_normal((W, N, 4)) + 1j * rng.standard_normal((W, N, 4)))
        w = RHFWalkers(host.copy())
    else:
        sys_ = make_system(N, (5, 3), 20, seed=6, trial="uhf")
        trial, o_trial = wavefunctions.uhf(N, (5, 3)), orc.UHFTrial(N, (5, 3))
        host = [m[None] + 0.3 * (rng.standard_normal((W, N, m.shape[1])) + 1j * rng.standard_normal((W, N, m.shape[1])))
                for m in sys_.mo_coeff]
        w = UHFWalkers([h.copy() for h in host])
    wave = sys_.wave_data()
    ref = o_trial.calc_overlap(host, wave)
    for _ in range(2):
        got = _static_overlap(trial, w, wave).cpu().numpy()
        assert np.allclose(got, ref, rtol=1e-10, atol=0)


def test_static_overlap_rejects_too_many_walkers():
    from ad_afqmc_b200 import wavefunctions
    from ad_afqmc_b200.wavefunctions import _ptrs
    from ad_afqmc_b200.walkers import RHFWalkers

    trial = wavefunctions.rhf(4, (2, 2))
    w = RHFWalkers(torch.zeros(STATIC_MAX_WALKERS + 1, 4, 2, dtype=torch.complex128, device="cuda"))
    d = trial._dims(w)
    mo = torch.eye(4, 2, dtype=torch.float64, device="cuda").contiguous()
    out = torch.empty(STATIC_MAX_WALKERS + 1, dtype=torch.complex128, device="cuda")
    rc = _lib.lib().afq_calc_overlap_static(C.byref(d), _lib.pair(mo.data_ptr(), mo.data_ptr()),
                                            _ptrs(w), out.data_ptr(), _lib.stream_handle())
    assert rc == 7  # AFQ_ERR_LIMIT
    assert b"static scratch" in _lib.lib().afq_status_string(rc)
