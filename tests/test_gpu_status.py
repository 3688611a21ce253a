"""Device-side wait timeouts surface as a status on the host.

A bounded mbarrier wait is made to run out on purpose through the
afq_test_wait_timeout hook (one thread waits on an mbarrier that nothing
arrives at; no copy or MMA is in flight, so nothing faults and nothing hangs).
The flag it sets must come back as AFQ_ERR_TIMEOUT from afq_check_status,
as an AfqError from the sampler and from a replayed block graph, and must be
cleared once read.  Normal blocks on the tensor-core path leave it clear."""

import ctypes as C

import pytest
import torch

from ad_afqmc_b200 import _lib, sampling
from ad_afqmc_b200.synthetic import make_system
from tests._helpers import device_system

pytestmark = pytest.mark.gpu


def _setup(precision="mixed", W=16):
    sys_ = make_system(24, (6, 6), 96, seed=77, trial="rhf", chol_scale=0.25)
    trial, ham_data, wave, prop, ham = device_system(sys_, "restricted", 0.005, W, precision=precision)
    pd = prop.init_prop_data(trial, wave, ham_data, 3)
    eng = prop.engine(ham_data, trial, wave)
    return trial, ham_data, wave, prop, ham, pd, eng


def _trip(eng, polls=64):
    _lib.check(_lib.lib().afq_test_wait_timeout(C.byref(eng.dims), eng.work.data_ptr(), eng.work_bytes,
                                                polls, _lib.stream_handle()), "afq_test_wait_timeout")


def test_check_status_reports_and_clears():
    *_, eng = _setup()
    lib = _lib.lib()
    args = (C.byref(eng.dims), eng.work.data_ptr(), eng.work_bytes)
    assert lib.afq_check_status(*args, _lib.stream_handle()) == _lib.AFQ_OK
    _trip(eng)
    assert lib.afq_check_status(*args, _lib.stream_handle()) == _lib.AFQ_ERR_TIMEOUT
    assert lib.afq_check_status(*args, _lib.stream_handle()) == _lib.AFQ_OK  # cleared when read
    assert int(eng.status_flag().item()) == 0
    # argument checks before any device access
    assert lib.afq_test_wait_timeout(*args, 0, _lib.stream_handle()) == 6
    assert lib.afq_check_status(C.byref(eng.dims), None, eng.work_bytes, _lib.stream_handle()) == 2
    assert lib.afq_check_status(C.byref(eng.dims), eng.work.data_ptr(), 8, _lib.stream_handle()) == 4


def test_sampler_raises_on_timeout_then_recovers():
    trial, ham_data, wave, prop, ham, pd, eng = _setup()
    smp = sampling.sampler(n_prop_steps=2, n_ene_blocks=1, n_sr_blocks=1, n_blocks=1)
    e, pd = smp.propagate_phaseless(ham, ham_data, prop, pd, trial, wave)  # clean block: no error
    assert torch.isfinite(e)
    _trip(eng)
    with pytest.raises(_lib.AfqError, match="timed out"):
        smp.propagate_phaseless(ham, ham_data, prop, pd, trial, wave)
    e, pd = smp.propagate_phaseless(ham, ham_data, prop, pd, trial, wave)
    assert torch.isfinite(e)


def test_block_graph_reports_timeout():
    from ad_afqmc_b200.graphs import BlockGraph

    trial, ham_data, wave, prop, ham, pd, eng = _setup()
    bg = BlockGraph(ham, ham_data, prop, trial, wave, pd, n_prop_steps=2).capture(warmup=1)
    bg.replay()
    bg.check_status()  # tensor-core blocks leave the flag clear
    _trip(eng)
    bg.replay()
    with pytest.raises(_lib.AfqError, match="timed out"):
        bg.check_status()
    bg.replay()
    bg.check_status()
