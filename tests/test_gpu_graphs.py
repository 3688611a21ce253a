"""CUDA-graph blocks: a replay equals the eagerly executed block body, and a
batch of independent solves recorded into one graph reproduces each solve run
alone, bit for bit."""

import numpy as np
import pytest
import torch

from ad_afqmc_b200.synthetic import make_system
from tests._helpers import device_system

pytestmark = pytest.mark.gpu


def _solve(norb, nocc, nchol, W, seed, precision="fp64", trial="rhf"):
    from ad_afqmc_b200.graphs import BlockGraph

    sys_ = make_system(norb, nocc, nchol, seed=seed, trial=trial, chol_scale=0.25)
    wt = "restricted" if trial == "rhf" else "unrestricted"
    d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, wt, 0.005, W, precision=precision)
    pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, seed)
    return BlockGraph(ham, d_ham, d_prop, d_trial, d_wave, pd, n_prop_steps=4)


def _state(b):
    return [t.clone() for t in b.tensors] + [b.pd["weights"].clone(), b.pd["_scalars"][:3].clone()]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_equals_eager(precision):
    a = _solve(24, (6, 6), 96, 32, 5, precision)
    b = _solve(24, (6, 6), 96, 32, 5, precision)
    ea = []
    for _ in range(3):
        a.body()
        ea.append(float(a.block_out[0]))
    b.capture(warmup=0)
    eb = []
    for _ in range(3):
        eb.append(float(b.replay()[0]))
    torch.cuda.synchronize()
    assert ea == eb
    for x, y in zip(_state(a), _state(b)):
        assert torch.equal(x, y)


def test_batch_graph_equals_solves_alone():
    from ad_afqmc_b200.graphs import BatchGraph

    shapes = [(24, (6, 6), 96, 32, 11), (40, (10, 10), 180, 48, 12), (30, (8, 7), 140, 16, 13)]
    alone, mixed = [], []
    for (n, no, g, W, seed) in shapes:
        tr = "rhf" if no[0] == no[1] else "uhf"
        b = _solve(n, no, g, W, seed, "fp64", tr).capture(warmup=0)
        for _ in range(2):
            b.replay()
        torch.cuda.synchronize()
        alone.append(_state(b))
    blocks = []
    for (n, no, g, W, seed) in shapes:
        tr = "rhf" if no[0] == no[1] else "uhf"
        blocks.append(_solve(n, no, g, W, seed, "fp64", tr))
    batch = BatchGraph(blocks, n_streams=3).capture(warmup=0)
    for _ in range(2):
        batch.replay()
    torch.cuda.synchronize()
    for b, ref in zip(blocks, alone):
        for x, y in zip(_state(b), ref):
            assert torch.equal(x, y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_fed_blocks_equal_device_fields(precision):
    """A block recorded with external_fields=True and fed the same fields from
    pinned host memory (HostFieldBlocks: uploads overlapped with the previous
    block) gives the block energy and weight of the block that drew them on
    the device, bit for bit, over several blocks (no comb, whose zeta comes
    from the device stream)."""
    from ad_afqmc_b200 import graphs

    def parts():
        sys_ = make_system(24, (6, 6), 96, seed=9, trial="rhf", chol_scale=0.25)
        d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, "restricted", 0.005, 32, precision=precision)
        pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, 9)
        return ham, d_ham, d_prop, d_trial, d_wave, pd

    a = graphs.BlockGraph(*parts(), n_prop_steps=4, reconfigure=False).capture(warmup=0)
    b = graphs.BlockGraph(*parts(), n_prop_steps=4, reconfigure=False, external_fields=True)
    n = 4
    host = [torch.empty(a.fields.shape, dtype=torch.float64).pin_memory() for _ in range(n)]
    ea = []
    for k in range(n):
        ea.append(a.replay()[:2].cpu().numpy().copy())
        host[k].copy_(a.fields.cpu())
    b.fields.copy_(host[0])
    b.capture(warmup=0)
    runner = graphs.HostFieldBlocks(b)
    runner.upload(host[0])
    eb = [runner.run(host[k + 1] if k + 1 < n else None)[:2] for k in range(n)]
    for x, y in zip(ea, eb):
        assert np.array_equal(x, y)
    assert runner.h2d_bytes == host[0].numel() * 8
