"""Grouped batches (afq_batch_*): the phaseless steps of several solves of
different sizes in grouped launches, the tensor-core contractions as
persistent grouped kernels over (solve, tile) work lists.  Every solve's
walkers, weights, scalars and block energies must equal its own block graph
replayed alone, bit for bit (the same kernels, tiles and summation orders),
eagerly and from a captured graph, for restricted and unrestricted walkers."""

import pytest
import torch

from ad_afqmc_b200.synthetic import make_system
from tests._helpers import device_system

pytestmark = pytest.mark.gpu

SHAPES = [  # norb, nelec, nchol, walkers, seed, trial
    (24, (6, 6), 96, 32, 11, "rhf"),
    (40, (10, 10), 180, 48, 12, "rhf"),
    (30, (8, 7), 140, 16, 13, "uhf"),
    (64, (16, 16), 300, 70, 14, "rhf"),
    (17, (4, 4), 70, 9, 15, "rhf"),
]


def _block(n, no, g, W, seed, tr, S=4, precision="mixed"):
    from ad_afqmc_b200.graphs import BlockGraph

    sys_ = make_system(n, no, g, seed=seed, trial=tr, chol_scale=0.25)
    wt = "restricted" if tr == "rhf" else "unrestricted"
    d_trial, d_ham, d_wave, d_prop, ham = device_system(sys_, wt, 0.005, W, precision=precision)
    pd = d_prop.init_prop_data(d_trial, d_wave, d_ham, seed)
    return BlockGraph(ham, d_ham, d_prop, d_trial, d_wave, pd, n_prop_steps=S)


def _state(b):
    return [t.clone() for t in b.tensors] + [b.pd["weights"].clone(), b.pd["overlaps"].clone(),
                                             b.pd["_scalars"][:3].clone(), b.block_out.clone()]


@pytest.mark.parametrize("graph", [False, True])
def test_grouped_batch_equals_solves_alone(graph):
    from ad_afqmc_b200.graphs import GroupedBatchGraph

    nblocks = 3
    alone, alone_launches = [], 0
    for sh in SHAPES:
        b = _block(*sh).capture(warmup=0)
        alone_launches += b.launches_per_block
        for _ in range(nblocks):
            b.replay()
        torch.cuda.synchronize()
        b.check_status()
        alone.append(_state(b))
    blocks = [_block(*sh) for sh in SHAPES]
    gb = GroupedBatchGraph(blocks, n_streams=4)
    if graph:
        gb.capture(warmup=0)
        for _ in range(nblocks):
            gb.replay()
    else:
        for _ in range(nblocks):
            gb.body()
    torch.cuda.synchronize()
    gb.check_status()
    for b, ref in zip(blocks, alone):
        for x, y in zip(_state(b), ref):
            assert torch.equal(x, y)
    # fewer launches than the solves' own blocks together
    assert 0 < gb.launches_per_block < alone_launches


def test_grouped_batch_rejects_fp64_and_mismatched_blocks():
    from ad_afqmc_b200 import _lib
    from ad_afqmc_b200.graphs import GroupedBatchGraph

    with pytest.raises(_lib.AfqError):
        GroupedBatchGraph([_block(24, (6, 6), 96, 8, 3, "rhf", precision="fp64")])
    with pytest.raises(_lib.AfqError):
        GroupedBatchGraph([_block(24, (6, 6), 96, 8, 3, "rhf", S=2), _block(24, (6, 6), 96, 8, 4, "rhf", S=3)])
