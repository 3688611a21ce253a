"""Device comb of the reconfiguration across ranks (afq_comb_indices_ranks):
indices and weights bit-exact against the rank-0 arithmetic of sr.py:52-153,
for several rank counts; one rank reproduces the single-rank global mode."""

import numpy as np
import pytest
import torch

from oracle import afqmc_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_per_rank,n_ranks", [(5, 1), (5, 3), (64, 2), (512, 4), (2048, 8)])
@pytest.mark.parametrize("zeta", [0.0, 0.4375, 0.999])
def test_comb_indices_ranks_bit_exact(n_per_rank, n_ranks, zeta):
    from ad_afqmc_b200.sr_ranks import comb_device

    rng = np.random.default_rng(n_per_rank * 10 + n_ranks)
    w = rng.random(n_per_rank * n_ranks) * 3.0
    w[rng.random(w.size) < 0.25] = 0.0
    idx_d, w_d = comb_device(torch.as_tensor(w, device="cuda"), n_per_rank, n_ranks, zeta)
    idx_o, w_o = orc.sr_indices_global(w, zeta, n_ranks=n_ranks)
    assert np.array_equal(idx_d.numpy(), idx_o)
    assert np.array_equal(w_d.cpu().numpy(), w_o)


def test_one_rank_equals_single_rank_global_mode():
    from ad_afqmc_b200.sr_ranks import comb_device
    from ad_afqmc_b200.walkers import RHFWalkers

    rng = np.random.default_rng(4)
    W = 37
    w = rng.random(W)
    walkers = RHFWalkers(rng.standard_normal((W, 6, 2)) + 0j)
    new, w_new = walkers.stochastic_reconfiguration_global(torch.as_tensor(w, device="cuda"), 0.61)
    idx, w_d = comb_device(torch.as_tensor(w, device="cuda"), W, 1, 0.61)
    assert torch.equal(new.data, walkers.data[idx.cuda()])
    assert torch.equal(w_new, w_d)
