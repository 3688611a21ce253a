"""Reconfiguration across ranks (sr_ranks.py) on CPU ranks over gloo.

Each rank holds W walkers; after the exchange, rank q's walkers and weights
must equal rank q's part of the reference's gather -> rank-0 comb -> scatter
(sr.py:52-153) over all ranks' walkers, bit for bit.  The comb itself runs
here with the oracle (the device comb is checked against the same oracle in
tests/test_gpu_sr_ranks.py); what is tested is the exchange: the all-gather,
the plan and the all-to-all."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import afqmc_oracle as orc

W, N, NA, NB = 7, 5, 3, 2


def _rank_data(rank: int, seed: int):
    rng = np.random.default_rng(seed * 100 + rank)
    up = rng.standard_normal((W, N, NA)) + 1j * rng.standard_normal((W, N, NA))
    dn = rng.standard_normal((W, N, NB)) + 1j * rng.standard_normal((W, N, NB))
    w = rng.random(W) * 2.0
    w[rng.random(W) < 0.3] = 0.0  # killed walkers
    if seed % 2 == 0 and rank == 0:
        w[:] = 0.0                  # a rank with no surviving walker
    return up, dn, w


def _oracle_comb(weights_all, n_per_rank, n_ranks, zeta):
    idx, w_new = orc.sr_indices_global(weights_all.numpy(), zeta, n_ranks=n_ranks)
    assert n_per_rank * n_ranks == weights_all.numel()
    return torch.as_tensor(idx), torch.as_tensor(w_new)


def _worker(rank, world, port, seed, zeta, errors):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ad_afqmc_b200.sr_ranks import reconfigure_across_ranks

        up, dn, w = _rank_data(rank, seed)
        outs, w_new = reconfigure_across_ranks([torch.from_numpy(up), torch.from_numpy(dn)],
                                               torch.from_numpy(w), zeta, comb=_oracle_comb)
        # reference: gather everything, comb on "rank 0", scatter
        all_up = np.concatenate([_rank_data(r, seed)[0] for r in range(world)])
        all_dn = np.concatenate([_rank_data(r, seed)[1] for r in range(world)])
        all_w = np.concatenate([_rank_data(r, seed)[2] for r in range(world)])
        idx, avg = orc.sr_indices_global(all_w, zeta, n_ranks=world)
        mine = slice(rank * W, (rank + 1) * W)
        assert np.array_equal(outs[0].numpy(), all_up[idx][mine])
        assert np.array_equal(outs[1].numpy(), all_dn[idx][mine])
        assert np.array_equal(w_new.numpy(), avg[mine])
    except Exception as e:  # reported to the parent
        errors.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world,seed,zeta", [(2, 1, 0.37), (2, 2, 0.91), (3, 3, 0.05)])
def test_reconfiguration_across_ranks_matches_gather_scatter(world, seed, zeta):
    ctx = mp.get_context("spawn")
    errors = ctx.Queue()
    mp.start_processes(_worker, args=(world, _free_port(), seed, zeta, errors), nprocs=world,
                       start_method="spawn")
    assert errors.empty()


def test_exchange_plan_moves_only_crossing_walkers():
    from ad_afqmc_b200.sr_ranks import exchange_plan

    Wr, R = 4, 3
    idx = np.array([0, 0, 5, 11, 4, 4, 4, 9, 1, 2, 10, 10])  # slots of ranks 0, 1, 2
    for rank in range(R):
        send_local, send_counts, recv_counts, recv_slots = exchange_plan(idx, Wr, R, rank)
        assert sum(send_counts) == send_local.size
        assert sum(recv_counts) == Wr
        # what every rank receives from `rank` is what `rank` sends it
        for q in range(R):
            _, _, rc_q, _ = exchange_plan(idx, Wr, R, q)
            assert rc_q[rank] == send_counts[q]
    # rank 1 sends walker 1 (global 5) to rank 0 and walker 0 (global 4) three times to itself
    send_local, send_counts, _, _ = exchange_plan(idx, Wr, R, 1)
    assert send_counts == [1, 3, 0] and list(send_local) == [1, 0, 0, 0]
