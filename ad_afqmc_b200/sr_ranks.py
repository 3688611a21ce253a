"""Stochastic reconfiguration across ranks (one process per GPU).

The reference (sr.py:52-153) gathers every rank's walkers and weights on rank
0, combs there and scatters the result back: 2 x R x W walker matrices cross
the network per reconfiguration, all through rank 0.  Here:

1. the weights are all-gathered (R x W doubles), so every rank holds the same
   global weights in rank order;
2. every rank combs them with the rank-0 arithmetic (``afq_comb_indices_ranks``
   on the device, bit-exact), so all ranks agree on which global walker fills
   each of the R x W slots without any further message;
3. only the walkers that change rank move, in one all-to-all with per-rank
   split sizes; a walker that stays is copied locally.

Slot k of rank q receives global walker idx[q W + k], exactly as rank q's
part of the reference's Scatter, so results are identical to the reference's
gather/comb/scatter.  The collectives run on a ``torch.distributed`` group
(NCCL for CUDA tensors, gloo for CPU ones).
"""

from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import _lib

CombFn = Callable[[torch.Tensor, int, int, float], Tuple[torch.Tensor, torch.Tensor]]


def comb_device(weights_all: torch.Tensor, n_per_rank: int, n_ranks: int,
                zeta: float) -> Tuple[torch.Tensor, torch.Tensor]:
    """Global comb of the gathered weights on the GPU (afq_comb_indices_ranks):
    (indices (R W,) int64 on the host, new weights (R W,) on the device)."""
    w = weights_all.to(torch.float64).contiguous()
    if not w.is_cuda:
        raise _lib.AfqError("comb_device needs CUDA weights (the walker path has no CPU fallback)")
    idx = torch.empty(w.numel(), dtype=torch.int32, device=w.device)
    wn = torch.empty_like(w)
    _lib.check(_lib.lib().afq_comb_indices_ranks(w.data_ptr(), int(n_per_rank), int(n_ranks),
                                                 float(zeta), wn.data_ptr(), idx.data_ptr(),
                                                 _lib.stream_handle()), "afq_comb_indices_ranks")
    return idx.to(torch.int64).cpu(), wn


def exchange_plan(idx: np.ndarray, W: int, R: int, rank: int):
    """Who sends what to whom, from the global slot -> walker indices.

    Returns (send_local, send_counts, recv_counts, recv_slots): send_local is
    this rank's local walker indices in the order they are sent (grouped by
    destination rank, slot order within a destination); recv_slots[p] are
    this rank's slots filled by source rank p, in the order p sends them.
    """
    idx = np.asarray(idx, dtype=np.int64).reshape(R, W)
    src_rank = idx // W
    send_local: List[np.ndarray] = []
    send_counts: List[int] = []
    for q in range(R):
        mine = idx[q][src_rank[q] == rank] - rank * W
        send_local.append(mine)
        send_counts.append(int(mine.size))
    recv_slots = [np.nonzero(src_rank[rank] == p)[0] for p in range(R)]
    recv_counts = [int(s.size) for s in recv_slots]
    return np.concatenate(send_local), send_counts, recv_counts, recv_slots


def _as_rows(t: torch.Tensor) -> torch.Tensor:
    """(W, ...) complex or real -> (W, n) float64 rows (a view when possible)."""
    if t.is_complex():
        t = torch.view_as_real(t)
    return t.reshape(t.shape[0], -1)


def reconfigure_across_ranks(walker_arrays: Sequence[torch.Tensor], weights: torch.Tensor, zeta: float,
                             group: Optional[dist.ProcessGroup] = None,
                             comb: Optional[CombFn] = None) -> Tuple[List[torch.Tensor], torch.Tensor]:
    """Global reconfiguration of R ranks x W walkers.

    walker_arrays: this rank's walker tensors, each (W, ...) (one for restricted
    walkers, two for unrestricted); weights (W,).  ``zeta`` must be the same on
    every rank (the reference draws it from the shared key).  Returns the new
    walker tensors (same shapes) and new weights (all equal to the global
    average weight).  ``comb`` defaults to the device comb."""
    R = dist.get_world_size(group)
    rank = dist.get_rank(group)
    W = int(weights.numel())
    comb = comb or comb_device
    w = weights.reshape(-1).to(torch.float64).contiguous()
    gathered = [torch.empty_like(w) for _ in range(R)]
    dist.all_gather(gathered, w, group=group)
    idx, w_new = comb(torch.cat(gathered), W, R, zeta)
    idx_np = idx.cpu().numpy() if isinstance(idx, torch.Tensor) else np.asarray(idx)
    send_local, send_counts, recv_counts, recv_slots = exchange_plan(idx_np, W, R, rank)
    dev = walker_arrays[0].device
    send_index = torch.as_tensor(send_local, dtype=torch.long, device=dev)
    outs = []
    for arr in walker_arrays:
        rows = _as_rows(arr)
        send_buf = rows.index_select(0, send_index).contiguous()
        recv_buf = torch.empty(sum(recv_counts), rows.shape[1], dtype=rows.dtype, device=dev)
        dist.all_to_all_single(recv_buf, send_buf, recv_counts, send_counts, group=group)
        new_rows = torch.empty_like(rows)
        off = 0
        for p in range(R):
            n = recv_counts[p]
            if n:
                slots = torch.as_tensor(recv_slots[p], dtype=torch.long, device=dev)
                new_rows.index_copy_(0, slots, recv_buf[off:off + n])
            off += n
        new = new_rows.reshape(_as_rows_shape(arr))
        outs.append(torch.view_as_complex(new) if arr.is_complex() else new)
    w_mine = w_new.reshape(R, W)[rank].to(weights.dtype).to(weights.device).contiguous()
    return outs, w_mine


def _as_rows_shape(t: torch.Tensor):
    return tuple(t.shape) + ((2,) if t.is_complex() else ())
