"""The serving loop: each fragment's result is the same solved alone and in
the mix (bit for bit), and the loop admits, advances and completes every
request."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _requests():
    from ad_afqmc_b200.serving import Request
    from ad_afqmc_b200.synthetic import make_system

    specs = [(30, 8, 140, 64, 101, 0.00), (46, 12, 200, 96, 102, 0.01), (38, 10, 170, 80, 103, 0.02),
             (52, 13, 230, 64, 104, 0.03)]
    out = []
    for i, (n, no, g, w, seed, t) in enumerate(specs):
        out.append(Request(i, make_system(n, (no, no), g, seed, "rhf", chol_scale=0.25), w, seed, t))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_identical_alone_and_in_the_mix(precision):
    from ad_afqmc_b200.serving import Server

    reqs = _requests()
    srv = Server(precision, n_prop_steps=4, min_blocks=3, max_blocks=5, target_error=-1.0)
    mixed = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert sorted(mixed) == [0, 1, 2, 3]
    for req in reqs:
        alone = srv.run([req], realtime=False)[0]
        assert alone.block_energies == mixed[req.rid].block_energies
        assert alone.n_blocks == 5


def test_admission_respects_memory_budget():
    from ad_afqmc_b200.serving import Server, footprint_bytes

    reqs = _requests()
    fp = max(footprint_bytes(r, "mixed") for r in reqs)
    # room for about two solves at a time: all still complete, in arrival order of admission
    srv = Server("mixed", hbm_budget_gb=2.5 * fp / 1e9, n_prop_steps=3, min_blocks=2, max_blocks=3,
                 target_error=-1.0)
    res = srv.run(reqs, realtime=False)
    assert len(res) == 4
    admitted = sorted(res, key=lambda r: r.admitted)
    assert [r.rid for r in admitted] == [0, 1, 2, 3]
