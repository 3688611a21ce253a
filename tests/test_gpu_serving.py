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
    # the mix: set up on the worker thread while other solves run
    srv = Server(precision, n_prop_steps=4, n_eql=2, max_blocks=5, target_error=-1.0)
    mixed = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert sorted(mixed) == [0, 1, 2, 3]
    # alone: one slot, set up inline
    one = Server(precision, max_slots=1, n_prop_steps=4, n_eql=2, max_blocks=5, target_error=-1.0,
                 setup_thread=False)
    for req in reqs:
        alone = one.run([req], realtime=False)[0]
        assert alone.block_energies == mixed[req.rid].block_energies
        assert alone.n_blocks == 5


def test_admission_respects_memory_budget():
    from ad_afqmc_b200.serving import Server, footprint_bytes

    reqs = _requests()
    fp = max(footprint_bytes(r, "mixed") for r in reqs)
    # room for about two solves at a time: all still complete, in arrival order of admission
    srv = Server("mixed", hbm_budget_gb=2.5 * fp / 1e9, n_prop_steps=3, n_eql=1, max_blocks=3,
                 target_error=-1.0)
    res = srv.run(reqs, realtime=False)
    assert len(res) == 4
    admitted = sorted(res, key=lambda r: r.admitted)
    assert [r.rid for r in admitted] == [0, 1, 2, 3]


def test_stop_rule_ends_converged_solves_early():
    """With a loose target every solve stops at the first SEM check (block
    index max_blocks // 5 = 6 > 4, i.e. after 7 blocks); the blocking rule
    stops after min_blocks."""
    from ad_afqmc_b200.serving import Server

    reqs = _requests()[:2]
    res = Server("mixed", n_prop_steps=3, n_eql=1, max_blocks=30, target_error=10.0).run(reqs, realtime=False)
    assert all(r.converged and r.n_blocks == 7 for r in res)
    res = Server("mixed", n_prop_steps=3, n_eql=1, max_blocks=30, target_error=10.0, stop_rule="blocking",
                 min_blocks=5).run(reqs, realtime=False)
    assert all(r.converged and r.n_blocks == 5 for r in res)


def test_lno_fragments_served_identically_alone_and_in_the_mix():
    """LNO fragments (rhf_lno, orbital energy per block): same block and
    orbital energies alone and in the mix; the orbital energy is reported."""
    from ad_afqmc_b200.serving import Request, Server

    reqs = _requests()
    rng = np.random.default_rng(17)
    for r in reqs:
        p = rng.standard_normal((1, r.system.nelec[0]))
        r.prjlo = p / np.linalg.norm(p)
    srv = Server("mixed", n_prop_steps=3, n_eql=1, max_blocks=4, target_error=-1.0)
    mixed = {r.rid: r for r in srv.run(reqs, realtime=False)}
    one = Server("mixed", max_slots=1, n_prop_steps=3, n_eql=1, max_blocks=4, target_error=-1.0,
                 setup_thread=False)
    for req in reqs[:2]:
        alone = one.run([req], realtime=False)[0]
        assert alone.block_energies == mixed[req.rid].block_energies
        assert alone.orbE == mixed[req.rid].orbE
        assert np.isfinite(alone.orbE) and alone.orbE_err is not None
