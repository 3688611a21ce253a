"""Constructor signatures of the drop-in trial classes (CPU, no device).

The reference declares its trials as dataclasses whose fields, in order, are
norb, nelec, n_opt_iter, n_chunks, projector (rhf wavefunctions.py:1053-1057,
uhf :1251-1255, rhf_lno inherits rhf's, :6871); its call sites build them
positionally (tests/test_propagation.py:16, :41) and with keywords
(launch_script.py:379-393, :638).  These tests build the trials the same ways.
"""

import dataclasses

import pytest

from ad_afqmc_b200 import launch_script, wavefunctions

REFERENCE_FIELDS = ["norb", "nelec", "n_opt_iter", "n_chunks", "projector"]


@pytest.mark.parametrize("cls", [wavefunctions.rhf, wavefunctions.uhf, wavefunctions.rhf_lno])
def test_field_order_matches_reference(cls):
    assert dataclasses.is_dataclass(cls)
    assert [f.name for f in dataclasses.fields(cls)] == REFERENCE_FIELDS
    defaults = {f.name: f.default for f in dataclasses.fields(cls)}
    assert defaults["n_opt_iter"] == 30
    assert defaults["n_chunks"] == 1
    assert defaults["projector"] is None


def test_positional_construction():
    t = wavefunctions.rhf(10, (5, 5), 20, 2)
    assert (t.norb, t.nelec, t.n_opt_iter, t.n_chunks, t.projector) == (10, (5, 5), 20, 2, None)
    u = wavefunctions.uhf(10, (3, 2), 30)
    assert (u.norb, u.nelec, u.n_opt_iter, u.n_chunks) == (10, (3, 2), 30, 1)
    assert wavefunctions.rhf(6, (3, 3), 30).n_chunks == 1


def test_keyword_construction_as_launch_script():
    options = {"n_chunks": 4, "symmetry_projector": None}
    t = wavefunctions.rhf(10, (5, 5), n_chunks=options["n_chunks"],
                          projector=options["symmetry_projector"])
    u = wavefunctions.uhf(10, (3, 2), n_chunks=options["n_chunks"],
                          projector=options["symmetry_projector"])
    lno = wavefunctions.rhf_lno(10, (5, 5), n_chunks=options["n_chunks"])
    assert t.n_chunks == u.n_chunks == lno.n_chunks == 4
    assert wavefunctions.uhf(10, (3, 2), n_opt_iter=30).n_opt_iter == 30


def test_rhf_requires_equal_spins():
    with pytest.raises(AssertionError):
        wavefunctions.rhf(10, (3, 2))


def test_trials_are_hashable():
    # the reference defines __hash__ on every trial (wavefunctions.py:1234, 1498, 6925)
    a = wavefunctions.rhf(10, (5, 5))
    b = wavefunctions.rhf(10, (5, 5))
    assert hash(a) == hash(b)
    assert hash(wavefunctions.uhf(10, (3, 2))) == hash(wavefunctions.uhf(10, (3, 2)))
    assert len({a, b}) == 1


def test_set_trial_passes_n_chunks():
    import numpy as np

    opts = launch_script.read_options({"n_chunks": 2, "trial": "uhf", "walker_type": "unrestricted"})
    mo = np.stack([np.eye(6), np.eye(6)])
    trial, wave_data = launch_script.set_trial(opts, mo, 6, (3, 2))
    assert isinstance(trial, wavefunctions.uhf)
    assert trial.n_chunks == 2 and trial.projector is None
    assert wave_data["mo_coeff"][0].shape == (6, 3) and wave_data["mo_coeff"][1].shape == (6, 2)
