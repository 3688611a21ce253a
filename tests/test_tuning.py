"""Tuning records (afq_set_tuning / afq_get_tuning): validation, effect on the
layout sizes, and the autotuner's cache (host side, no GPU)."""

import json

import pytest

from ad_afqmc_b200 import _lib


def _dims(norb=200, no=40, nchol=1000, W=512, precision=1):
    return _lib.make_dims(norb, (no, no), nchol, W, _lib.AFQ_RESTRICTED, _lib.AFQ_TRIAL_RHF, 6, precision,
                          0.005)


def test_defaults_reported():
    d = _dims()
    t = _lib.get_tuning(d).as_dict()
    assert t["fb_bn"] == 128 and t["vhs_bn"] == 128
    assert t["exch_bn"] == 80            # 2 No = 80 columns: one walker per tile, no padding
    assert t["f64_exch_bn"] == 80
    assert 1 <= t["fb_splitk"] <= 8
    assert t["max_stages"] == 0 and t["grid_cap"] == 0


def test_record_changes_choice_and_workspace_follows():
    d = _dims(W=256)
    _, w0 = _lib.sizes(d)
    try:
        _lib.set_tuning(d, _lib.afq_tuning.from_dict({"fb_splitk": 1, "exch_bn": 128, "vhs_bn": 64}))
        t = _lib.get_tuning(d).as_dict()
        assert (t["fb_splitk"], t["exch_bn"], t["vhs_bn"]) == (1, 128, 64)
        _, w1 = _lib.sizes(d)
        assert w1 != w0   # fewer split-K partials, different exchange partial sums
        # another shape is untouched
        assert _lib.get_tuning(_dims(W=128)).as_dict()["exch_bn"] == 80
    finally:
        _lib.set_tuning(d, None)
    assert _lib.sizes(d)[1] == w0


@pytest.mark.parametrize("rec", [{"fb_splitk": 9}, {"fb_bn": 96}, {"vhs_bn": 256}, {"max_stages": 1},
                                 {"exch_bn": 64},       # 2 No = 80 columns do not fit 64
                                 {"f64_exch_bn": 100}, {"grid_cap": -1},
                                 {"prop_chunk": 3}, {"vhs_chunk": 3}, {"qr_mode": 3},
                                 {"prop_bn": 40},       # not a compiled column tile
                                 {"prop_bn": -16}, {"prop_order": 2}, {"prop_epi_groups": 4}])
def test_invalid_records_rejected_and_not_registered(rec):
    d = _dims()
    before = _lib.get_tuning(d).as_dict()
    with pytest.raises(_lib.AfqError):
        _lib.set_tuning(d, _lib.afq_tuning.from_dict(rec))
    assert _lib.get_tuning(d).as_dict() == before


def test_fp64_exchange_tile_choices():
    d = _dims(no=62, precision=0, norb=70, nchol=90, W=3)
    assert _lib.get_tuning(d).as_dict()["f64_exch_bn"] == 160
    with pytest.raises(_lib.AfqError):
        _lib.set_tuning(d, _lib.afq_tuning.from_dict({"f64_exch_bn": 120}))
    d = _dims(no=20, precision=0, norb=70, nchol=90, W=3)
    try:
        for bn in (80, 120, 160):
            _lib.set_tuning(d, _lib.afq_tuning.from_dict({"f64_exch_bn": bn}))
            assert _lib.get_tuning(d).as_dict()["f64_exch_bn"] == bn
    finally:
        _lib.set_tuning(d, None)


def test_autotuner_cache_roundtrip(tmp_path):
    from ad_afqmc_b200.autotune import Autotuner, candidates, shape_key

    d = _dims()
    key = shape_key(d)
    assert key == "N200_na40_nb40_G1000_W512_wt0_tt0_p1"
    assert set(candidates(d)) >= {"vhs_bn", "fb_bn", "fb_splitk", "exch_bn", "max_stages"}
    assert "vhs_bn" not in candidates(_dims(precision=0))
    path = tmp_path / "t.json"
    tu = Autotuner(cache_path=str(path))
    tu.cache[key] = {"tuning": {"fb_splitk": 4}, "ms": 1.0, "ms_default": 1.2, "steps": 10}
    tu.save()
    assert json.loads(path.read_text())[key]["tuning"] == {"fb_splitk": 4}
    assert Autotuner(cache_path=str(path)).cache == tu.cache


def test_accumulation_and_tile_knobs_accepted():
    """The knobs that change how the mixed GEMMs accumulate K (prop_chunk,
    vhs_chunk: 2 = FP32 chunk sums), the propagator's column tile and the QR
    placement are registered and read back; 0 keeps the built-in choice."""
    d = _dims(W=64)
    try:
        rec = {"prop_chunk": 2, "vhs_chunk": 2, "prop_bn": 48, "qr_mode": 2}
        _lib.set_tuning(d, _lib.afq_tuning.from_dict(rec))
        t = _lib.get_tuning(d).as_dict()
        for k, v in rec.items():
            assert t[k] == v
    finally:
        _lib.set_tuning(d, None)
    t = _lib.get_tuning(d).as_dict()
    assert t["prop_chunk"] == 0 and t["vhs_chunk"] == 0 and t["prop_bn"] == 0 and t["qr_mode"] == 0
