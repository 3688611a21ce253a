"""FCIDUMP_chol input and output (CPU): the minimal HDF5 reader and writer,
read_fcidump / write_fcidump, and the run set-up from a calculation
directory.  Pinned to the reference's driver-test Hamiltonian
(tests/driver_test_files), whose decoded datasets are committed in
golden/fcidump_golden.npz by golden/make_fcidump_golden.py."""

import hashlib
import importlib.util
import json
import os
import struct

import numpy as np
import pytest

from ad_afqmc_b200 import fcidump, launch_script
from oracle import afqmc_oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_DIR = "/root/reference/tests/driver_test_files"


def _golden():
    z = np.load(os.path.join(GOLD, "fcidump_golden.npz"))
    ds = {k[3:]: z[k] for k in z.files if k.startswith("ds_")}
    with open(os.path.join(GOLD, "fcidump_golden.json")) as f:
        meta = json.load(f)
    return ds, z["mo_coeff"], float(z["e_uhf"]), meta


def _object_header_fn():
    spec = importlib.util.spec_from_file_location("make_fcidump_golden",
                                                  os.path.join(GOLD, "make_fcidump_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.object_header, mod.uhf_energy


def _write_dir(tmp_path, ds, mo):
    norb = int(ds["header"][1])
    fcidump.write_fcidump(ds["hcore"].reshape(norb, norb), ds["hcore_mod"].reshape(norb, norb),
                          ds["chol"].reshape(int(ds["header"][3]), -1), int(ds["header"][0]), norb,
                          float(ds["energy_core"]), int(ds["header"][2]),
                          filename=str(tmp_path / "FCIDUMP_chol"),
                          mo_coeffs=[ds["mo_coeffs_up"], ds["mo_coeffs_dn"]])
    fcidump.write_mo_coeff(mo, str(tmp_path))
    return str(tmp_path)


def test_golden_datasets_consistent():
    ds, mo, e_uhf, meta = _golden()
    assert sorted(ds) == ["chol", "energy_core", "hcore", "hcore_mod", "header", "mo_coeffs_dn", "mo_coeffs_up"]
    assert ds["header"].dtype == np.int64 and list(ds["header"]) == [6, 6, 0, 15]
    assert ds["energy_core"].shape == ()
    h1 = ds["hcore"].reshape(6, 6)
    chol = ds["chol"].reshape(15, 6, 6)
    assert np.abs(h1 - h1.T).max() < 1e-12
    assert np.abs(chol - chol.transpose(0, 2, 1)).max() < 1e-12
    assert np.array_equal(ds["mo_coeffs_up"], mo[0]) and np.array_equal(ds["mo_coeffs_dn"], mo[1])
    # the trial's HF energy sits above the reference's AFQMC energy by a correlation energy
    e_qmc = meta["reference_values"]["afqmc_energy_1proc"][0]
    assert 0.0 < e_uhf - e_qmc < 0.5


@pytest.mark.skipif(not os.path.isdir(REF_DIR), reason="reference checkout not present")
def test_reader_matches_reference_file():
    ds, _, _, meta = _golden()
    path = os.path.join(REF_DIR, "FCIDUMP_chol")
    with open(path, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == meta["sha256"]
    got = fcidump.read_hdf5_datasets(path)
    assert sorted(got) == sorted(ds)
    for k, v in ds.items():
        assert got[k].dtype == v.dtype and got[k].shape == v.shape and np.array_equal(got[k], v), k


def test_write_read_roundtrip(tmp_path):
    ds, mo, _, _ = _golden()
    d = _write_dir(tmp_path, ds, mo)
    got = fcidump.read_hdf5_datasets(os.path.join(d, "FCIDUMP_chol"))
    assert sorted(got) == sorted(ds)
    for k, v in ds.items():
        assert got[k].dtype == v.dtype and got[k].shape == v.shape and np.array_equal(got[k], v), k


def test_writer_object_headers_match_hdf5_library(tmp_path):
    """The writer's dataset headers are byte-identical to the ones the HDF5
    library wrote into the reference's file (data addresses aside)."""
    ds, mo, _, meta = _golden()
    object_header, _ = _object_header_fn()
    d = _write_dir(tmp_path, ds, mo)
    with open(os.path.join(d, "FCIDUMP_chol"), "rb") as f:
        raw = f.read()
    for name, hexed in meta["object_headers"].items():
        assert object_header(raw, name) == hexed, name


def test_read_fcidump_api(tmp_path):
    ds, mo, _, _ = _golden()
    d = _write_dir(tmp_path, ds, mo)
    h0, h1, chol, norb, nelec = fcidump.read_fcidump(d)
    assert float(h0) == float(ds["energy_core"])
    assert h1.shape == (6, 6) and chol.shape == (15, 6, 6) and norb == 6 and nelec == (3, 3)
    assert np.array_equal(chol.reshape(15, -1), ds["chol"].reshape(15, -1))
    with pytest.raises(AssertionError):
        fcidump.read_fcidump(str(tmp_path / "missing"))


@pytest.mark.parametrize("nelec,ms,expect", [(6, 0, (3, 3)), (7, 1, (4, 3)), (5, -1, (3, 2))])
def test_spin_split(tmp_path, nelec, ms, expect):
    rng = np.random.default_rng(3)
    n = 4
    h = rng.standard_normal((n, n))
    fcidump.write_fcidump(h + h.T, h + h.T, rng.standard_normal((3, n * n)), nelec, n, 0.5, ms,
                          filename=str(tmp_path / "FCIDUMP_chol"))
    assert fcidump.read_fcidump(str(tmp_path))[4] == expect


def test_dtypes_and_scalars(tmp_path):
    fn = str(tmp_path / "x.h5")
    data = {"a": np.arange(5, dtype=np.int32), "b": np.float32(2.5), "c": np.ones((2, 3), np.float32),
            "u": np.arange(3, dtype=np.uint16), "e": np.zeros((0,), np.float64), "s": np.int64(-7)}
    fcidump.write_hdf5_datasets(fn, data)
    got = fcidump.read_hdf5_datasets(fn)
    for k, v in data.items():
        v = np.asarray(v)
        assert got[k].dtype == v.dtype and got[k].shape == v.shape and np.array_equal(got[k], v), k
    with pytest.raises(ValueError):
        fcidump.write_hdf5_datasets(fn, {f"d{i}": np.zeros(1) for i in range(9)})
    with pytest.raises(ValueError):
        fcidump.write_hdf5_datasets(fn, {"z": np.zeros(2, np.complex128)})


def test_big_endian_and_non_hdf5_refused(tmp_path):
    fn = str(tmp_path / "x.h5")
    fcidump.write_hdf5_datasets(fn, {"a": np.arange(3, dtype=np.int64)})
    raw = bytearray(open(fn, "rb").read())
    # flip the byte-order bit of the one datatype message (class 0, version 1)
    p = raw.index(bytes([0x10, 0x08, 0, 0]) + struct.pack("<I", 8))
    raw[p + 1] |= 1
    open(fn, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="big-endian"):
        fcidump.read_hdf5_datasets(fn)
    open(fn, "wb").write(b"not hdf5 at all")
    with pytest.raises(ValueError):
        fcidump.read_hdf5_datasets(fn)


def test_ham_data_and_system(tmp_path):
    ds, mo, e_uhf, _ = _golden()
    d = _write_dir(tmp_path, ds, mo)
    ham, wave, nelec, norb = fcidump.ham_data_from_fcidump(d)
    assert ham["h1"].shape == (2, 6, 6) and ham["chol"].shape == (15, 36) and nelec == (3, 3)
    assert wave["mo_coeff"][0].shape == (6, 3) and wave["rdm1"].shape == (2, 6, 6)
    s = fcidump.system_from_fcidump(d, trial="uhf")
    assert s.trial == "uhf" and s.nchol == 15 and s.norb == 6
    # the oracle's UHF energy of the trial determinant equals the golden HF energy
    trial = orc.UHFTrial(s.norb, s.nelec)
    wd = s.wave_data()
    hd = trial.build_measurement_intermediates(s.ham_data(), wd)
    e = trial.calc_energy([s.mo_coeff[0][None].astype(complex), s.mo_coeff[1][None].astype(complex)], hd, wd)
    assert abs(float(np.real(e[0])) - e_uhf) < 1e-12


def test_launch_script_setup(tmp_path):
    ds, mo, _, meta = _golden()
    d = _write_dir(tmp_path, ds, mo)
    ham_data, ham, prop, trial, wave_data, smp, options = launch_script.setup_afqmc(
        dict(meta["driver_options"]), d)
    assert options["walker_type"] == "unrestricted" and options["trial"] == "uhf"
    assert prop.n_walkers == 50 and prop.dt == 0.01 and prop.n_exp_terms == 6
    assert (smp.n_prop_steps, smp.n_ene_blocks, smp.n_sr_blocks, smp.n_blocks) == (50, 1, 10, 10)
    assert type(trial).__name__ == "uhf" and len(wave_data["mo_coeff"]) == 2
    assert ham_data["h1"].shape == (2, 6, 6) and ham_data["chol"].shape == (15, 36)
    o = launch_script.read_options({"walker_type": "rhf", "free_projection": True})
    assert o["walker_type"] == "restricted" and o["trial"] == "rhf"
    assert launch_script.set_prop(o).n_exp_terms == 10
    assert launch_script.read_options({"vhs_mixed_precision": True})["precision"] == "mixed"
    o = launch_script.read_options({"prjlo": np.ones((1, 3)), "trial": "uhf"})
    t, wd = launch_script.set_trial(o, mo, 6, (3, 3))
    assert type(t).__name__ == "rhf_lno" and wd["mo_coeff"].shape == (6, 3) and "prjlo" in wd
    for bad in ({"ad_mode": "forward"}, {"trial": "cisd"}, {"walker_type": "generalized"},
                {"symmetry_projector": "s2"}, {"precision": "fp16"}):
        with pytest.raises(ValueError):
            launch_script.read_options(bad)
    with pytest.raises(ValueError):
        launch_script.run_afqmc(dict(meta["driver_options"]), nproc=2, tmpdir=d)


def test_reader_follows_continuation_blocks(tmp_path):
    """A dataset whose layout message sits in a continuation block (what the
    HDF5 library writes once an object header overflows) reads back the same."""
    fn = str(tmp_path / "x.h5")
    arr = np.arange(12, dtype=np.float64).reshape(3, 4)
    fcidump.write_hdf5_datasets(fn, {"a": arr})
    raw = bytearray(open(fn, "rb").read())
    u = lambda o, n: int.from_bytes(raw[o:o + n], "little")  # noqa: E731
    heap, btree = u(88, 8), u(80, 8)
    snod = u(btree + 32, 8)
    oh = u(snod + 8 + 8, 8)  # object header of the only dataset
    # find the layout message (type 8) in the header's message block
    p, end = oh + 16, oh + 16 + u(oh + 8, 4)
    while p < end and u(p, 2) != 8:
        p += 8 + u(p + 2, 2)
    assert p < end
    size = u(p + 2, 2)
    layout_msg = bytes(raw[p:p + 8 + size])
    # append a continuation block holding the layout message (plus a NIL message)
    cont_addr = len(raw)
    block = layout_msg + struct.pack("<HHB3x", 0, 8, 0) + bytes(8)
    raw += block
    # replace the layout message in place by a continuation message of the same size
    cont = struct.pack("<QQ", cont_addr, len(block)) + bytes(size - 16)
    raw[p:p + 8 + size] = struct.pack("<HHB3x", 0x10, size, 0) + cont
    raw[oh + 2:oh + 4] = struct.pack("<H", u(oh + 2, 2) + 2)  # the block adds layout + NIL
    open(fn, "wb").write(bytes(raw))
    got = fcidump.read_hdf5_datasets(fn)["a"]
    assert got.dtype == arr.dtype and got.shape == arr.shape and np.array_equal(got, arr)
