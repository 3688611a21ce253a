"""C-ABI checks that need no GPU: the library loads, exports every symbol
declared in include/afqmc_b200.h, and rejects bad arguments with the
documented status codes before touching the device."""

import ctypes as C
import os
import re

import pytest

from ad_afqmc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "afqmc_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(afq_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    # the ctypes binding covers every declared entry point
    assert set(names) <= set(_lib.EXPORTED)


def test_version_and_status_strings():
    lib = _lib.lib()
    assert lib.afq_version() >= 100
    assert lib.afq_status_string(0) == b"ok"
    assert b"size" in lib.afq_status_string(1)


def _dims(**kw):
    base = dict(norb=20, nocc=(5, 5), nchol=40, nwalkers=16, walker_type=0, trial_type=0,
                n_exp_terms=6, precision=0, dt=0.01)
    base.update(kw)
    return _lib.make_dims(**base)


def test_sizes_scale_with_shape():
    p1, w1 = _lib.sizes(_dims())
    p2, w2 = _lib.sizes(_dims(nwalkers=32))
    assert p1 == p2 and w2 > w1
    p3, _ = _lib.sizes(_dims(nchol=80))
    assert p3 > p1


@pytest.mark.parametrize("kw,code", [
    (dict(norb=0), 1), (dict(nocc=(0, 0)), 1), (dict(nocc=(65, 65), norb=80), 1),
    (dict(nocc=(5, 4), walker_type=1), 1),                   # rhf needs Na == Nb
    (dict(walker_type=0, trial_type=1, nocc=(5, 4)), 1),     # uhf trial + restricted walkers
    (dict(walker_type=3), 6), (dict(precision=7), 6), (dict(n_exp_terms=0), 6),
])
def test_bad_shapes_rejected(kw, code):
    d = _dims(**kw)
    b = C.c_size_t()
    assert _lib.lib().afq_workspace_size(C.byref(d), C.byref(b)) == code


def test_null_pointers_rejected_without_device_work():
    lib = _lib.lib()
    d = _dims()
    z = _lib.pair(None, None)
    assert lib.afq_calc_overlap(C.byref(d), z, z, None, None, 0, None) == 2
    assert lib.afq_calc_energy(C.byref(d), None, z, None, None, 0, None) == 2
    assert lib.afq_propagate_constrained(C.byref(d), None, None, None, None, 0, None) == 2
    assert lib.afq_normal_fields(None, 10, 1, 0, None) == 2


def test_workspace_too_small_and_misaligned():
    lib = _lib.lib()
    d = _dims()
    buf = (C.c_double * 64)()
    addr = C.addressof(buf)
    addr16 = (addr + 15) & ~15
    z = _lib.pair(addr16, None)
    # prepared/work present but far too small -> workspace error
    assert lib.afq_calc_energy(C.byref(d), addr16, z, addr16, addr16, 8, None) == 4
    assert lib.afq_calc_energy(C.byref(d), addr16 + 8, z, addr16, addr16, 1 << 40, None) == 5
