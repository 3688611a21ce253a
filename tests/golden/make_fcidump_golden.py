"""Generate the FCIDUMP_chol golden fixture.

The reference's driver tests (tests/test_driver.py:16-86) run AFQMC on the
Hamiltonian in tests/driver_test_files/FCIDUMP_chol (an HDF5 file written by
pyscf_interface.write_dqmc) with the orbitals of mo_coeff.npz beside it: 6
orbitals, 3 + 3 electrons, 15 Cholesky vectors.  They assert the AFQMC energy
-3.238196747261496 (one process, tests/test_driver.py:86) and
-3.239302058353345 (two processes, :33), each from one stochastic run with
the reference's random stream (UHF trial, 50 walkers, 10 blocks of 10 x 50
steps at dt = 0.01).

h5py is absent here, so the file is decoded with this package's minimal HDF5
reader.  That decoding is checked against properties the reference's data
must have whatever the reader: the header is [6, 6, 0, 15], hcore and every
Cholesky vector are symmetric, mo_coeffs_up/dn equal mo_coeff.npz, and the
Hartree-Fock energy of the UHF trial (computed below from the decoded
arrays with plain NumPy) lies above the reference's AFQMC energy by a
correlation energy of a plausible size.

Running this script (with the reference checked out at REF) writes
``fcidump_golden.npz`` (every dataset, the orbitals and the HF energy) and
``fcidump_golden.json`` (the reference's asserted energies with their source
lines, the file's SHA-256, and the library-written object-header bytes of
three datasets, for the writer's layout check).
"""

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ad_afqmc_b200 import fcidump  # noqa: E402

REF = "/root/reference/tests/driver_test_files"

REFERENCE_VALUES = {
    "afqmc_energy_1proc": [-3.238196747261496, "tests/test_driver.py:74-86"],
    "afqmc_energy_2proc": [-3.239302058353345, "tests/test_driver.py:19-33"],
}
DRIVER_OPTIONS = {  # tests/test_driver.py:75-84
    "n_eql": 1, "n_ene_blocks": 1, "n_sr_blocks": 10, "n_blocks": 10, "n_walkers": 50,
    "seed": 98, "trial": "uhf", "walker_type": "unrestricted",
}


def uhf_energy(h0, h1, chol, mo_a, mo_b):
    """E = h0 + sum_s tr(h1 P_s) + 1/2 sum_g [tr(L_g P)^2 - sum_s tr(L_g P_s L_g P_s)]."""
    pa, pb = mo_a @ mo_a.T, mo_b @ mo_b.T
    ej = np.einsum("gij,ji->g", chol, pa + pb)
    ek = sum(np.einsum("gij,jk,gkl,li->", chol, p, chol, p) for p in (pa, pb))
    return float(h0 + np.sum(h1 * pa) + np.sum(h1 * pb) + 0.5 * (np.sum(ej ** 2) - ek))


def object_header(buf: bytes, name: str) -> str:
    """Hex of the 272-byte object header of a root-group dataset, with the
    8-byte data address in its layout message zeroed."""
    u = lambda o, n: int.from_bytes(buf[o:o + n], "little")  # noqa: E731
    heap, btree = u(88, 8), u(80, 8)
    dseg, snod = u(heap + 24, 8), u(btree + 32, 8)
    for i in range(u(snod + 6, 2)):
        e = snod + 8 + 40 * i
        off = dseg + u(e, 8)
        if buf[off:buf.index(b"\0", off)] == name.encode():
            oh = u(e + 8, 8)
            h = bytearray(buf[oh:oh + 272])
            p = 16
            while p < len(h):
                mtype, msize = int.from_bytes(h[p:p + 2], "little"), int.from_bytes(h[p + 2:p + 4], "little")
                if mtype == 8:
                    h[p + 8 + 2:p + 8 + 10] = bytes(8)
                p += 8 + msize
            return h.hex()
    raise KeyError(name)


def main():
    path = os.path.join(REF, "FCIDUMP_chol")
    raw = open(path, "rb").read()
    d = fcidump.read_hdf5_datasets(path)
    mo = np.load(os.path.join(REF, "mo_coeff.npz"))["mo_coeff"]
    h0, h1, chol, norb, nelec = fcidump.read_fcidump(REF)
    assert list(d["header"]) == [6, 6, 0, 15] and nelec == (3, 3)
    assert np.abs(h1 - h1.T).max() < 1e-12
    assert np.abs(chol - chol.transpose(0, 2, 1)).max() < 1e-12
    assert np.array_equal(d["mo_coeffs_up"], mo[0]) and np.array_equal(d["mo_coeffs_dn"], mo[1])
    e_hf = uhf_energy(float(h0), h1, chol, mo[0][:, :3], mo[1][:, :3])
    e_qmc = REFERENCE_VALUES["afqmc_energy_1proc"][0]
    assert 0.0 < e_hf - e_qmc < 0.5, (e_hf, e_qmc)

    np.savez(os.path.join(HERE, "fcidump_golden.npz"), mo_coeff=mo, e_uhf=np.float64(e_hf),
             **{f"ds_{k}": v for k, v in d.items()})
    meta = {
        "source": "tests/driver_test_files/FCIDUMP_chol, tests/driver_test_files/mo_coeff.npz",
        "sha256": hashlib.sha256(raw).hexdigest(),
        "reference_values": REFERENCE_VALUES,
        "driver_options": DRIVER_OPTIONS,
        "e_uhf": e_hf,
        "object_headers": {k: object_header(raw, k) for k in ("chol", "energy_core", "header")},
    }
    with open(os.path.join(HERE, "fcidump_golden.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("E_UHF", e_hf, "AFQMC (reference)", e_qmc)


if __name__ == "__main__":
    main()
