"""FCIDUMP_chol input (launch_script.read_fcidump, launch_script.py:60-94) and
its writer (pyscf_interface.write_dqmc, pyscf_interface.py:399-420).

FCIDUMP_chol is an HDF5 file with the datasets header = [nelec, nmo, ms,
nchol] (int64), hcore, hcore_mod, chol (all flattened float64), energy_core
(a float64 scalar) and optionally mo_coeffs_up / mo_coeffs_dn.  The trial
orbitals sit beside it in mo_coeff.npz (key "mo_coeff", shape (2, N, N)).

h5py is used when it is importable.  Otherwise a minimal HDF5 reader and
writer cover exactly what the HDF5 library writes for such a file with its
default settings:

* superblock version 0 with 8-byte offsets and lengths;
* a root group held in a symbol table: a version-1 B-tree of group nodes,
  a local heap of link names and symbol-table nodes (SNOD);
* version-1 object headers (with continuation blocks);
* dataspace messages of version 1 or 2, fixed-point and IEEE floating-point
  datatypes in little-endian order, data layout version 3 (compact or
  contiguous storage).

Chunked or compressed datasets, big-endian data and the version-2 object
headers of newer file formats are refused with an error.  The writer emits
the same structures (one symbol-table node, so at most 8 datasets), with the
object-header layout the HDF5 library itself uses for small datasets.
"""

from __future__ import annotations

import os
import struct
from typing import Dict, Tuple

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF

# object-header message types
_MSG_NIL, _MSG_SPACE, _MSG_TYPE, _MSG_FILL, _MSG_LAYOUT = 0x0, 0x1, 0x3, 0x5, 0x8
_MSG_CONT, _MSG_STAB = 0x10, 0x11


# ---------------------------------------------------------------------------
# minimal HDF5 reader
# ---------------------------------------------------------------------------
def _u(buf: bytes, off: int, n: int) -> int:
    return int.from_bytes(buf[off:off + n], "little")


def _dtype(msg: bytes) -> np.dtype:
    """Datatype message: class in the low nibble of byte 0, bit field in
    bytes 1-3, element size in bytes 4-7."""
    cls = msg[0] & 0x0F
    bits = msg[1] | (msg[2] << 8) | (msg[3] << 16)
    size = _u(msg, 4, 4)
    if bits & 1:
        raise ValueError("big-endian HDF5 data are not supported")
    if cls == 0:  # fixed point; bit 3 = signed
        return np.dtype(("<i" if bits & 0x08 else "<u") + str(size))
    if cls == 1:  # IEEE floating point
        if size not in (2, 4, 8):
            raise ValueError(f"unsupported floating-point size {size}")
        return np.dtype("<f" + str(size))
    raise ValueError(f"unsupported HDF5 datatype class {cls}")


def _shape(msg: bytes) -> Tuple[int, ...]:
    """Dataspace message, version 1 (8-byte preamble) or 2 (4-byte preamble
    whose last byte is the space type: 0 scalar, 1 simple, 2 null)."""
    version, rank = msg[0], msg[1]
    if version == 1:
        off = 8
    elif version == 2:
        if msg[3] == 2:
            raise ValueError("null dataspaces are not supported")
        off = 4
    else:
        raise ValueError(f"unsupported dataspace version {version}")
    return tuple(_u(msg, off + 8 * i, 8) for i in range(rank))


def _messages(buf: bytes, addr: int):
    """(type, data) of every message of a version-1 object header,
    following continuation messages."""
    if buf[addr] != 1:
        raise ValueError(f"unsupported object header version {buf[addr]} at {addr}")
    nmsg = _u(buf, addr + 2, 2)
    blocks = [(addr + 16, _u(buf, addr + 8, 4))]
    out = []
    while blocks and len(out) < nmsg:
        p, size = blocks.pop(0)
        end = p + size
        while p + 8 <= end and len(out) < nmsg:
            mtype, msize = _u(buf, p, 2), _u(buf, p + 2, 2)
            data = buf[p + 8:p + 8 + msize]
            out.append((mtype, data))
            if mtype == _MSG_CONT:
                blocks.append((_u(data, 0, 8), _u(data, 8, 8)))
            p += 8 + msize
    return out


def _dataset(buf: bytes, addr: int) -> np.ndarray:
    shape = dtype = layout = None
    for mtype, data in _messages(buf, addr):
        if mtype == _MSG_SPACE:
            shape = _shape(data)
        elif mtype == _MSG_TYPE:
            dtype = _dtype(data)
        elif mtype == _MSG_LAYOUT:
            layout = data
    if shape is None or dtype is None or layout is None:
        raise ValueError(f"object at {addr} is not a dataset this reader understands")
    if layout[0] != 3:
        raise ValueError(f"unsupported data layout version {layout[0]}")
    count = int(np.prod(shape, dtype=np.int64)) if shape else 1
    nbytes = count * dtype.itemsize
    if layout[1] == 0:  # compact: size (2) + raw data
        raw = layout[4:4 + _u(layout, 2, 2)]
    elif layout[1] == 1:  # contiguous: address (8) + size (8)
        a, size = _u(layout, 2, 8), _u(layout, 10, 8)
        raw = b"" if a == _UNDEF else buf[a:a + size]
    else:
        raise ValueError("chunked HDF5 datasets are not supported")
    if len(raw) < nbytes:
        if len(raw) == 0:  # never written: the default fill value (zero)
            raw = bytes(nbytes)
        else:
            raise ValueError(f"dataset at {addr}: {len(raw)} bytes stored, {nbytes} expected")
    arr = np.frombuffer(raw[:nbytes], dtype=dtype).copy()
    return arr.reshape(shape) if shape else arr.reshape(())


def _group_entries(buf: bytes, btree: int, heap_data: int):
    """(name, object header address) of every link below a group B-tree."""
    if buf[btree:btree + 4] != b"TREE":
        raise ValueError(f"no B-tree node at {btree}")
    if buf[btree + 4] != 0:
        raise ValueError("not a group B-tree")
    level, used = buf[btree + 5], _u(buf, btree + 6, 2)
    out = []
    for i in range(used):
        child = _u(buf, btree + 24 + 8 + 16 * i, 8)  # key0, child0, key1, child1, ...
        if level > 0:
            out.extend(_group_entries(buf, child, heap_data))
            continue
        if buf[child:child + 4] != b"SNOD":
            raise ValueError(f"no symbol-table node at {child}")
        for k in range(_u(buf, child + 6, 2)):
            e = child + 8 + 40 * k
            noff = heap_data + _u(buf, e, 8)
            name = buf[noff:buf.index(b"\0", noff)].decode()
            out.append((name, _u(buf, e + 8, 8)))
    return out


def read_hdf5_datasets(path: str) -> Dict[str, np.ndarray]:
    """All datasets directly under the root group of an HDF5 file (superblock
    version 0, 8-byte offsets), as NumPy arrays."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != _SIG:
        raise ValueError(f"{path} is not an HDF5 file (or has a user block)")
    if buf[8] not in (0, 1):
        raise ValueError(f"superblock version {buf[8]} is not supported")
    if buf[13] != 8 or buf[14] != 8:
        raise ValueError("only 8-byte offsets and lengths are supported")
    root = 56 if buf[8] == 0 else 60  # version 1 adds 4 bytes (indexed-storage K)
    root_oh = _u(buf, root + 8, 8)
    stab = [d for t, d in _messages(buf, root_oh) if t == _MSG_STAB]
    if not stab:
        raise ValueError("the root group has no symbol table (newer file format)")
    btree, heap = _u(stab[0], 0, 8), _u(stab[0], 8, 8)
    if buf[heap:heap + 4] != b"HEAP":
        raise ValueError(f"no local heap at {heap}")
    heap_data = _u(buf, heap + 24, 8)
    return {name: _dataset(buf, oh) for name, oh in _group_entries(buf, btree, heap_data)}


# ---------------------------------------------------------------------------
# minimal HDF5 writer
# ---------------------------------------------------------------------------
_LEAF_K, _NODE_K = 4, 16
_BTREE_BYTES = 24 + 2 * _NODE_K * 8 + (2 * _NODE_K + 1) * 8
_SNOD_BYTES = 8 + 2 * _LEAF_K * 40
_DSET_OH_DATA = 256  # message bytes per dataset header (the library's default size)


def _pad8(b: bytes) -> bytes:
    return b + bytes(-len(b) % 8)


def _msg(mtype: int, data: bytes, flags: int = 0) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _type_msg(dt: np.dtype) -> bytes:
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0x00
        head = struct.pack("<B3BI", 0x10, bits, 0, 0, dt.itemsize)
        return head + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        exp_bits, mant_bits = {2: (5, 10), 4: (8, 23), 8: (11, 52)}[dt.itemsize]
        sign = 8 * dt.itemsize - 1
        head = struct.pack("<B3BI", 0x11, 0x20, sign, 0, dt.itemsize)
        return head + struct.pack("<HHBBBBI", 0, 8 * dt.itemsize, mant_bits, exp_bits, 0, mant_bits,
                                  (1 << (exp_bits - 1)) - 1)
    raise ValueError(f"unsupported dtype {dt}")


def _space_msg(shape: Tuple[int, ...]) -> bytes:
    if not shape:
        return struct.pack("<BBB5x", 1, 0, 0)
    dims = b"".join(struct.pack("<Q", n) for n in shape)
    return struct.pack("<BBB5x", 1, len(shape), 1) + dims + dims  # current and maximum dims


def _dataset_header(arr: np.ndarray, data_addr: int) -> bytes:
    msgs = (_msg(_MSG_SPACE, _space_msg(arr.shape))
            + _msg(_MSG_TYPE, _type_msg(arr.dtype), flags=1)
            + _msg(_MSG_FILL, struct.pack("<BBBBI", 2, 2, 2, 1, 0), flags=1)
            + _msg(_MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, data_addr, arr.nbytes)))
    nmsg = 5
    pad = _DSET_OH_DATA - len(msgs)
    if pad < 8:
        raise AssertionError("dataset header overflow")
    msgs += struct.pack("<HHB3x", _MSG_NIL, pad - 8, 0) + bytes(pad - 8)
    return struct.pack("<BBHII4x", 1, 0, nmsg, 1, len(msgs)) + msgs


def write_hdf5_datasets(path: str, datasets: Dict[str, np.ndarray]) -> None:
    """Write up to 8 arrays as contiguous datasets under the root group of a
    new HDF5 file (superblock version 0)."""
    items = []
    for name, v in datasets.items():
        a = np.asarray(v)
        if a.dtype.kind not in "iuf":
            raise ValueError(f"dataset {name!r}: unsupported dtype {a.dtype}")
        items.append((name, np.array(a, dtype=a.dtype.newbyteorder("<"), order="C")))  # keeps 0-d shapes
    if not 1 <= len(items) <= 2 * _LEAF_K:
        raise ValueError(f"between 1 and {2 * _LEAF_K} datasets per file")
    items.sort(key=lambda kv: kv[0].encode())  # symbol-table nodes keep names sorted

    # local heap data: the empty name at offset 0, then each name, 8-byte padded
    heap_data = bytearray(8)
    name_off = {}
    for name, _ in items:
        name_off[name] = len(heap_data)
        heap_data += _pad8(name.encode() + b"\0")
    # a trailing free block (next = 1: end of list, size), as the library leaves one
    free_off = len(heap_data)
    heap_data += struct.pack("<QQ", 1, 16)

    root_oh = 96
    root_oh_bytes = 16 + 24
    btree = root_oh + root_oh_bytes
    heap = btree + _BTREE_BYTES
    heap_data_addr = heap + 32
    snod = heap_data_addr + len(heap_data)
    oh = snod + _SNOD_BYTES
    headers_end = oh + len(items) * (16 + _DSET_OH_DATA)
    data_addr = []
    p = headers_end
    for _, a in items:
        data_addr.append(p)
        p += -(-a.nbytes // 8) * 8
    eof = p

    out = bytearray()
    out += _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", _LEAF_K, _NODE_K, 0)
    out += struct.pack("<QQQQ", 0, _UNDEF, eof, _UNDEF)
    out += struct.pack("<QQII", 0, root_oh, 1, 0) + struct.pack("<QQ", btree, heap)
    assert len(out) == root_oh
    out += struct.pack("<BBHII4x", 1, 0, 1, 1, 24) + _msg(_MSG_STAB, struct.pack("<QQ", btree, heap))
    assert len(out) == btree
    node = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", 1, _UNDEF, _UNDEF))
    node += struct.pack("<QQQ", 0, snod, name_off[items[-1][0]])
    out += node + bytes(_BTREE_BYTES - len(node))
    assert len(out) == heap
    out += b"HEAP" + bytes(4) + struct.pack("<QQQ", len(heap_data), free_off, heap_data_addr)
    out += heap_data
    assert len(out) == snod
    sn = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(items)))
    for i, (name, _) in enumerate(items):
        sn += struct.pack("<QQII", name_off[name], oh + i * (16 + _DSET_OH_DATA), 0, 0) + bytes(16)
    out += sn + bytes(_SNOD_BYTES - len(sn))
    for i, (_, a) in enumerate(items):
        out += _dataset_header(a, data_addr[i])
    assert len(out) == headers_end
    for i, (_, a) in enumerate(items):
        raw = a.tobytes()
        out += raw + bytes(-len(raw) % 8)
    assert len(out) == eof
    with open(path, "wb") as f:
        f.write(out)


# ---------------------------------------------------------------------------
# FCIDUMP_chol
# ---------------------------------------------------------------------------
def _read(path: str) -> Dict[str, np.ndarray]:
    try:
        import h5py
    except ImportError:
        return read_hdf5_datasets(path)
    with h5py.File(path, "r") as f:
        return {k: np.array(f[k]) for k in f.keys()}


def read_fcidump(tmp_dir: str = "."):
    """launch_script.read_fcidump (launch_script.py:60-94): (h0, h1 (N, N),
    chol (nchol, N, N), norb, (n_alpha, n_beta)) with n_alpha/beta =
    (nelec +- |ms|) // 2.  A missing file raises AssertionError as there."""
    path = os.path.join(tmp_dir, "FCIDUMP_chol")
    if not os.path.isfile(path):
        raise AssertionError(f"File '{path}' does not exist.")
    d = _read(path)
    header = np.asarray(d["header"])
    if header.dtype != np.int64 or header.shape != (4,):
        raise AssertionError(f"header must be 4 int64 values, got {header.dtype} {header.shape}")
    nelec, norb, ms, _ = (int(x) for x in header)
    h0 = np.asarray(d["energy_core"], dtype=np.float64)
    h1 = np.asarray(d["hcore"], dtype=np.float64).reshape(norb, norb)
    chol = np.asarray(d["chol"], dtype=np.float64).reshape(-1, norb, norb)
    return h0, h1, chol, norb, ((nelec + abs(ms)) // 2, (nelec - abs(ms)) // 2)


def read_mo_coeff(tmp_dir: str = ".") -> np.ndarray:
    """launch_script.load_mo_coefficients (launch_script.py:697-711)."""
    path = os.path.join(tmp_dir, "mo_coeff.npz")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"Could not find mo_coeff.npz in {tmp_dir}")
    return np.load(path)["mo_coeff"]


def write_fcidump(hcore, hcore_mod, chol, nelec, nmo, enuc, ms=0, filename="FCIDUMP_chol",
                  mo_coeffs=None) -> None:
    """pyscf_interface.write_dqmc (pyscf_interface.py:399-420): chol is
    (nchol, N*N); hcore / hcore_mod / chol are stored flattened."""
    chol = np.asarray(chol)
    assert len(chol.shape) == 2
    data = {"header": np.array([nelec, nmo, ms, chol.shape[0]], dtype=np.int64),
            "hcore": np.asarray(hcore, dtype=np.float64).flatten(),
            "hcore_mod": np.asarray(hcore_mod, dtype=np.float64).flatten(),
            "chol": chol.astype(np.float64).flatten(), "energy_core": np.float64(enuc)}
    if mo_coeffs is not None:
        data["mo_coeffs_up"] = np.asarray(mo_coeffs[0], dtype=np.float64)
        data["mo_coeffs_dn"] = np.asarray(mo_coeffs[1], dtype=np.float64)
    try:
        import h5py
    except ImportError:
        write_hdf5_datasets(filename, data)
        return
    with h5py.File(filename, "w") as fh5:
        for k, v in data.items():
            fh5[k] = v


def write_mo_coeff(mo_coeff, tmp_dir: str = ".") -> None:
    """mo_coeff.npz beside FCIDUMP_chol: the (2, N, N) trial orbitals."""
    np.savez(os.path.join(tmp_dir, "mo_coeff.npz"), mo_coeff=np.asarray(mo_coeff, dtype=np.float64))


def ham_data_from_fcidump(tmp_dir: str = ".") -> Tuple[dict, dict, Tuple[int, int], int]:
    """ham_data {h0, h1 (2, N, N), chol (nchol, N*N), ene0} and wave_data
    {mo_coeff, rdm1} of a FCIDUMP_chol + mo_coeff.npz pair, as setup_afqmc
    builds them (launch_script.py:213-260 replicates h1 per spin; rdm1 from
    the occupied orbitals when there is no rdm1.npz, :298-316)."""
    h0, h1, chol, norb, nelec = read_fcidump(tmp_dir)
    ham = {"h0": float(h0), "h1": np.array([h1, h1]), "chol": chol.reshape(chol.shape[0], -1), "ene0": 0.0}
    wave = {}
    if os.path.isfile(os.path.join(tmp_dir, "mo_coeff.npz")):
        mo = read_mo_coeff(tmp_dir)
        wave["mo_coeff"] = [mo[0][:, :nelec[0]], mo[1][:, :nelec[1]]]
        wave["rdm1"] = np.array([m @ m.T for m in wave["mo_coeff"]])
    return ham, wave, nelec, norb


def system_from_fcidump(tmp_dir: str = ".", trial: str = "rhf"):
    """The FCIDUMP_chol + mo_coeff.npz pair as a ``SyntheticSystem`` (the
    container the walker path and the serving loop take a Hamiltonian and a
    trial from).  ``trial`` "rhf" takes the alpha occupied orbitals for both
    spins (set_trial with trial "rhf", launch_script.py:385); "uhf" keeps
    both spins' orbitals."""
    from .synthetic import SyntheticSystem

    ham, wave, nelec, norb = ham_data_from_fcidump(tmp_dir)
    if "mo_coeff" not in wave:
        raise FileNotFoundError(f"Could not find mo_coeff.npz in {tmp_dir}")
    if trial == "rhf":
        if nelec[0] != nelec[1]:
            raise ValueError("an RHF trial needs n_alpha == n_beta")
        mo = np.ascontiguousarray(wave["mo_coeff"][0])
    elif trial == "uhf":
        mo = [np.ascontiguousarray(m) for m in wave["mo_coeff"]]
    else:
        raise ValueError(f"unsupported trial {trial!r}")
    return SyntheticSystem(norb=norb, nelec=tuple(nelec), nchol=int(ham["chol"].shape[0]),
                           h1=np.ascontiguousarray(ham["h1"]), chol=np.ascontiguousarray(ham["chol"]),
                           h0=float(ham["h0"]), mo_coeff=mo, trial=trial)
