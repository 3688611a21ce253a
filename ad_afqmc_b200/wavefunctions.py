"""RHF / UHF trial measurements on the device (mirror of ad_afqmc/wavefunctions.py).

Method names, arguments and the ``ham_data`` / ``wave_data`` keys follow the
reference classes ``rhf`` (wavefunctions.py:1038-1235) and ``uhf``
(:1238-1499); the batched dispatch on the walker type follows the base class
``wave_function`` (:19-493).  Overlap, Green's function, force bias and local
energy run in libafqmc_b200 (FP64), and so do the half-rotated
intermediates and the natural orbitals of the initial walkers
(``intermediates.py``).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib, intermediates
from ._engine import drop_engines, get_engine, small_work, to_dev
from .walkers import RHFWalkers, UHFWalkers, walker_batch


def _walker_type(walkers) -> str:
    if isinstance(walkers, UHFWalkers):
        return "unrestricted"
    if isinstance(walkers, RHFWalkers):
        return "restricted"
    raise NotImplementedError("Walker type not supported")


def _ptrs(walkers):
    if isinstance(walkers, UHFWalkers):
        return _lib.pair(walkers.data[0].data_ptr(), walkers.data[1].data_ptr())
    return _lib.pair(walkers.data.data_ptr(), None)


class wave_function:
    """Base class (wavefunctions.py:19-493) restricted to the single-determinant
    trials.  As in the reference it is not a dataclass itself: each trial class
    declares its own fields, so their order is the reference's."""

    norb: int
    nelec: Tuple[int, int]
    n_chunks: int = 1

    # -- trial orbitals on the device, cached in wave_data -------------------
    def _mo_list(self, wave_data: dict) -> List[torch.Tensor]:
        cached = wave_data.get("_afq_mo")
        if cached is not None:
            return cached
        mo = wave_data["mo_coeff"]
        if isinstance(self, uhf):
            out = [to_dev(mo[0]), to_dev(mo[1])]
        else:
            out = [to_dev(mo)]
        wave_data["_afq_mo"] = out
        return out

    def _dims(self, walkers, nchol=1):
        from ._engine import dims_for

        return dims_for(self, _walker_type(walkers), walkers.n_walkers, nchol)

    # -- measurements --------------------------------------------------------
    def calc_overlap(self, walkers: walker_batch, wave_data: dict) -> torch.Tensor:
        """<psi_T|walker> for all walkers, (W,) complex128 (wavefunctions.py:93-200)."""
        mos = self._mo_list(wave_data)
        d = self._dims(walkers)
        W = walkers.n_walkers
        out = torch.empty(W, dtype=torch.complex128, device=mos[0].device)
        work = small_work(W)
        mo = _lib.pair(mos[0].data_ptr(), mos[-1].data_ptr())
        _lib.check(
            _lib.lib().afq_calc_overlap(C.byref(d), mo, _ptrs(walkers), out.data_ptr(),
                                        work.data_ptr(), work.numel() * 8, _lib.stream_handle()),
            "afq_calc_overlap",
        )
        return out

    def calc_green(self, walkers: walker_batch, wave_data: dict):
        """Half-rotated Green's functions (rhf._calc_green :1089-1100, uhf :1289-1312).

        Restricted walkers: (W, No, N); unrestricted: [(W, Na, N), (W, Nb, N)]."""
        mos = self._mo_list(wave_data)
        d = self._dims(walkers)
        W = walkers.n_walkers
        dev = mos[0].device
        if isinstance(walkers, UHFWalkers):
            g = [torch.empty(W, walkers.data[s].shape[2], self.norb, dtype=torch.complex128, device=dev)
                 for s in range(2)]
        else:
            g = [torch.empty(W, walkers.data.shape[2], self.norb, dtype=torch.complex128, device=dev)]
        work = small_work(W)
        mo = _lib.pair(mos[0].data_ptr(), mos[-1].data_ptr())
        gp = _lib.pair(g[0].data_ptr(), g[-1].data_ptr() if len(g) > 1 else None)
        _lib.check(
            _lib.lib().afq_calc_green(C.byref(d), mo, _ptrs(walkers), gp, work.data_ptr(),
                                      work.numel() * 8, _lib.stream_handle()),
            "afq_calc_green",
        )
        return g if len(g) > 1 else g[0]

    def calc_force_bias(self, walkers: walker_batch, ham_data: dict, wave_data: dict) -> torch.Tensor:
        """Force bias (W, G) complex128 (wavefunctions.py:202-262)."""
        eng = get_engine(ham_data, self, wave_data, _walker_type(walkers), walkers.n_walkers)
        W, G = walkers.n_walkers, int(ham_data["chol"].shape[0])
        out = torch.empty(W, G, dtype=torch.complex128, device=eng.prepared.device)
        p, w, wb = eng.handle
        _lib.check(
            _lib.lib().afq_calc_force_bias(C.byref(eng.dims), p, _ptrs(walkers), out.data_ptr(), w, wb,
                                           _lib.stream_handle()),
            "afq_calc_force_bias",
        )
        return out

    def calc_energy(self, walkers: walker_batch, ham_data: dict, wave_data: dict, *,
                    engine=None) -> torch.Tensor:
        """Local energy (W,) complex128 (wavefunctions.py:264-394).  ``engine``
        (keyword only) evaluates it on an existing engine, e.g. the propagator's,
        instead of the FP64 engine of this shape."""
        eng = engine if engine is not None else get_engine(ham_data, self, wave_data, _walker_type(walkers),
                                                           walkers.n_walkers)
        W = walkers.n_walkers
        out = torch.empty(W, dtype=torch.complex128, device=eng.prepared.device)
        p, w, wb = eng.handle
        _lib.check(
            _lib.lib().afq_calc_energy(C.byref(eng.dims), p, _ptrs(walkers), out.data_ptr(), w, wb,
                                       _lib.stream_handle()),
            "afq_calc_energy",
        )
        return out

    # -- trial data ----------------------------------------------------------
    def get_rdm1(self, wave_data: dict) -> torch.Tensor:
        """wavefunctions.py:396-411."""
        if "rdm1" in wave_data:
            return to_dev(wave_data["rdm1"])
        return self._calc_rdm1(wave_data)

    def get_init_walkers(self, wave_data: dict, n_walkers: int, walker_type: str) -> walker_batch:
        """Natural orbitals of the trial rdm1, descending (wavefunctions.py:427-466)."""
        rdm1 = self.get_rdm1(wave_data)
        na, nb = self.nelec
        if walker_type == "restricted":
            nat = intermediates.natural_orbitals(rdm1[0] + rdm1[1], na)
            return RHFWalkers(nat.to(torch.complex128).unsqueeze(0).repeat(n_walkers, 1, 1))
        if walker_type == "unrestricted":
            up = intermediates.natural_orbitals(rdm1[0], na).to(torch.complex128)
            dn = intermediates.natural_orbitals(rdm1[1], nb).to(torch.complex128)
            return UHFWalkers([up.unsqueeze(0).repeat(n_walkers, 1, 1),
                               dn.unsqueeze(0).repeat(n_walkers, 1, 1)])
        raise Exception("Unknown walker_type.")

    def optimize(self, ham_data: dict, wave_data: dict) -> dict:
        return wave_data

    def __hash__(self) -> int:
        """wavefunctions.py:492-493."""
        return hash(tuple(self.__dict__.values()))


@dataclass
class rhf(wave_function):
    """Restricted Hartree-Fock trial (wavefunctions.py:1038-1235).  Fields in the
    reference's order (:1053-1057): norb, nelec, n_opt_iter, n_chunks, projector."""

    norb: int
    nelec: Tuple[int, int]
    n_opt_iter: int = 30
    n_chunks: int = 1
    projector: Optional[str] = None

    def __post_init__(self):
        assert self.nelec[0] == self.nelec[1], "RHF requires equal number of up and down electrons."

    def __hash__(self) -> int:
        """wavefunctions.py:1234-1235."""
        return hash(tuple(self.__dict__.values()))

    def _calc_rdm1(self, wave_data: dict) -> torch.Tensor:
        mo = to_dev(wave_data["mo_coeff"])
        return torch.stack([mo @ mo.T, mo @ mo.T])

    def _build_measurement_intermediates(self, ham_data: dict, wave_data: dict) -> dict:
        """h1 symmetrized, rot_h1 = C^H (h1a + h1b)/2, rot_chol[g] = C^H L_g
        (wavefunctions.py:1215-1232), by afq_measurement_intermediates."""
        ham_data["chol"] = to_dev(ham_data["chol"])
        mo = to_dev(wave_data["mo_coeff"])
        h1, rh1, rc = intermediates.measurement(self.norb, self.nelec, ham_data["h1"], ham_data["chol"],
                                                [mo], uhf=False)
        ham_data["h1"] = h1
        ham_data["rot_h1"] = rh1[0]
        ham_data["rot_chol"] = rc[0]
        wave_data.pop("_afq_mo", None)
        drop_engines(ham_data)
        return ham_data


@dataclass
class rhf_lno(rhf):
    """RHF trial of an LNO fragment (wavefunctions.py:6871-6926): the rhf
    measurements plus the orbital energy of the fragment's localized orbital,
    whose projector is wave_data["prjlo"] ((n_lo, nocc), lnoafqmc.py:147)."""

    def __hash__(self) -> int:
        """wavefunctions.py:6925-6926."""
        return hash(tuple(self.__dict__.values()))

    def calc_orbenergy(self, walkers: walker_batch, ham_data: dict, wave_data: dict, *,
                       engine=None) -> torch.Tensor:
        """wavefunctions.py:6898-6923 -> afq_calc_orbenergy (W,) complex128."""
        if not isinstance(walkers, RHFWalkers):
            raise NotImplementedError("Walker type not supported")  # as the reference
        eng = engine if engine is not None else get_engine(ham_data, self, wave_data, "restricted",
                                                           walkers.n_walkers)
        prj = to_dev(wave_data["prjlo"], torch.float64).reshape(-1, self.nelec[0]).contiguous()
        out = torch.empty(walkers.n_walkers, dtype=torch.complex128, device=eng.prepared.device)
        p, w, wb = eng.handle
        _lib.check(
            _lib.lib().afq_calc_orbenergy(C.byref(eng.dims), p, _ptrs(walkers), prj.data_ptr(),
                                          int(prj.shape[0]), out.data_ptr(), w, wb, _lib.stream_handle()),
            "afq_calc_orbenergy",
        )
        return out


@dataclass
class uhf(wave_function):
    """Unrestricted Hartree-Fock trial (wavefunctions.py:1238-1499).  Fields in the
    reference's order (:1251-1255): norb, nelec, n_opt_iter, n_chunks, projector."""

    norb: int
    nelec: Tuple[int, int]
    n_opt_iter: int = 30
    n_chunks: int = 1
    projector: Optional[str] = None

    def __hash__(self) -> int:
        """wavefunctions.py:1498-1499."""
        return hash(tuple(self.__dict__.values()))

    def _calc_rdm1(self, wave_data: dict) -> torch.Tensor:
        m0, m1 = to_dev(wave_data["mo_coeff"][0]), to_dev(wave_data["mo_coeff"][1])
        return torch.stack([m0 @ m0.T, m1 @ m1.T])

    def _build_measurement_intermediates(self, ham_data: dict, wave_data: dict) -> dict:
        """h1 symmetrized, rot_h1[s] = C_s^H h1[s], rot_chol[s][g] = C_s^H L_g
        (wavefunctions.py:1472-1496), by afq_measurement_intermediates."""
        ham_data["chol"] = to_dev(ham_data["chol"])
        mos = [to_dev(wave_data["mo_coeff"][0]), to_dev(wave_data["mo_coeff"][1])]
        h1, rh1, rc = intermediates.measurement(self.norb, self.nelec, ham_data["h1"], ham_data["chol"],
                                                mos, uhf=True)
        ham_data["h1"] = h1
        ham_data["rot_h1"] = rh1
        ham_data["rot_chol"] = rc
        wave_data.pop("_afq_mo", None)
        drop_engines(ham_data)
        return ham_data
