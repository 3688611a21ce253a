"""NumPy FP64 oracle for the phaseless AFQMC walker path of ad_afqmc.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it may be imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``.  The product package
(``ad_afqmc_b200``) never imports it and has no CPU fallback.

Every function restates, in plain NumPy/SciPy FP64, one function of the
reference implementation (JAX) and cites the reference file:line it follows.
The reference cannot be imported here (it needs jax and pyscf), so the
oracle is pinned against the reference's own golden values from
``tests/test_wavefunctions.py:128-184`` (see ``tests/test_oracle_golden.py``).
Full-step propagation, QR, reconfiguration and block energies have no golden
values in the reference's tests (``tests/test_propagation.py`` checks shapes
only); for those rows the oracle is a line-by-line restatement and its parity
is pinned only through the pinned building blocks (overlap, Green's function,
force bias, energy).

Randomness: the reference draws fields and reconfiguration uniforms with JAX
threefry, whose bits cannot be reproduced here.  The oracle therefore takes
all random inputs (auxiliary fields, zeta) from an injected source object
with ``fields(n_steps, n_walkers, n_chol)`` and ``uniform()`` methods, called
in the same order the reference splits its key.

Data conventions (as in the reference):
  restricted walkers    (W, N, No) complex128
  unrestricted walkers  [(W, N, Na) , (W, N, Nb)] complex128
  ham_data["chol"]      (G, N*N) float64
  rhf rot_chol          (G, No, N);  uhf rot_chol [(G, Na, N), (G, Nb, N)]
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, List, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg


# ----------------------------------------------------------------------------
# Trial wave functions: rhf / uhf measurements
# ----------------------------------------------------------------------------


def green(walker: np.ndarray, mo: np.ndarray) -> np.ndarray:
    """Half-rotated Green's function (No, N).

    wavefunctions.py:1089-1100 (rhf._calc_green), :1289-1312 (uhf._calc_green).
    """
    return (walker @ np.linalg.inv(mo.T.conj() @ walker)).T


@dataclass
class RHFTrial:
    """Restricted Hartree-Fock trial; wavefunctions.py:1038-1235."""

    norb: int
    nelec: Tuple[int, int]

    # -- single walker -----------------------------------------------------
    def overlap_restricted(self, walker, wave_data):
        """wavefunctions.py:1064-1066: det(C^H W)^2."""
        return np.linalg.det(wave_data["mo_coeff"].T.conj() @ walker) ** 2

    def overlap_unrestricted(self, wu, wd, wave_data):
        """wavefunctions.py:1068-1074."""
        mo = wave_data["mo_coeff"]
        return np.linalg.det(mo.T.conj() @ wu) * np.linalg.det(mo.T.conj() @ wd)

    def force_bias_restricted(self, walker, ham_data, wave_data):
        """wavefunctions.py:1102-1110: 2 * sum_ij rot_chol[g,i,j] G[i,j]."""
        g = green(walker, wave_data["mo_coeff"])
        return 2.0 * np.einsum("gij,ij->g", ham_data["rot_chol"], g, optimize=True)

    def force_bias_unrestricted(self, wu, wd, ham_data, wave_data):
        """wavefunctions.py:1112-1126."""
        mo = wave_data["mo_coeff"]
        g = green(wu, mo) + green(wd, mo)
        return np.einsum("gij,ij->g", ham_data["rot_chol"], g, optimize=True)

    def energy_restricted(self, walker, ham_data, wave_data):
        """wavefunctions.py:1128-1141."""
        h0, rot_h1, rot_chol = ham_data["h0"], ham_data["rot_h1"], ham_data["rot_chol"]
        g = green(walker, wave_data["mo_coeff"])
        ene1 = 2.0 * np.sum(g * rot_h1)
        f = np.einsum("gij,jk->gik", rot_chol, g.T, optimize=True)
        c = np.einsum("gii->g", f)
        exc = np.sum(f * f.transpose(0, 2, 1))
        ene2 = 2.0 * np.sum(c * c) - exc
        return ene2 + ene1 + h0

    def orbenergy_restricted(self, walker, ham_data, wave_data):
        """rhf_lno._calc_orbenergy, wavefunctions.py:6904-6923: orbital energy of
        the fragment's localized orbital (projector prjlo, (n_lo, nocc)).  f is
        rot_chol's virtual columns times the virtual rows of G^T."""
        rot_h1, rot_chol = ham_data["rot_h1"], ham_data["rot_chol"]
        m = np.asarray(wave_data["prjlo"]).T @ np.asarray(wave_data["prjlo"])
        nocc = rot_h1.shape[0]
        g = green(walker, wave_data["mo_coeff"])
        f = np.einsum("gij,jk->gik", rot_chol[:, :nocc, nocc:], g.T[nocc:, :nocc], optimize=True)
        c = np.einsum("gii->g", f)
        j2 = np.einsum("Gxk,xk,G->", f, m, c, optimize=True) * 2
        x2 = np.einsum("Gxy,Gyk,xk->", f, f, m, optimize=True)
        return j2 - x2

    def calc_orbenergy(self, walkers, ham_data, wave_data):
        return np.array([self.orbenergy_restricted(w, ham_data, wave_data) for w in walkers])

    def energy_unrestricted(self, wu, wd, ham_data, wave_data):
        """wavefunctions.py:1143-1174."""
        h0, rot_h1, rot_chol = ham_data["h0"], ham_data["rot_h1"], ham_data["rot_chol"]
        mo = wave_data["mo_coeff"]
        gu, gd = green(wu, mo), green(wd, mo)
        ene1 = np.sum((gu + gd) * rot_h1)
        fu = np.einsum("gij,jk->gik", rot_chol, gu.T, optimize=True)
        fd = np.einsum("gij,jk->gik", rot_chol, gd.T, optimize=True)
        cu, cd = np.einsum("gii->g", fu), np.einsum("gii->g", fd)
        exu = np.sum(fu * fu.transpose(0, 2, 1))
        exd = np.sum(fd * fd.transpose(0, 2, 1))
        ene2 = (np.sum(cu * cu) + np.sum(cd * cd) + 2.0 * np.sum(cu * cd) - exu - exd) / 2.0
        return ene2 + ene1 + h0

    def green_sum(self, walker, wave_data):
        return green(walker, wave_data["mo_coeff"])

    def rdm1(self, wave_data):
        """wavefunctions.py:1176-1178 (rhf._calc_rdm1) and :396-411 (get_rdm1)."""
        if "rdm1" in wave_data:
            return np.array(wave_data["rdm1"])
        mo = wave_data["mo_coeff"]
        return np.array([mo @ mo.T] * 2)

    def build_measurement_intermediates(self, ham_data, wave_data):
        """wavefunctions.py:1215-1232 (rhf._build_measurement_intermediates)."""
        h1 = np.array(ham_data["h1"], dtype=np.float64)
        h1[0] = (h1[0] + h1[0].T) / 2.0
        h1[1] = (h1[1] + h1[1].T) / 2.0
        ham_data["h1"] = h1
        mo = wave_data["mo_coeff"]
        ham_data["rot_h1"] = mo.T.conj() @ ((h1[0] + h1[1]) / 2.0)
        L = np.asarray(ham_data["chol"]).reshape(-1, self.norb, self.norb)
        ham_data["rot_chol"] = np.einsum("pi,gij->gpj", mo.T.conj(), L, optimize=True)
        return ham_data

    # -- batched (wave_function base dispatch :181-186, :237-244, :366-373) --
    def calc_overlap(self, walkers, wave_data):
        if isinstance(walkers, list):
            return np.array([self.overlap_unrestricted(a, b, wave_data) for a, b in zip(*walkers)])
        return np.array([self.overlap_restricted(w, wave_data) for w in walkers])

    def calc_force_bias(self, walkers, ham_data, wave_data):
        if isinstance(walkers, list):
            return np.array(
                [self.force_bias_unrestricted(a, b, ham_data, wave_data) for a, b in zip(*walkers)]
            )
        return np.array([self.force_bias_restricted(w, ham_data, wave_data) for w in walkers])

    def calc_energy(self, walkers, ham_data, wave_data):
        if isinstance(walkers, list):
            return np.array(
                [self.energy_unrestricted(a, b, ham_data, wave_data) for a, b in zip(*walkers)]
            )
        return np.array([self.energy_restricted(w, ham_data, wave_data) for w in walkers])


@dataclass
class UHFTrial:
    """Unrestricted Hartree-Fock trial; wavefunctions.py:1238-1499."""

    norb: int
    nelec: Tuple[int, int]

    def overlap_unrestricted(self, wu, wd, wave_data):
        """wavefunctions.py:1259-1268."""
        mo = wave_data["mo_coeff"]
        return np.linalg.det(mo[0].T.conj() @ wu) * np.linalg.det(mo[1].T.conj() @ wd)

    def overlap_restricted(self, walker, wave_data):
        """wavefunctions.py:181-186: restricted = unrestricted on column slices."""
        return self.overlap_unrestricted(
            walker[:, : self.nelec[0]], walker[:, : self.nelec[1]], wave_data
        )

    def greens(self, wu, wd, wave_data):
        """wavefunctions.py:1289-1312."""
        mo = wave_data["mo_coeff"]
        return [green(wu, mo[0]), green(wd, mo[1])]

    def force_bias_unrestricted(self, wu, wd, ham_data, wave_data):
        """wavefunctions.py:1314-1329."""
        gu, gd = self.greens(wu, wd, wave_data)
        rc = ham_data["rot_chol"]
        return np.einsum("gij,ij->g", rc[0], gu, optimize=True) + np.einsum(
            "gij,ij->g", rc[1], gd, optimize=True
        )

    def energy_unrestricted(self, wu, wd, ham_data, wave_data):
        """wavefunctions.py:1331-1363."""
        h0, rot_h1, rot_chol = ham_data["h0"], ham_data["rot_h1"], ham_data["rot_chol"]
        gu, gd = self.greens(wu, wd, wave_data)
        ene1 = np.sum(gu * rot_h1[0]) + np.sum(gd * rot_h1[1])
        fu = np.einsum("gij,jk->gik", rot_chol[0], gu.T, optimize=True)
        fd = np.einsum("gij,jk->gik", rot_chol[1], gd.T, optimize=True)
        cu, cd = np.einsum("gii->g", fu), np.einsum("gii->g", fd)
        exu = np.sum(fu * fu.transpose(0, 2, 1))
        exd = np.sum(fd * fd.transpose(0, 2, 1))
        ene2 = (np.sum(cu * cu) + np.sum(cd * cd) + 2.0 * np.sum(cu * cd) - exu - exd) / 2.0
        return ene2 + ene1 + h0

    def rdm1(self, wave_data):
        """wavefunctions.py:1413-1416 (uhf._calc_rdm1)."""
        if "rdm1" in wave_data:
            return np.array(wave_data["rdm1"])
        mo = wave_data["mo_coeff"]
        return np.array([mo[0] @ mo[0].T.conj(), mo[1] @ mo[1].T.conj()])

    def build_measurement_intermediates(self, ham_data, wave_data):
        """wavefunctions.py:1472-1496 (uhf._build_measurement_intermediates)."""
        h1 = np.array(ham_data["h1"], dtype=np.float64)
        h1[0] = (h1[0] + h1[0].T) / 2.0
        h1[1] = (h1[1] + h1[1].T) / 2.0
        ham_data["h1"] = h1
        mo = wave_data["mo_coeff"]
        ham_data["rot_h1"] = [mo[0].T.conj() @ h1[0], mo[1].T.conj() @ h1[1]]
        L = np.asarray(ham_data["chol"]).reshape(-1, self.norb, self.norb)
        ham_data["rot_chol"] = [
            np.einsum("pi,gij->gpj", mo[0].T.conj(), L, optimize=True),
            np.einsum("pi,gij->gpj", mo[1].T.conj(), L, optimize=True),
        ]
        return ham_data

    def calc_overlap(self, walkers, wave_data):
        if isinstance(walkers, list):
            return np.array([self.overlap_unrestricted(a, b, wave_data) for a, b in zip(*walkers)])
        return np.array([self.overlap_restricted(w, wave_data) for w in walkers])

    def calc_force_bias(self, walkers, ham_data, wave_data):
        if isinstance(walkers, list):
            return np.array(
                [self.force_bias_unrestricted(a, b, ham_data, wave_data) for a, b in zip(*walkers)]
            )
        na, nb = self.nelec
        return np.array(
            [self.force_bias_unrestricted(w[:, :na], w[:, :nb], ham_data, wave_data) for w in walkers]
        )

    def calc_energy(self, walkers, ham_data, wave_data):
        if isinstance(walkers, list):
            return np.array(
                [self.energy_unrestricted(a, b, ham_data, wave_data) for a, b in zip(*walkers)]
            )
        na, nb = self.nelec
        return np.array(
            [self.energy_unrestricted(w[:, :na], w[:, :nb], ham_data, wave_data) for w in walkers]
        )


def get_init_walkers(trial, wave_data, n_walkers: int, walker_type: str):
    """wavefunctions.py:427-466: natural orbitals of the trial rdm1 (descending)."""
    rdm1 = trial.rdm1(wave_data)
    na, nb = trial.nelec
    if walker_type == "restricted":
        nat = np.linalg.eigh(rdm1[0] + rdm1[1])[1][:, ::-1]
        return np.array([nat[:, :na] + 0.0j] * n_walkers)
    nat_u = np.linalg.eigh(rdm1[0])[1][:, ::-1][:, :na]
    nat_d = np.linalg.eigh(rdm1[1])[1][:, ::-1][:, :nb]
    return [np.array([nat_u + 0.0j] * n_walkers), np.array([nat_d + 0.0j] * n_walkers)]


# ----------------------------------------------------------------------------
# Walker linear algebra: QR and stochastic reconfiguration
# ----------------------------------------------------------------------------


def qr_restricted(walkers: np.ndarray):
    """linalg_utils.py:51-55: batched Householder QR, norms = prod diag R."""
    qs, norms = [], []
    for w in walkers:
        q, r = np.linalg.qr(w)
        qs.append(q)
        norms.append(np.prod(np.diag(r)))
    return np.array(qs), np.array(norms)


def _csign(z):
    """jnp.sign for complex: z / |z| (0 for 0)."""
    a = np.abs(z)
    return np.where(a == 0, 0.0, z / np.where(a == 0, 1.0, a))


def qr_unrestricted(walkers: List[np.ndarray]):
    """linalg_utils.py:58-72: per-spin QR; column 0 times sign(prod diag R)."""
    q0, n0 = qr_restricted(walkers[0])
    q1, n1 = qr_restricted(walkers[1])
    q0[:, :, 0] = q0[:, :, 0] * _csign(n0).reshape(-1, 1)
    q1[:, :, 0] = q1[:, :, 0] * _csign(n1).reshape(-1, 1)
    return [q0, q1], np.array([np.abs(n0), np.abs(n1)])


def orthogonalize(walkers):
    """walkers.py:159-162 (norms**2) and :264-267 (|norm_up| |norm_dn|)."""
    if isinstance(walkers, list):
        q, n = qr_unrestricted(walkers)
        return q, n[0] * n[1]
    q, n = qr_restricted(walkers)
    return q, n ** 2


def orthonormalize(walkers):
    """walkers.py:155-157 (RHFWalkers) and :260-262 (UHFWalkers)."""
    if isinstance(walkers, list):
        return qr_unrestricted(walkers)[0]
    return qr_restricted(walkers)[0]


def sr_indices(weights: np.ndarray, zeta: float):
    """sr.py:24-34: comb indices, serial cumsum, searchsorted side='left'.

    Returns (indices, new_weights).  Index arithmetic follows the reference
    expression order ``total * (i + zeta) / W``.
    """
    nw = weights.shape[0]
    cum = np.cumsum(np.abs(weights))
    total = cum[-1]
    avg = total / nw
    z = total * (np.arange(nw) + zeta) / nw
    idx = np.searchsorted(cum, z)
    idx = np.minimum(idx, nw - 1)  # JAX gathers clamp out-of-range indices
    return idx, np.ones(nw) * avg


def sr_indices_global(weights: np.ndarray, zeta: float, n_ranks: int = 1):
    """sr.py:93-124 (stochastic_reconfiguration_mpi_restricted), rank 0 part.

    The driver's global reconfiguration uses ``z = (i + zeta) / W / size * total``;
    a different rounding order from the local variant above.
    """
    nw = weights.shape[0] // n_ranks
    cum = np.cumsum(np.abs(weights))
    total = cum[-1]
    avg = total / nw / n_ranks
    idx = np.empty(nw * n_ranks, dtype=np.int64)
    for i in range(nw * n_ranks):
        z = (i + zeta) / nw / n_ranks
        idx[i] = np.searchsorted(cum, z * total)
    idx = np.minimum(idx, nw * n_ranks - 1)
    return idx, np.ones(nw * n_ranks) * avg


def stochastic_reconfiguration(walkers, weights, zeta, mode: str = "local"):
    """walkers.py:139-145/244-250 -> sr.py:24-48 (local) or sr.py:52-153 (global, 1 rank)."""
    if mode == "local":
        idx, w_new = sr_indices(weights, zeta)
    else:
        idx, w_new = sr_indices_global(weights, zeta)
    if isinstance(walkers, list):
        return [walkers[0][idx], walkers[1][idx]], w_new
    return walkers[idx], w_new


# ----------------------------------------------------------------------------
# Propagator
# ----------------------------------------------------------------------------


@dataclass
class Propagator:
    """propagator_afqmc, propagation.py:111-441."""

    dt: float = 0.01
    n_walkers: int = 50
    n_exp_terms: int = 6
    walker_type: str = "restricted"

    def build_propagation_intermediates(self, ham_data, trial, wave_data):
        """propagation.py:378-438."""
        norb = trial.norb
        rdm1 = np.asarray(wave_data["rdm1"])
        rdm1 = rdm1[0] + rdm1[1]
        L = np.asarray(ham_data["chol"]).reshape(-1, norb, norb)
        ham_data["mf_shifts"] = 1.0j * np.einsum("gij,ij->g", L, rdm1)
        ham_data["h0_prop"] = -ham_data["h0"] - np.sum(ham_data["mf_shifts"] ** 2) / 2.0
        na, nb = trial.nelec
        if self.walker_type == "unrestricted":
            ham_data["mf_shifts_fp"] = np.stack(
                (ham_data["mf_shifts"] / na / 2.0, ham_data["mf_shifts"] / nb / 2.0)
            )
            ham_data["h0_prop_fp"] = np.stack(
                (
                    (ham_data["h0_prop"] + ham_data["ene0"]) / na / 2.0,
                    (ham_data["h0_prop"] + ham_data["ene0"]) / nb / 2.0,
                )
            )
        else:
            ham_data["mf_shifts_fp"] = ham_data["mf_shifts"] / 2.0 / na
            ham_data["h0_prop_fp"] = (ham_data["h0_prop"] + ham_data["ene0"]) / na / 2.0
        v0 = 0.5 * np.einsum("gik,gkj->ij", L, L, optimize=True)
        mf_r = (1.0j * ham_data["mf_shifts"]).real
        v1 = np.einsum("g,gik->ik", mf_r, L, optimize=True)
        h1 = np.asarray(ham_data["h1"])
        if self.walker_type == "unrestricted":
            h1_mod = h1 - np.array([v0 + v1, v0 + v1])
            ham_data["exp_h1"] = np.array(
                [
                    scipy.linalg.expm(-self.dt * h1_mod[0] / 2.0),
                    scipy.linalg.expm(-self.dt * h1_mod[1] / 2.0),
                ]
            )
        else:
            h1_mod = (h1[0] + h1[1]) / 2.0 - v0 - v1
            ham_data["exp_h1"] = scipy.linalg.expm(-self.dt * h1_mod / 2.0)
        return ham_data

    def init_prop_data(self, trial, wave_data, ham_data, init_walkers=None):
        """propagation.py:123-152 (the PRNG key is replaced by an injected source)."""
        pd = {}
        pd["weights"] = np.ones(self.n_walkers)
        if init_walkers is not None:
            pd["walkers"] = init_walkers
        else:
            pd["walkers"] = get_init_walkers(trial, wave_data, self.n_walkers, self.walker_type)
        if "e_estimate" in ham_data:
            pd["e_estimate"] = ham_data["e_estimate"]
        else:
            e = np.real(trial.calc_energy(pd["walkers"], ham_data, wave_data))
            pd["e_estimate"] = np.sum(e) / self.n_walkers
        pd["pop_control_ene_shift"] = pd["e_estimate"]
        pd["overlaps"] = trial.calc_overlap(pd["walkers"], wave_data)
        pd["normed_overlaps"] = pd["overlaps"]
        pd["norms"] = np.ones(self.n_walkers) + 0.0j
        return pd

    # propagation.py:154-176
    def apply_trotprop_single_det_vhs(self, walker, vhs, exp_h1):
        walker = exp_h1 @ walker
        fact_recip = np.array([1.0 / math.factorial(n + 1) for n in range(self.n_exp_terms - 1)])
        carry = walker
        powers = []
        for _ in range(1, self.n_exp_terms):
            carry = vhs @ carry  # VHS^n y
            powers.append(carry)
        # jnp.sum(vhs_n_walker * fact_recip, axis=0)
        walker = walker + np.sum(np.array(powers) * fact_recip.reshape(-1, 1, 1), axis=0)
        return exp_h1 @ walker

    def vhs(self, fields_i, chol, norb):
        """propagation.py:196-203: i sqrt(dt) (x @ chol).reshape(N, N)."""
        return 1.0j * np.sqrt(self.dt) * (fields_i @ chol).reshape(norb, norb)

    def apply_trotprop(self, walkers, fields, ham_data, norb):
        """propagation.py:178-272 via walkers.py:115-137.

        The VHS of all walkers is one batched product (the reference vmaps
        ``fields_i @ chol`` over walkers); the complex fields times the real
        ``chol`` are split into two real products."""
        chol = np.asarray(ham_data["chol"])
        W = fields.shape[0]
        vhs = 1.0j * np.sqrt(self.dt) * (fields.real @ chol + 1.0j * (fields.imag @ chol))
        vhs = vhs.reshape(W, norb, norb)
        if isinstance(walkers, list):
            up = [self.apply_trotprop_single_det_vhs(w, v, ham_data["exp_h1"][0])
                  for w, v in zip(walkers[0], vhs)]
            dn = [self.apply_trotprop_single_det_vhs(w, v, ham_data["exp_h1"][1])
                  for w, v in zip(walkers[1], vhs)]
            return [np.array(up), np.array(dn)]
        return np.array([self.apply_trotprop_single_det_vhs(w, v, ham_data["exp_h1"])
                         for w, v in zip(walkers, vhs)])

    def propagate_free(self, trial, ham_data, prop_data, fields, wave_data, zeta):
        """propagation.py:338-376 (zeta injected in place of the key split)."""
        sdt = np.sqrt(self.dt)
        if self.walker_type == "unrestricted":
            shift = np.einsum("wg,sg->sw", fields, ham_data["mf_shifts_fp"])
            const = np.exp(-sdt * shift) * np.exp(self.dt * np.asarray(ham_data["h0_prop_fp"])).reshape(-1, 1)
        else:
            shift = fields @ ham_data["mf_shifts_fp"]
            const = np.exp(-sdt * shift) * np.exp(self.dt * ham_data["h0_prop_fp"])
        w = self.apply_trotprop(prop_data["walkers"], fields, ham_data, trial.norb)
        if isinstance(w, list):
            w = [w[0] * const[0].reshape(-1, 1, 1), w[1] * const[1].reshape(-1, 1, 1)]
        else:
            w = w * const.reshape(-1, 1, 1)
        w, norms = orthogonalize(w)
        prop_data["weights"] = prop_data["weights"] * norms.real
        prop_data["walkers"], prop_data["weights"] = stochastic_reconfiguration(
            w, prop_data["weights"], zeta)
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        return prop_data

    def propagate_constrained(self, trial, ham_data, prop_data, fields, wave_data):
        """propagation.py:274-336."""
        sdt = np.sqrt(self.dt)
        fb = trial.calc_force_bias(prop_data["walkers"], ham_data, wave_data)
        field_shifts = -sdt * (1.0j * fb - ham_data["mf_shifts"])
        shifted = fields - field_shifts
        shift_term = np.sum(shifted * ham_data["mf_shifts"], axis=1)
        fb_term = np.sum(fields * field_shifts - field_shifts * field_shifts / 2.0, axis=1)
        prop_data["walkers"] = self.apply_trotprop(
            prop_data["walkers"], shifted, ham_data, trial.norb
        )
        ov_new = trial.calc_overlap(prop_data["walkers"], wave_data)
        imp = (
            np.exp(
                -sdt * shift_term
                + fb_term
                + self.dt * (prop_data["pop_control_ene_shift"] + ham_data["h0_prop"])
            )
            * ov_new
            / prop_data["overlaps"]
        )
        theta = np.angle(np.exp(-sdt * shift_term) * ov_new / prop_data["overlaps"])
        imp_pl = np.abs(imp) * np.cos(theta)
        imp_pl = np.where(np.isnan(imp_pl), 0.0, imp_pl)
        imp_pl = np.where(imp_pl < 1.0e-3, 0.0, imp_pl)
        imp_pl = np.where(imp_pl > 100.0, 0.0, imp_pl)
        w = imp_pl * prop_data["weights"]
        w = np.where(w > 100.0, 0.0, w)
        prop_data["weights"] = w
        prop_data["pop_control_ene_shift"] = prop_data["e_estimate"] - 0.1 * np.log(
            np.sum(w) / self.n_walkers
        ) / self.dt
        prop_data["overlaps"] = ov_new
        return prop_data


# ----------------------------------------------------------------------------
# Sampler and driver loop
# ----------------------------------------------------------------------------


class InjectedRandom:
    """Deterministic stand-in for the reference's JAX PRNG key stream.

    ``fields`` replaces ``random.normal(subkey, (S, W, G))`` (sampling.py:63-71)
    and ``uniform`` replaces ``random.uniform(subkey)`` (sampling.py:161-163,
    driver.py:163-164).  Draws come from ``numpy.random.default_rng(seed)``.
    """

    def __init__(self, seed: int):
        self.rng = np.random.default_rng(seed)

    def fields(self, n_steps: int, n_walkers: int, n_chol: int) -> np.ndarray:
        return self.rng.standard_normal((n_steps, n_walkers, n_chol))

    def uniform(self) -> float:
        return float(self.rng.random())


@dataclass
class Sampler:
    """sampling.sampler, sampling.py:15-168 and 343-365."""

    n_prop_steps: int = 50
    n_ene_blocks: int = 50
    n_sr_blocks: int = 1
    n_blocks: int = 50

    def block_scan(self, prop, trial, ham_data, prop_data, wave_data, rnd):
        """sampling.py:52-94."""
        n_chol = np.asarray(ham_data["chol"]).shape[0]
        fields = rnd.fields(self.n_prop_steps, prop.n_walkers, n_chol)
        for s in range(self.n_prop_steps):
            prop_data = prop.propagate_constrained(trial, ham_data, prop_data, fields[s], wave_data)
        prop_data["n_killed_walkers"] += prop_data["weights"].size - np.count_nonzero(
            prop_data["weights"]
        )
        prop_data["walkers"] = orthonormalize(prop_data["walkers"])
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        e = np.real(trial.calc_energy(prop_data["walkers"], ham_data, wave_data))
        e = np.where(
            np.abs(e - prop_data["e_estimate"]) > np.sqrt(2.0 / prop.dt), prop_data["e_estimate"], e
        )
        block_weight = np.sum(prop_data["weights"])
        block_energy = np.sum(e * prop_data["weights"]) / block_weight
        prop_data["pop_control_ene_shift"] = (
            0.9 * prop_data["pop_control_ene_shift"] + 0.1 * block_energy
        )
        return prop_data, (block_energy, block_weight)

    def sr_block_scan(self, prop, trial, ham_data, prop_data, wave_data, rnd):
        """sampling.py:146-168."""
        be, bw = [], []
        for _ in range(self.n_ene_blocks):
            prop_data, (e, w) = self.block_scan(prop, trial, ham_data, prop_data, wave_data, rnd)
            be.append(e)
            bw.append(w)
        zeta = rnd.uniform()
        prop_data["walkers"], prop_data["weights"] = stochastic_reconfiguration(
            prop_data["walkers"], prop_data["weights"], zeta
        )
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        return prop_data, (np.array(be), np.array(bw))

    def propagate_phaseless(self, prop, trial, ham_data, prop_data, wave_data, rnd):
        """sampling.py:343-365."""
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        prop_data["n_killed_walkers"] = 0
        prop_data["pop_control_ene_shift"] = prop_data["e_estimate"]
        be, bw = [], []
        for _ in range(self.n_sr_blocks):
            prop_data, (e, w) = self.sr_block_scan(prop, trial, ham_data, prop_data, wave_data, rnd)
            be.append(e)
            bw.append(w)
        be, bw = np.array(be), np.array(bw)
        prop_data["n_killed_walkers"] /= self.n_sr_blocks * self.n_ene_blocks * prop.n_walkers
        return np.sum(be * bw) / np.sum(bw), prop_data


def sampler_propagate_free(sampler, prop, trial, ham_data, prop_data, wave_data, rnd):
    """sampling.py:96-144 (_block_scan_free) over sampling.py:367-384
    (propagate_free): n_blocks blocks of n_prop_steps free steps; per block the
    overlap-weighted energy (clamped against ene0), its weight, sum of overlaps
    and of their moduli.  Returns (ov, abs_ov, block_energy, block_weight)."""
    prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
    n_chol = np.asarray(ham_data["chol"]).shape[0]
    ov, aov, be, bw = [], [], [], []
    for _ in range(sampler.n_blocks):
        fields = rnd.fields(sampler.n_prop_steps, prop.n_walkers, n_chol)
        for s in range(sampler.n_prop_steps):
            prop_data = prop.propagate_free(trial, ham_data, prop_data, fields[s], wave_data, rnd.uniform())
        e = trial.calc_energy(prop_data["walkers"], ham_data, wave_data)
        ene0 = ham_data.get("ene0", 0.0)
        e = np.where(np.abs(e - ene0) > np.sqrt(2.0 / prop.dt), ene0, e)
        o, w = prop_data["overlaps"], prop_data["weights"]
        be.append(np.sum(e * o * w) / np.sum(o * w))
        bw.append(np.sum(o * w))
        ov.append(np.sum(o))
        aov.append(np.sum(np.abs(o)))
    return np.array(ov), np.array(aov), np.array(be), np.array(bw)


class SamplerLNO(Sampler):
    """sampling.sampler_lno, sampling.py:583-694: blocks also average the
    orbital energy; both samples are clamped against pop_control_ene_shift
    (the orbital energy where the total energy is clamped)."""

    def block_scan(self, prop, trial, ham_data, prop_data, wave_data, rnd):
        """sampling.py:586-631."""
        n_chol = np.asarray(ham_data["chol"]).shape[0]
        fields = rnd.fields(self.n_prop_steps, prop.n_walkers, n_chol)
        for s in range(self.n_prop_steps):
            prop_data = prop.propagate_constrained(trial, ham_data, prop_data, fields[s], wave_data)
        prop_data["n_killed_walkers"] += prop_data["weights"].size - np.count_nonzero(
            prop_data["weights"]
        )
        prop_data["walkers"] = orthonormalize(prop_data["walkers"])
        prop_data["overlaps"] = trial.calc_overlap(prop_data["walkers"], wave_data)
        e = np.real(trial.calc_energy(prop_data["walkers"], ham_data, wave_data))
        shift = prop_data["pop_control_ene_shift"]
        clamp = np.abs(e - shift) > np.sqrt(2.0 / prop.dt)
        e = np.where(clamp, shift, e)
        o = np.real(trial.calc_orbenergy(prop_data["walkers"], ham_data, wave_data))
        o = np.where(np.abs(e - shift) > np.sqrt(2.0 / prop.dt), shift, o)
        block_weight = np.sum(prop_data["weights"])
        block_energy = np.sum(e * prop_data["weights"]) / block_weight
        block_orbe = np.sum(o * prop_data["weights"]) / block_weight
        prop_data["pop_control_ene_shift"] = 0.9 * shift + 0.1 * block_energy
        self._orbe.append((block_orbe, block_weight))
        return prop_data, (block_energy, block_weight)

    def propagate_phaseless(self, prop, trial, ham_data, prop_data, wave_data, rnd):
        """sampling.py:663-689: (energy, prop_data, orbital energy)."""
        self._orbe = []
        e, prop_data = super().propagate_phaseless(prop, trial, ham_data, prop_data, wave_data, rnd)
        o = np.array([x[0] for x in self._orbe])
        w = np.array([x[1] for x in self._orbe])
        return e, prop_data, np.sum(o * w) / np.sum(w)


def afqmc_blocks(prop, trial, ham_data, prop_data, wave_data, sampler, rnd, n_blocks):
    """Sampling loop of driver.afqmc_energy, driver.py:133-168, on one rank.

    Returns (block_energies, block_weights, prop_data).  Energies are kept in
    FP64 (the reference casts them to float32 for MPI at driver.py:138-139).
    """
    energies, weights = [], []
    for _ in range(n_blocks):
        e, prop_data = sampler.propagate_phaseless(prop, trial, ham_data, prop_data, wave_data, rnd)
        energies.append(e)
        weights.append(np.sum(prop_data["weights"]))
        prop_data["walkers"] = orthonormalize(prop_data["walkers"])
        zeta = rnd.uniform()
        prop_data["walkers"], prop_data["weights"] = stochastic_reconfiguration(
            prop_data["walkers"], prop_data["weights"], zeta, mode="global"
        )
        prop_data["e_estimate"] = 0.9 * prop_data["e_estimate"] + 0.1 * e
    return np.array(energies), np.array(weights), prop_data


# ----------------------------------------------------------------------------
# stat_utils (host-side; used by the serving stop rule)
# ----------------------------------------------------------------------------


def blocking_analysis(weights, energies, neql=0):
    """stat_utils.py:8-64 (without printing)."""
    n = weights.shape[0] - neql
    weights = weights[neql:]
    energies = energies[neql:]
    we = weights * energies
    mean_energy = we.sum() / weights.sum()
    block_sizes = np.array([1, 2, 5, 10, 20, 50, 100, 200, 300, 400, 500, 1000, 10000])
    prev, plateau, errors = 0.0, None, []
    for i in block_sizes[block_sizes < n / 2.0]:
        nb = int(n // i)
        bw = np.array([weights[j * i : (j + 1) * i].sum() for j in range(nb)])
        be = np.array([we[j * i : (j + 1) * i].sum() for j in range(nb)]) / bw
        v1, v2 = bw.sum(), (bw**2).sum()
        mean = (bw * be).sum() / v1
        err = ((bw * (be - mean) ** 2).sum() / (v1 - v2 / v1) / (nb - 1)) ** 0.5
        errors.append(err)
        if err < 1.05 * prev and plateau is None:
            plateau = max(err, prev)
        prev = err
    if plateau is None and errors:
        plateau = 2 * errors[0]
    return mean_energy, plateau
