"""Hamiltonian wrapper (mirror of ad_afqmc/hamiltonian.py:12-84)."""

from __future__ import annotations

from dataclasses import dataclass

import torch

from ._engine import drop_engines, to_dev


@dataclass
class hamiltonian:
    norb: int

    def rotate_orbs(self, ham_data: dict, mo_coeff) -> dict:
        """hamiltonian.py:23-46: h1 -> C^T h1 C, L_g -> C^T L_g C (device GEMMs)."""
        c = to_dev(mo_coeff)
        h1 = to_dev(ham_data["h1"])
        ham_data["h1"] = torch.stack([c.T @ h1[0] @ c, c.T @ h1[1] @ c])
        L = to_dev(ham_data["chol"]).reshape(-1, self.norb, self.norb)
        ham_data["chol"] = torch.matmul(torch.matmul(c.T, L), c).reshape(-1, self.norb * self.norb).contiguous()
        drop_engines(ham_data)
        return ham_data

    def build_measurement_intermediates(self, ham_data: dict, trial, wave_data: dict) -> dict:
        """hamiltonian.py:48-63."""
        return trial._build_measurement_intermediates(ham_data, wave_data)

    def build_propagation_intermediates(self, ham_data: dict, prop, trial, wave_data: dict) -> dict:
        """hamiltonian.py:65-81."""
        return prop._build_propagation_intermediates(ham_data, trial, wave_data)

    def __hash__(self) -> int:
        return hash(self.norb)
