"""Generate the golden known-answer fixture for the trial measurements.

The reference pins its RHF/UHF overlap, Green's function, force bias and
energy with values asserted in ``tests/test_wavefunctions.py:128-184``.  Those
values were produced from inputs drawn with ``np.random.seed(102)`` in the
fixed order of ``tests/test_wavefunctions.py:12-86``:

  1. RHF walker  = rand(10,5) + 1j*rand(10,5)
  2. h0          = rand(1)[0]
  3. rot_h1      = rand(5,10)
  4. rot_chol    = rand(5,5,10)        (nchol, nocc, norb)
  5. h1          = rand(10,10)
  6. chol        = rand(5,10,10)
  7. UHF mo_coeff = [rand(10,3), rand(10,2)]
  8. UHF walkers = rand(10,3)+1j*rand(10,3), rand(10,2)+1j*rand(10,2)

The RHF trial is the identity's first 5 columns; the UHF test slices
``rot_h1[:na]``, ``rot_chol[:, :na]`` (and likewise for the beta spin).

Running this script writes ``trial_golden.npz`` (inputs) and
``trial_golden.json`` (the reference's asserted values, copied as numbers
with their source lines).  It needs only NumPy.
"""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Values asserted by the reference test-suite (tests/test_wavefunctions.py).
REFERENCE_VALUES = {
    "rhf_overlap_real": [-0.10794844182417201, "tests/test_wavefunctions.py:128-130"],
    "rhf_green_sum_real": [12.181348093111438, "tests/test_wavefunctions.py:133-136"],
    "rhf_force_bias_sum_real": [66.13455680423321, "tests/test_wavefunctions.py:139-142"],
    "rhf_energy_real": [217.79874063608622, "tests/test_wavefunctions.py:145-147"],
    "uhf_overlap_real": [-0.4029825074695857, "tests/test_wavefunctions.py:157-159"],
    "uhf_green_sum_real": [3.6324117896217394, "tests/test_wavefunctions.py:162-169"],
    "uhf_force_bias_sum_real": [10.441272099672341, "tests/test_wavefunctions.py:172-175"],
    "uhf_energy_real": [-1.7203463308366032, "tests/test_wavefunctions.py:178-186"],
}


def build_inputs():
    np.random.seed(102)
    norb, no, nchol = 10, 5, 5
    walker = np.random.rand(norb, no) + 1.0j * np.random.rand(norb, no)
    h0 = np.random.rand(1)[0]
    rot_h1 = np.random.rand(no, norb)
    rot_chol = np.random.rand(nchol, no, norb)
    h1 = np.random.rand(norb, norb)
    chol = np.random.rand(nchol, norb, norb)
    mo_u0 = np.random.rand(norb, 3)
    mo_u1 = np.random.rand(norb, 2)
    wu = np.random.rand(norb, 3) + 1.0j * np.random.rand(norb, 3)
    wd = np.random.rand(norb, 2) + 1.0j * np.random.rand(norb, 2)
    return dict(
        walker=walker, h0=np.array(h0), rot_h1=rot_h1, rot_chol=rot_chol, h1=h1,
        chol=chol, mo_coeff=np.eye(norb)[:, :no], mo_u0=mo_u0, mo_u1=mo_u1,
        walker_up=wu, walker_dn=wd,
    )


def main():
    inputs = build_inputs()
    np.savez(os.path.join(HERE, "trial_golden.npz"), **inputs)
    with open(os.path.join(HERE, "trial_golden.json"), "w") as f:
        json.dump(REFERENCE_VALUES, f, indent=1)


if __name__ == "__main__":
    main()
