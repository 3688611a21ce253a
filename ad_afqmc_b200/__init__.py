"""B200 (sm_100a) phaseless-AFQMC walker path behind the ad_afqmc interfaces.

Modules mirror the reference package: ``wavefunctions`` (rhf, uhf),
``propagation`` (propagator_afqmc), ``walkers`` (RHFWalkers, UHFWalkers),
``sampling`` (sampler), ``hamiltonian``, ``driver`` and ``stat_utils``.  The
numerical work runs in ``lib/libafqmc_b200.so`` (hand-written CUDA, C ABI in
``include/afqmc_b200.h``); there is no CPU fallback.
"""

__version__ = "0.1.0"

from . import _lib  # noqa: F401
