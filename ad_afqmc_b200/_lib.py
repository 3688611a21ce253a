"""ctypes binding of libafqmc_b200.so (the C ABI in include/afqmc_b200.h).

The library is required: importing the walker-path classes without it, or
calling them without a CUDA device, raises.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import torch

_PKG = os.path.dirname(os.path.abspath(__file__))
# AFQ_CHECKS=1 selects the debug build (python -m ad_afqmc_b200.build --checks)
LIB_PATH = os.path.join(_PKG, "lib", "libafqmc_b200_checks.so" if os.environ.get("AFQ_CHECKS") == "1"
                        else "libafqmc_b200.so")

AFQ_OK = 0
AFQ_ERR_TIMEOUT = 8
AFQ_ERR_BOUNDS = 9
AFQ_RESTRICTED, AFQ_UNRESTRICTED = 0, 1
AFQ_TRIAL_RHF, AFQ_TRIAL_UHF = 0, 1
AFQ_FP64, AFQ_MIXED, AFQ_MIXED_HI = 0, 1, 2
AFQ_SR_LOCAL, AFQ_SR_GLOBAL = 0, 1

_dp = C.POINTER(C.c_double)


class afq_dims(C.Structure):
    _fields_ = [
        ("norb", C.c_int32),
        ("nocc", C.c_int32 * 2),
        ("nchol", C.c_int32),
        ("nwalkers", C.c_int32),
        ("walker_type", C.c_int32),
        ("trial_type", C.c_int32),
        ("n_exp_terms", C.c_int32),
        ("precision", C.c_int32),
        ("reserved", C.c_int32),
        ("dt", C.c_double),
    ]


class afq_ham(C.Structure):
    _fields_ = [
        ("mo", C.c_void_p * 2),
        ("rot_h1", C.c_void_p * 2),
        ("rot_chol", C.c_void_p * 2),
        ("chol", C.c_void_p),
        ("exp_h1", C.c_void_p * 2),
        ("mf_shifts", C.c_void_p),
        ("h0", C.c_double),
        ("h0_prop", C.c_double * 2),
    ]


class afq_state(C.Structure):
    _fields_ = [
        ("walkers", C.c_void_p * 2),
        ("weights", C.c_void_p),
        ("overlaps", C.c_void_p),
        ("scalars", C.c_void_p),
        ("flags", C.c_int32),
        ("reserved", C.c_int32),
    ]


AFQ_STATE_GREEN_CURRENT = 1


class afq_tuning(C.Structure):
    """Tile/schedule record of one problem shape (0 = built-in heuristic)."""
    _fields_ = [
        ("fb_splitk", C.c_int32),
        ("fb_bn", C.c_int32),
        ("vhs_bn", C.c_int32),
        ("exch_bn", C.c_int32),
        ("f64_exch_bn", C.c_int32),
        ("max_stages", C.c_int32),
        ("grid_cap", C.c_int32),
        ("prop_epi_groups", C.c_int32),
        ("prop_order", C.c_int32),
        ("prop_chunk", C.c_int32),
        ("qr_mode", C.c_int32),
        ("vhs_chunk", C.c_int32),
        ("prop_bn", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]

    KNOBS = ("fb_splitk", "fb_bn", "vhs_bn", "exch_bn", "f64_exch_bn", "max_stages", "grid_cap",
             "prop_epi_groups", "prop_order", "prop_chunk", "qr_mode", "vhs_chunk", "prop_bn")

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k in self.KNOBS}

    @classmethod
    def from_dict(cls, d: dict) -> "afq_tuning":
        t = cls()
        for k, v in d.items():
            setattr(t, k, int(v))
        return t


class AfqError(RuntimeError):
    pass


_lib: Optional[C.CDLL] = None

_SIGS = {
    "afq_version": ([], C.c_int),
    "afq_status_string": ([C.c_int], C.c_char_p),
    "afq_prepared_size": ([C.POINTER(afq_dims), C.POINTER(C.c_size_t)], C.c_int),
    "afq_workspace_size": ([C.POINTER(afq_dims), C.POINTER(C.c_size_t)], C.c_int),
    "afq_small_workspace_size": ([C.POINTER(afq_dims), C.POINTER(C.c_size_t)], C.c_int),
    "afq_prepare": ([C.POINTER(afq_dims), C.POINTER(afq_ham), C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_calc_overlap": ([C.POINTER(afq_dims), C.c_void_p * 2, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_calc_overlap_static": ([C.POINTER(afq_dims), C.c_void_p * 2, C.c_void_p * 2, C.c_void_p, C.c_void_p], C.c_int),
    "afq_calc_green": ([C.POINTER(afq_dims), C.c_void_p * 2, C.c_void_p * 2, C.c_void_p * 2, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_calc_force_bias": ([C.POINTER(afq_dims), C.c_void_p, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_calc_energy": ([C.POINTER(afq_dims), C.c_void_p, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_propagate_constrained": ([C.POINTER(afq_dims), C.c_void_p, C.POINTER(afq_state), C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_orthonormalize": ([C.POINTER(afq_dims), C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_stochastic_reconfiguration": ([C.POINTER(afq_dims), C.c_void_p, C.c_double, C.c_int, C.c_void_p * 2, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "afq_block_end": ([C.POINTER(afq_dims), C.c_void_p, C.POINTER(afq_state), C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_normal_fields": ([C.c_void_p, C.c_int64, C.c_uint64, C.c_uint64, C.c_void_p], C.c_int),
    "afq_split_bf16": ([C.c_void_p, C.c_int64, C.c_int, C.c_void_p * 3, C.c_void_p], C.c_int),
    "afq_gemm_split_bf16": ([C.c_void_p * 3, C.c_int, C.c_void_p * 3, C.c_int, C.c_int, C.c_void_p,
                             C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64,
                             C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p], C.c_int),
    "afq_stochastic_reconfiguration_dev": ([C.POINTER(afq_dims), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p * 2, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "afq_normal_fields_dev": ([C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p, C.c_void_p], C.c_int),
    "afq_uniform_dev": ([C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p], C.c_int),
    "afq_apply_trotprop": ([C.POINTER(afq_dims), C.c_void_p, C.c_void_p * 2, C.c_void_p, C.c_void_p, C.c_size_t,
                            C.c_void_p], C.c_int),
    "afq_calc_orbenergy": ([C.POINTER(afq_dims), C.c_void_p, C.c_void_p * 2, C.c_void_p, C.c_int32, C.c_void_p,
                            C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_comb_indices_ranks": ([C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                C.c_void_p], C.c_int),
    "afq_set_tuning": ([C.POINTER(afq_dims), C.c_void_p], C.c_int),
    "afq_get_tuning": ([C.POINTER(afq_dims), C.POINTER(afq_tuning)], C.c_int),
    "afq_batch_table_size": ([C.c_int32, C.c_void_p, C.POINTER(C.c_size_t)], C.c_int),
    "afq_batch_create": ([C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                          C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)], C.c_int),
    "afq_batch_propagate_constrained": ([C.c_void_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int),
    "afq_batch_destroy": ([C.c_void_p], C.c_int),
    "afq_intermediates_workspace_size": ([C.c_int32, C.c_int32, C.POINTER(C.c_size_t)], C.c_int),
    "afq_measurement_intermediates": ([C.c_int32, C.c_int32 * 2, C.c_int32, C.c_int32, C.c_void_p * 2,
                                       C.c_void_p, C.c_void_p, C.c_void_p * 2, C.c_void_p * 2, C.c_void_p,
                                       C.c_size_t, C.c_void_p], C.c_int),
    "afq_propagation_intermediates": ([C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_expm": ([C.c_int32, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p],
                 C.c_int),
    "afq_eigh_desc": ([C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p],
                      C.c_int),
    "afq_natural_orbitals_workspace_size": ([C.c_int32, C.c_int32, C.POINTER(C.c_size_t)], C.c_int),
    "afq_natural_orbitals": ([C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_size_t, C.c_void_p], C.c_int),
    "afq_check_status": ([C.POINTER(afq_dims), C.c_void_p, C.c_size_t, C.c_void_p], C.c_int),
    "afq_status_flag": ([C.POINTER(afq_dims), C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)], C.c_int),
    "afq_test_wait_timeout": ([C.POINTER(afq_dims), C.c_void_p, C.c_size_t, C.c_uint32, C.c_void_p],
                              C.c_int),
    "afq_launch_count": ([C.c_int, C.POINTER(C.c_ulonglong)], C.c_int),
    "afq_profile_begin": ([C.c_int], C.c_int),
    "afq_profile_end": ([C.POINTER(C.c_double), C.POINTER(C.c_int)], C.c_int),
}

KERNEL_IDS = {"green": 0, "fb": 1, "prep": 2, "vhs": 3, "prop": 4, "exchange": 5, "ecomb": 6,
              "weights": 7, "qr": 8, "sr": 9, "gather": 10, "block_end": 11, "normal": 12,
              "misc": 13}


def launch_count(kernel: Optional[str] = None) -> int:
    c = C.c_ulonglong()
    kid = -1 if kernel is None else KERNEL_IDS[kernel]
    check(lib().afq_launch_count(kid, C.byref(c)), "afq_launch_count")
    return int(c.value)


def profile_begin(kernel: str) -> None:
    check(lib().afq_profile_begin(KERNEL_IDS[kernel]), "afq_profile_begin")


def profile_end():
    ms, n = C.c_double(), C.c_int()
    check(lib().afq_profile_end(C.byref(ms), C.byref(n)), "afq_profile_end")
    return float(ms.value), int(n.value)

EXPORTED = tuple(_SIGS)


def lib() -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AfqError(
                f"{LIB_PATH} is missing: build it with `python -m ad_afqmc_b200.build` "
                "(the walker path has no CPU fallback)"
            )
        l = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(l, name)
            f.argtypes = args
            f.restype = res
        _lib = l
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != AFQ_OK:
        msg = lib().afq_status_string(rc).decode()
        raise AfqError(f"{what}: {msg} (status {rc})")


def require_cuda(t: torch.Tensor, name: str = "tensor") -> None:
    if not t.is_cuda:
        raise AfqError(f"{name} must be a CUDA tensor (the walker path has no CPU fallback)")
    if not t.is_contiguous():
        raise AfqError(f"{name} must be contiguous")


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    if t is None:
        return None
    return t.data_ptr()


def pair(a, b=None):
    arr = (C.c_void_p * 2)()
    arr[0] = a
    arr[1] = b
    return arr


def stream_handle(stream: Optional[torch.cuda.Stream] = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def triple(a=None, b=None, c=None):
    arr = (C.c_void_p * 3)()
    arr[0], arr[1], arr[2] = a, b, c
    return arr


def split_bf16(x: torch.Tensor, npieces: int):
    """bf16 pieces of a float64 CUDA tensor (same shape each)."""
    x = x.contiguous()
    outs = [torch.empty(x.shape, dtype=torch.bfloat16, device=x.device) for _ in range(npieces)]
    ptrs = triple(*[o.data_ptr() for o in outs])
    check(lib().afq_split_bf16(x.data_ptr(), x.numel(), npieces, ptrs, stream_handle()), "afq_split_bf16")
    return outs


BF16X3 = ((0, 0), (0, 1), (1, 0))
BF16X6 = ((0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0))


def gemm_split_bf16(a_pieces, b_pieces, pairs, out=None):
    """C[b] = sum_pairs A_i[b] @ B_j[b]^T for (batch, rows, K) bf16 pieces."""
    a0, b0 = a_pieces[0], b_pieces[0]
    if a0.dim() == 2:
        a_pieces = [a.unsqueeze(0) for a in a_pieces]
        b_pieces = [b.unsqueeze(0) for b in b_pieces]
        a0, b0 = a_pieces[0], b_pieces[0]
        squeeze = True
    else:
        squeeze = False
    batch, M, K = a0.shape
    N = b0.shape[1]
    if out is None:
        out = torch.empty(batch, M, N, dtype=torch.float32, device=a0.device)
    pr = torch.tensor([v for p in pairs for v in p], dtype=torch.int32)
    err = torch.zeros(1, dtype=torch.int32, device=a0.device)
    rc = lib().afq_gemm_split_bf16(
        triple(*[a.data_ptr() for a in a_pieces]), len(a_pieces),
        triple(*[b.data_ptr() for b in b_pieces]), len(b_pieces), len(pairs),
        pr.data_ptr(), M, N, K, batch, a0.stride(1), a0.stride(0), b0.stride(1), b0.stride(0),
        out.data_ptr(), out.stride(1), out.stride(0), err.data_ptr(), stream_handle())
    check(rc, "afq_gemm_split_bf16")
    if int(err.item()) != 0:
        raise AfqError("afq_gemm_split_bf16: a device wait timed out")
    return out[0] if squeeze else out


def make_dims(norb, nocc, nchol, nwalkers, walker_type, trial_type, n_exp_terms, precision, dt):
    d = afq_dims()
    d.norb = int(norb)
    d.nocc[0] = int(nocc[0])
    d.nocc[1] = int(nocc[1])
    d.nchol = int(nchol)
    d.nwalkers = int(nwalkers)
    d.walker_type = int(walker_type)
    d.trial_type = int(trial_type)
    d.n_exp_terms = int(n_exp_terms)
    d.precision = int(precision)
    d.reserved = 0
    d.dt = float(dt)
    return d


def set_tuning(d: afq_dims, t: Optional[afq_tuning]) -> None:
    """Register `t` for every call with dims equal to `d` (None removes it)."""
    check(lib().afq_set_tuning(C.byref(d), C.cast(C.byref(t), C.c_void_p) if t is not None else None),
          "afq_set_tuning")


def get_tuning(d: afq_dims) -> afq_tuning:
    t = afq_tuning()
    check(lib().afq_get_tuning(C.byref(d), C.byref(t)), "afq_get_tuning")
    return t


def sizes(d: afq_dims):
    p, w = C.c_size_t(), C.c_size_t()
    check(lib().afq_prepared_size(C.byref(d), C.byref(p)), "afq_prepared_size")
    check(lib().afq_workspace_size(C.byref(d), C.byref(w)), "afq_workspace_size")
    return p.value, w.value
