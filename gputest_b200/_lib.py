"""ctypes binding of ``libb2simplec.so`` (the C ABI declared in ``include/b2simplec.h``).

The library is the only compute path: there is no CPU fallback. ``lib()`` raises when the
shared library is missing or stale, and ``require_device()`` raises when no CUDA device is
visible, so that a product call never silently runs anything else.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "csrc", "libb2simplec.so")
ABI_VERSION = 5

B2S_OK = 0
_ERRORS = {-1: "invalid argument", -2: "kernel launch failed", -3: "work space too small", -4: "no usable CUDA device",
           -5: "problem larger than the fixed capacity"}

P = ctypes.c_void_p
I32, I64, F64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double


class Mesh(ctypes.Structure):
    _fields_ = [("nc", I32), ("nf", I32), ("nb", I32), ("dim", I32), ("nnz", I32)] + [
        (name, P) for name in ("fP", "fN", "forig", "own_ptr", "nei_ptr", "nei_face", "bP", "bptr", "w", "alpha", "wl",
                               "S", "d", "Tv", "dxm", "dPf", "dNf", "alpha_b", "wlb", "Sb_mag", "Sb", "db", "nbv",
                               "dbt", "vol", "Ginv", "rowptr", "col", "slot_diag", "slot_PN", "slot_NP")] + [
        ("tiles", P), ("ntiles", I32), ("pad_", I32)]


class TeamConfig(ctypes.Structure):
    """``b2s_team_config``: the thread-block cluster that solves one case of a batch."""
    _fields_ = [("cluster_blocks", I32), ("block_threads", I32), ("wide_row", I32), ("pad_", I32)]


class BC(ctypes.Structure):
    _fields_ = [(name, P) for name in ("m_wall", "m_inlet", "m_pres", "m_sym", "m_dirvel", "ub_fixed", "pb_fixed",
                                       "m_tfix", "m_tflux", "m_out", "tval")]


class FlowParams(ctypes.Structure):
    _fields_ = [("rho", F64), ("mu", F64), ("relax_u", F64), ("relax_p", F64), ("body", F64 * 3),
                ("simplec", I32), ("second_order", I32), ("singular_p", I32), ("pad", I32),
                ("relax_u_cell", P), ("relax_p_cell", P), ("simplec_cell", P)]


class SST(ctypes.Structure):
    """``b2s_sst``: constants and set-up arrays of the k-omega SST model."""
    _fields_ = [(name, F64) for name in ("rho", "mu", "nu", "k_min", "w_min", "relax_k", "relax_w", "k_over_cp", "eb",
                                         "cmu25", "g1", "g2")] + [("second_order", I32), ("pad_", I32)] + [
        (name, P) for name in ("y", "y_wall", "yb", "kb_in", "wb_in")]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", I32), ("converged", I32), ("residual", F64)]


MAX_LEVELS = 20


class AmgLevel(ctypes.Structure):
    _fields_ = [("n", I32), ("nnz", I32), ("nc", I32), ("p_nnz", I32), ("w_nnz", I32)] + [
        (name, P) for name in ("rowptr", "col", "val", "diag_slot", "dinv", "agg", "tval", "x0", "p_rowptr", "p_col",
                               "p_val", "r_rowptr", "r_col", "r_from_p", "r_val", "w_rowptr", "w_col", "w_val", "rho",
                               "strong", "group_ptr", "p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te",
                               "c_ts")] + [("c_nnz", I32), ("pad_", I32)]


class Amg32(ctypes.Structure):
    """Float copies of the hierarchy's per-level values (``b2s_amg_f32``)."""
    _fields_ = [(name, P * MAX_LEVELS) for name in ("val", "dinv", "p_val", "r_val")]


class Amg(ctypes.Structure):
    _fields_ = [("nlevels", I32), ("coarse_n", I32), ("singular", I32), ("sweeps", I32), ("omega", F64),
                ("coarse_rowptr", P), ("coarse_col", P), ("coarse_val", P), ("coarse_inv", P),
                ("ngroups", I32), ("pad_", I32), ("coarse_group_ptr", P), ("coarse_inv_off", P), ("group_singular", P),
                ("levels", AmgLevel * MAX_LEVELS)]


_SIGS = {
    "b2s_abi_version": ([], ctypes.c_int),
    "b2s_device_sm_count": ([], ctypes.c_int),
    "b2s_part_blocks": ([I32], ctypes.c_int),
    "b2s_face_interp_d": ([P, ctypes.c_int, P, P, P], ctypes.c_int),
    "b2s_ls_gradient_d": ([P, ctypes.c_int, P, P, P, P], ctypes.c_int),
    "b2s_gg_gradient_d": ([P, P, P, P, P, P], ctypes.c_int),
    "b2s_assemble_d": ([P, P, P, P, P, P], ctypes.c_int),
    "b2s_spmv_d": ([I32, ctypes.c_int, P, P, P, P, P, P], ctypes.c_int),
    "b2s_bicgstab_workspace_bytes": ([I32, ctypes.c_int], I64),
    "b2s_bicgstab_jacobi_d": ([I32, ctypes.c_int, P, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, P, I64, P, P],
                              ctypes.c_int),
    "b2s_flow_bvals_d": ([P, P, P, P, P, P, P], ctypes.c_int),
    "b2s_momentum_assemble_d": ([P] * 18 + [P], ctypes.c_int),
    "b2s_pressure_assemble_d": ([P] * 14 + [P], ctypes.c_int),
    "b2s_correct_d": ([P] * 15 + [P], ctypes.c_int),
    "b2s_remove_mean_d": ([I32, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P], ctypes.c_int),
    "b2s_sum_partials_d": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P], ctypes.c_int),
    "b2s_energy_bvals_d": ([P, P, P, P, P, P, P], ctypes.c_int),
    "b2s_energy_assemble_d": ([P, P, F64, F64, F64, ctypes.c_int] + [P] * 12 + [P], ctypes.c_int),
    "b2s_face_geometry_d": ([I32, I32, P, P, P, P, P, P, P], ctypes.c_int),
    "b2s_host_geometry": ([I32, I32, I32, P, P, P, P, P, I32, P, P, P, P, P], ctypes.c_int),
    "b2s_host_face_geometry": ([I32, I32, P, P, P, P, P], ctypes.c_int),
    "b2s_cell_geometry_d": ([I32, I32, I32] + [P] * 12 + [P], ctypes.c_int),
    "b2s_fv_faces_d": ([I32, I32, P, P, P, I32, P, P] + [P] * 19 + [P], ctypes.c_int),
    "b2s_ls_matrices_d": ([I32, I32] + [P] * 13 + [P], ctypes.c_int),
    "b2s_amg_workspace_bytes": ([P], I64),
    "b2s_amg_rebuild_d": ([P, P, I64, P], ctypes.c_int),
    "b2s_pcg_workspace_bytes": ([P], I64),
    "b2s_pcg_set_launch": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "b2s_pcg_amg_d": ([P, I32, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, P, I64, P, P], ctypes.c_int),
    "b2s_amg_vcycle_d": ([P, P, P, P, I64, P], ctypes.c_int),
    "b2s_host_aggregate": ([I64, P, P, P], I64),
    "b2s_amg_strength_changes_d": ([P, F64, P, P], ctypes.c_int),
    "b2s_amg_level_strength_changes_d": ([P, F64, P, P], ctypes.c_int),
    "b2s_amg_strength_d": ([I32, P, P, P, P, F64, P, P], ctypes.c_int),
    "b2s_csr_transpose_slots_d": ([I32, P, P, I32, P, P, P], ctypes.c_int),
    "b2s_amg_aggregate_workspace_bytes": ([I32, I64], I64),
    "b2s_amg_aggregate_d": ([I32, P, P, P, P, P, P, P, P, P, P, I64, P], ctypes.c_int),
    "b2s_amg_level_workspace_bytes": ([P], I64),
    "b2s_amg_level_rebuild_d": ([P, P, P, P, P, I64, P], ctypes.c_int),
    "b2s_amg_coarse_inverse_d": ([P, P, I64, P], ctypes.c_int),
    "b2s_amg_p_pattern_d": ([I32, I32, P, P, P, I32, P, P, I64, P, P, P, I64, P, P], ctypes.c_int),
    "b2s_amg_w_pattern_d": ([I32, I32, P, P, P, P, I32, P, P, P, P, I64, I64, P, P, P, P, P, P], ctypes.c_int),
    "b2s_amg_pattern_warp_cols": ([I32], ctypes.c_int),
    "b2s_amg_r_workspace_bytes": ([I32], I64),
    "b2s_amg_r_pattern_d": ([I32, I32, P, P, I64, P, P, P, P, I64, P, P], ctypes.c_int),
    "b2s_amg_c_pattern_d": ([I32, P, P, P, P, I32, P, P, P, P, I64, I64, P, P, P, P, P, P, P], ctypes.c_int),
    "b2s_scan_workspace_bytes": ([I32], I64),
    "b2s_scan_counts_d": ([I32, P, P, P, I64, P], ctypes.c_int),
    "b2s_row_residuals_d": ([I32, P, P, P, P, P, P, P, P, P, P], ctypes.c_int),
    "b2s_flux_balance_d": ([P, P, P, P, P, P], ctypes.c_int),
    "b2s_matrix_properties_workspace_bytes": ([], I64),
    "b2s_matrix_properties_d": ([P, P, P, I64, P, P], ctypes.c_int),
    "b2s_bicgstab_jacobi_noalloc_d": ([I32, ctypes.c_int, P, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, P, P],
                                      ctypes.c_int),
    # mixed precision
    "b2s_momentum_assemble_mixed_d": ([P] * 16 + [P], ctypes.c_int),
    "b2s_pressure_assemble_mixed_d": ([P] * 14 + [P], ctypes.c_int),
    "b2s_energy_assemble_mixed_d": ([P, P, F64, F64, F64, ctypes.c_int] + [P] * 10 + [P], ctypes.c_int),
    "b2s_bicgstab_f32_workspace_bytes": ([I32, ctypes.c_int], I64),
    "b2s_bicgstab_jacobi_f32_d": ([I32, ctypes.c_int, P, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   P, P, P, I64, P, P], ctypes.c_int),
    "b2s_amg_to_f32_d": ([P, P, P], ctypes.c_int),
    "b2s_pcg_mixed_workspace_bytes": ([P], I64),
    "b2s_pcg_amg_mixed_d": ([P, P, P, P, P, I32, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, ctypes.c_int, F64, P,
                             I64, P, P], ctypes.c_int),
    # batches
    "b2s_mesh_part_blocks": ([P], ctypes.c_int),
    "b2s_group_sums_d": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P], ctypes.c_int),
    "b2s_remove_group_means_d": ([P, P, P, ctypes.c_int, ctypes.c_int, P, P, P, P, P], ctypes.c_int),
    "b2s_bicgstab_groups_workspace_bytes": ([I32, ctypes.c_int, ctypes.c_int], I64),
    "b2s_bicgstab_groups_f32_d": ([ctypes.c_int, P, P, I32, ctypes.c_int, P, P, P, P, P, P, F64, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, P, P, P, I64, P, P, P], ctypes.c_int),
    "b2s_pcg_groups_workspace_bytes": ([P], I64),
    "b2s_residual_vjp_d": ([P, P, F64, F64, F64, ctypes.c_int] + [P] * 18 + [P], ctypes.c_int),
    # k-omega SST
    "b2s_momentum_assemble_turb_d": ([P] * 21 + [P], ctypes.c_int),
    "b2s_momentum_assemble_mixed_turb_d": ([P] * 19 + [P], ctypes.c_int),
    "b2s_energy_assemble_mixed_turb_d": ([P, P, P, P, F64, F64, ctypes.c_int] + [P] * 10 + [P], ctypes.c_int),
    "b2s_energy_assemble_turb_d": ([P, P, P, P, F64, F64, ctypes.c_int] + [P] * 12 + [P], ctypes.c_int),
    "b2s_sst_part_blocks": ([P], ctypes.c_int),
    "b2s_sst_momentum_terms_d": ([P] * 12 + [P], ctypes.c_int),
    "b2s_sst_bvals_d": ([P] * 7 + [P], ctypes.c_int),
    "b2s_sst_sources_d": ([P] * 7 + [P], ctypes.c_int),
    "b2s_sst_transport_assemble_d": ([P, P, ctypes.c_int] + [P] * 11 + [P], ctypes.c_int),
    "b2s_sst_transport_finish_d": ([P, P, ctypes.c_int] + [P] * 9 + [P], ctypes.c_int),
    "b2s_sst_update_d": ([P] * 6 + [P], ctypes.c_int),
    "b2s_pcg_groups_mixed_d": ([P, P, P, P, P, P, P, I32, P, P, P, P, P, F64, ctypes.c_int, ctypes.c_int, F64, P, I64,
                                P, P, P], ctypes.c_int),
}

_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """The loaded library; raises RuntimeError if it is missing or has another ABI version."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m gputest_b200.csrc.build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes, fn.restype = args, res
    if L.b2s_abi_version() != ABI_VERSION:
        raise RuntimeError(f"stale {LIB_PATH}: ABI {L.b2s_abi_version()}, expected {ABI_VERSION}")
    _lib = L
    return L


def require_device():
    """The CUDA device the solver runs on; raises when none is visible (no CPU fallback)."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("gputest_b200 needs a CUDA device (sm_100a); none is visible and there is no CPU fallback")
    lib()
    return torch.device("cuda", torch.cuda.current_device())


def check(rc: int, what: str) -> None:
    if rc != B2S_OK:
        raise RuntimeError(f"{what} failed: {_ERRORS.get(rc, rc)} (status {rc})")


def ptr(t) -> Optional[int]:
    """Device pointer of a tensor (None for None)."""
    return None if t is None else t.data_ptr()


def stream_ptr(stream=None) -> Optional[int]:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None
