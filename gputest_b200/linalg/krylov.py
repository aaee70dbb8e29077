"""Krylov solves on the device: Jacobi-BiCGSTAB and AMG-PCG behind the reference's result type.

``KrylovInfo`` is ``flowtrace/linalg/krylov.py:14-18``. The solves themselves are single
cooperative kernels of ``libb2simplec.so`` (``b2s_bicgstab_jacobi_d``, ``b2s_pcg_amg_d``)
that keep the iteration and its stopping tests on the device and write their outcome to a
device ``b2s_solve_info`` record; ``read_info`` turns such records into ``KrylovInfo``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from .. import _lib

INFO_DTYPE = np.dtype([("iterations", np.int32), ("converged", np.int32), ("residual", np.float64)])


@dataclass
class KrylovInfo:
    iterations: int
    residual: float  # final relative residual
    converged: bool


def info_buffer(k: int, device):
    """Device storage for k b2s_solve_info records."""
    import torch

    return torch.zeros(k * INFO_DTYPE.itemsize, dtype=torch.uint8, device=device)


def read_info(raw) -> List[KrylovInfo]:
    """KrylovInfo list from b2s_solve_info bytes (a host numpy uint8 array or a tensor)."""
    a = raw.cpu().numpy() if hasattr(raw, "cpu") else np.asarray(raw)
    rec = np.frombuffer(a.tobytes(), dtype=INFO_DTYPE)
    return [KrylovInfo(int(r["iterations"]), float(r["residual"]), bool(r["converged"])) for r in rec]


def bicgstab_jacobi(rowptr, col, val, b, x0, inv_diag, tol=0.1, maxiter=30, relative_to_initial=True, stream=None):
    """Jacobi-preconditioned BiCGSTAB (``flowtrace/linalg/krylov.py:68-121``) on one matrix and
    1..3 right-hand sides: b and x0 are [k][n] (or [n]), inv_diag [n]. Returns (x, [KrylovInfo])."""
    import torch

    single = b.dim() == 1
    B = b.reshape(1, -1) if single else b
    k, n = B.shape
    x = x0.reshape(k, n).clone().contiguous().double()
    L = _lib.lib()
    nbytes = L.b2s_bicgstab_workspace_bytes(n, k)
    work = torch.empty(nbytes // 8 + 1, dtype=torch.float64, device=b.device)
    info = info_buffer(k, b.device)
    _lib.check(L.b2s_bicgstab_jacobi_d(n, k, rowptr.data_ptr(), col.data_ptr(), val.data_ptr(),
                                       B.contiguous().double().data_ptr(), inv_diag.contiguous().double().data_ptr(),
                                       x.data_ptr(), float(tol), int(maxiter), int(bool(relative_to_initial)),
                                       work.data_ptr(), work.numel() * 8, info.data_ptr(), _lib.stream_ptr(stream)),
               "b2s_bicgstab_jacobi_d")
    infos = read_info(info)
    return (x[0] if single else x), infos
