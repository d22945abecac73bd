"""Shared pieces of the facades: row status, precision / device / scheduling
parsing, timings, and array-tuple normalisation.

Mirrors ``src/gpusim2grid/contingency_analysis/_scheduling.py`` (RowStatus,
scheduling names) and the device parsing of the reference's facades.
"""

from __future__ import annotations

import dataclasses
from enum import IntEnum

import numpy as np
import scipy.sparse as sp

from ._native import lib

__all__ = ["RowStatus", "AcPfTimings", "BatchTimings", "normalize_device", "resolve_precision",
           "resolve_scheduling", "grid_arrays", "default_tol"]


class RowStatus(IntEnum):
    """Outcome of one row of a batched solve (``get_row_status()``), the
    reference's ``RowStatus`` (``contingency_analysis/_scheduling.py:61-79``)."""
    CONVERGED = 0       # ||F||inf < tol
    MAX_ITER = 1        # budget used, residual finite but >= tol
    DIVERGED = 2        # residual not finite
    NOT_SIMULATED = 3   # dropped by the islanding pre-check, never solved


_PRECISION = {"fp64": lib.PREC_FP64, "mixed": lib.PREC_MIXED, "fp32": lib.PREC_MIXED, None: lib.PREC_FP64}


def resolve_precision(precision):
    """'fp64' (J/LU in FP64) or 'mixed' (J/LU in FP32, mismatch and V in FP64).
    'fp32' is accepted as the reference's name for its FP32 build and maps to
    'mixed': the mismatch and the voltages always stay FP64 here, so the
    default tol stays 1e-8."""
    if precision not in _PRECISION:
        raise ValueError(f"Unknown precision {precision!r}. Choose from: ['fp64', 'mixed']")
    return _PRECISION[precision]


def default_tol():
    """Per unit.  1e-8: the mismatch is evaluated in FP64 in both precisions."""
    return 1e-8


_SCHEDULING = ("chunked", "continuous")


def resolve_scheduling(value):
    """'chunked': every row runs exactly ``nb_iter`` Newton steps, then its
    residual is evaluated (the reference's default).  'continuous': a row
    leaves as soon as ``residual < tol`` or its budget is used."""
    if value not in _SCHEDULING:
        raise ValueError(f"Unknown scheduling {value!r}. Choose from: {list(_SCHEDULING)}")
    return value


def normalize_device(device):
    """None / int / 'cuda' / 'cuda:N' -> CUDA device index (-1 = current)."""
    if device is None:
        return -1
    if isinstance(device, (int, np.integer)):
        return int(device)
    if isinstance(device, str):
        if device == "cuda":
            return -1
        if device.startswith("cuda:"):
            return int(device.split(":", 1)[1])
    if hasattr(device, "type") and getattr(device, "type") == "cuda":
        return -1 if device.index is None else int(device.index)
    raise ValueError(f"Unsupported device {device!r}")


def grid_arrays(grid):
    """Validate and normalise the array tuple ``(Ybus, Vinit, Sbus, slack_ids,
    slack_weights, pv, pq)``.  Returns a dict of canonical arrays."""
    if not isinstance(grid, (tuple, list)) or len(grid) != 7:
        raise ValueError("grid must be the array tuple (Ybus, Vinit, Sbus, slack_ids, slack_weights, pv, pq); "
                         "lightsim2grid grid objects are not accepted (pass their array tuple)")
    Ybus, Vinit, Sbus, slack_ids, slack_weights, pv, pq = grid
    Y = sp.csr_matrix(Ybus, dtype=np.complex128)
    Y.sum_duplicates()
    Y.sort_indices()
    n = Y.shape[0]
    if Y.shape != (n, n):
        raise ValueError("Ybus must be square")
    V = np.ascontiguousarray(Vinit, dtype=np.complex128).reshape(-1)
    S = np.ascontiguousarray(Sbus, dtype=np.complex128).reshape(-1)
    if V.size != n or S.size != n:
        raise ValueError("Vinit and Sbus must have n_bus entries")
    return dict(Ybus=Y, n_bus=n, Vinit=V, Sbus=S,
                slack=np.asarray(slack_ids, dtype=np.int32).reshape(-1),
                slack_weights=np.asarray(slack_weights, dtype=np.float64).reshape(-1),
                pv=np.ascontiguousarray(pv, dtype=np.int32).reshape(-1),
                pq=np.ascontiguousarray(pq, dtype=np.int32).reshape(-1))


def make_session(d, device, tail_policy=1):
    Y = d["Ybus"]
    return lib.Session(normalize_device(device), d["n_bus"], Y.indptr.astype(np.int32),
                       Y.indices.astype(np.int32), Y.data, d["Vinit"], d["Sbus"], d["pv"], d["pq"],
                       tail_policy)


@dataclasses.dataclass
class AcPfTimings:
    """Timings of one single-system solve (the reference's ``AcPfTimings``,
    ``src/_cpp/timing_utils.hpp:131-215``; phase split in ``phase_share``)."""
    converged: bool = False
    nb_iter: int = 0
    residual: float = float("nan")
    t_plan_ms: float = 0.0
    t_kernel_ms: float = 0.0
    t_total_ms: float = 0.0

    def to_dict(self):
        return dataclasses.asdict(self)


@dataclasses.dataclass
class BatchTimings:
    """Timings of one batched run (the reference's ``BatchTimings``,
    ``src/_cpp/timing_utils.hpp:348-560``)."""
    n_rows: int = 0
    total_iters: int = 0
    t_plan_ms: float = 0.0
    t_upload_ms: float = 0.0
    t_kernel_ms: float = 0.0
    t_total_ms: float = 0.0
    phase_share: tuple = ()

    def to_dict(self):
        return dataclasses.asdict(self)
