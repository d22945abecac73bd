"""gpusim2grid_b200: a B200-native batched Newton–Raphson AC power flow.

Drop-in for the bare ``[pvpq | pq]`` Newton–Raphson path of gpusim2grid
(array-tuple mode): ``acpf_nr_gpu``, ``AcPfGPU``, ``ContingencyAnalysisGPU``,
``InjectionSweepGPU`` and ``ScenarioSweepGPU``, plus ``compute_many`` (rows of
several grids in one launch).  Python calls a pybind11
binding of the C-ABI in ``include/gs2g.h``; the C++ host code drives one
persistent sm_100a kernel.  There is no CPU fallback: importing this package
fails if the native library is not built.
"""

from ._common import AcPfTimings, BatchTimings, RowStatus  # noqa: F401
from ._native import lib as _lib  # noqa: F401
from .acpf_nr import AcPfGPU, acpf_nr_gpu  # noqa: F401
from .batch import ContingencyAnalysisGPU, InjectionSweepGPU, ScenarioSweepGPU, compute_many  # noqa: F401

__version__ = "0.1.0"

__all__ = ["AcPfGPU", "acpf_nr_gpu", "ContingencyAnalysisGPU", "InjectionSweepGPU", "ScenarioSweepGPU",
           "compute_many", "RowStatus", "AcPfTimings", "BatchTimings"]
