"""Loader of the native extension.

The product path has no CPU fallback: if the compiled library is missing the
import fails loudly, telling the user how to build it.
"""

from __future__ import annotations

try:
    from . import _gs2g as lib  # noqa: F401  (pybind11 binding of include/gs2g.h)
except ImportError as e:  # pragma: no cover - exercised only on a broken install
    raise ImportError(
        "gpusim2grid_b200: the native library is not built "
        "(run `python gpusim2grid_b200/_build.py`): " + str(e)) from e

from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgs2g.so"

__all__ = ["lib", "LIB_PATH"]
