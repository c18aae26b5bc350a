"""Calibration: GRAPPA shift table and the GROG interpolator (GPU)."""

from ._grappa import KernelTable, grappa_power, lstsq, prepare_grappa_table, train_grappa  # noqa: F401
from ._autotune import autotune_gridder  # noqa: F401
from ._grog import BrickPlan, GrogInterpolator, GrogPlan  # noqa: F401

__all__ = [
    "GrogInterpolator",
    "autotune_gridder",
    "GrogPlan",
    "BrickPlan",
    "KernelTable",
    "grappa_power",
    "lstsq",
    "prepare_grappa_table",
    "train_grappa",
]
