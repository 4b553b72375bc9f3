"""Typed solve request (reference solweig_core/request.py:29-259)."""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Mapping

import numpy as np

from .status import RefusalReason, RequestValidationError, TypedRefusal

DEFAULT_DTYPE_PLAN = {"dsm": "float32", "trees": "float32", "dem": "float32", "walls": "float32",
                      "aspect": "float32", "landcover": "float32"}
DEFAULT_OUTPUT_DTYPE_PLAN = {"utci": "float32", "tmrt": "float32", "shadow": "float32"}


def _refusal(detail, context=None):
    return RequestValidationError(TypedRefusal(RefusalReason.REQUEST_INVALID, detail, context))


@dataclass(frozen=True)
class PhysicalWindow:
    """Half-open (row0, row1, col0, col1) window of the logical domain."""

    row0: int
    row1: int
    col0: int
    col1: int

    def validate(self, *, rows, cols, label="window"):
        if not (0 <= self.row0 < self.row1 <= rows and 0 <= self.col0 < self.col1 <= cols):
            raise _refusal(f"{label} {self.list()} escapes the ({rows}, {cols}) grid or is empty",
                           {label: self.list()})

    def contains(self, other: "PhysicalWindow") -> bool:
        return (self.row0 <= other.row0 and other.row1 <= self.row1 and self.col0 <= other.col0
                and other.col1 <= self.col1)

    def list(self):
        return [self.row0, self.row1, self.col0, self.col1]


@dataclass(frozen=True)
class TimeCoverage:
    time_start: int
    time_stop: int
    total_steps: int

    def validate(self):
        if not 0 <= int(self.time_start) < int(self.time_stop):
            raise _refusal(f"time range [{self.time_start}, {self.time_stop}) is empty or negative",
                           {"time": [self.time_start, self.time_stop]})
        if int(self.time_stop) > int(self.total_steps):
            raise _refusal(f"time_stop {self.time_stop} exceeds the forcing series ({self.total_steps} global "
                           "timesteps)", {"time": [self.time_start, self.time_stop]})

    @property
    def global_indices(self):
        return tuple(range(int(self.time_start), int(self.time_stop)))


@dataclass(frozen=True)
class SolveRequestView:
    """Everything needed to route one window solve; the device is declared."""

    logical_domain_id: str
    rows: int
    cols: int
    origin_x_m: float
    origin_y_m: float
    pixel_size_m: float
    read_window: PhysicalWindow
    write_window: PhysicalWindow
    time: TimeCoverage
    requested_variables: tuple = ("utci", "tmrt", "shadow")
    dtype_plan: Mapping[str, str] = field(default_factory=lambda: dict(DEFAULT_DTYPE_PLAN))
    output_dtype_plan: Mapping[str, str] = field(default_factory=lambda: dict(DEFAULT_OUTPUT_DTYPE_PLAN))
    profile_id: str = ""
    device: str = "cuda"

    def validate(self) -> None:
        if not isinstance(self.logical_domain_id, str) or not self.logical_domain_id:
            raise _refusal("logical_domain_id must be a non-empty string")
        if self.rows <= 0 or self.cols <= 0:
            raise _refusal(f"logical domain shape ({self.rows}, {self.cols}) is empty")
        if not (self.pixel_size_m > 0.0):
            raise _refusal(f"pixel_size_m must be positive, got {self.pixel_size_m!r}")
        self.read_window.validate(rows=self.rows, cols=self.cols, label="read window")
        self.write_window.validate(rows=self.rows, cols=self.cols, label="write window")
        if not self.read_window.contains(self.write_window):
            raise _refusal(f"write window {self.write_window} is not contained in the read window "
                           f"{self.read_window}", {"read": self.read_window.list(), "write": self.write_window.list()})
        self.time.validate()
        if not self.requested_variables:
            raise _refusal("requested_variables must be non-empty")
        for name, plan in (("dtype_plan", self.dtype_plan), ("output_dtype_plan", self.output_dtype_plan)):
            for plane, dt in dict(plan).items():
                try:
                    np.dtype(dt)
                except TypeError as err:
                    raise _refusal(f"{name}[{plane!r}] = {dt!r} is not a numpy dtype") from err
        if not self.profile_id:
            raise _refusal("profile_id is required")
        if self.device not in ("cpu", "cuda"):
            raise _refusal(f"device {self.device!r} is outside the request vocabulary ('cpu' or 'cuda')")

    def describe(self) -> dict[str, Any]:
        return {"logical_domain_id": self.logical_domain_id, "rows": self.rows, "cols": self.cols,
                "pixel_size_m": self.pixel_size_m, "read_window": self.read_window.list(),
                "write_window": self.write_window.list(), "time_start": self.time.time_start,
                "time_stop": self.time.time_stop, "total_steps": self.time.total_steps,
                "requested_variables": list(self.requested_variables), "profile_id": self.profile_id,
                "device": self.device}
