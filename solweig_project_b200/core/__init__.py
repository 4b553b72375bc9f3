"""Typed request / dispatch / buffer-view seam (the solweig_core interface).

Mirrors ``solweig_core`` of the reference (request.py, abi.py, dispatch.py,
status.py): a solve is DECLARED for a device and resolved explicitly; the
``cuda`` device resolves to this library's exact chain, and nothing is ever
re-targeted silently (there is no CPU backend here).
"""
from .status import (AbiValidationError, DispatchBlockedError, DispatchStatus, FallbackReason,  # noqa: F401
                     NonContiguousError, RefusalReason, RequestValidationError, SolweigCoreError,
                     StaleBufferError, TypedRefusal)
from .request import PhysicalWindow, SolveRequestView, TimeCoverage  # noqa: F401
from .abi import ArrayView  # noqa: F401
from .dispatch import DispatchPlan, DispatchResult, resolve, supported_devices  # noqa: F401
