"""Refusal / fallback vocabulary and typed errors (reference solweig_core/status.py:21-172)."""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from typing import Any


class RefusalReason(str, Enum):
    CUDA_UNAVAILABLE = "cuda_unavailable"
    UNSUPPORTED_DEVICE = "unsupported_device"
    ABI_INVALID = "abi_invalid"
    REQUEST_INVALID = "request_invalid"
    STALE_BUFFER = "stale_buffer"
    UNKNOWN_BACKEND = "unknown_backend"
    NON_CONTIGUOUS = "non_contiguous"


class FallbackReason(str, Enum):
    LEGACY_ROUNDTRIP = "legacy_roundtrip"
    FULL_TILE_UNSAFE_LOCAL = "full_tile_unsafe_local"
    KERNEL_REFUSED = "kernel_refused"


class DispatchStatus(str, Enum):
    READY = "ready"
    BLOCKED = "blocked"


@dataclass(frozen=True)
class TypedRefusal:
    reason: RefusalReason
    detail: str = ""
    context: dict[str, Any] | None = None

    def to_dict(self) -> dict[str, Any]:
        return {"reason": self.reason.value, "detail": self.detail,
                "context": dict(self.context) if self.context else None}

    def __str__(self) -> str:
        ctx = f" context={self.context}" if self.context else ""
        return f"TypedRefusal({self.reason.value}: {self.detail}{ctx})"


class SolweigCoreError(RuntimeError):
    """Base class of the typed errors."""


class _WithRefusal(SolweigCoreError):
    def __init__(self, refusal: TypedRefusal) -> None:
        super().__init__(str(refusal))
        self.refusal = refusal


class AbiError(SolweigCoreError):
    """A buffer view violated the buffer ABI."""


class AbiValidationError(_WithRefusal, AbiError):
    pass


class StaleBufferError(_WithRefusal, AbiError):
    pass


class NonContiguousError(_WithRefusal, AbiError):
    pass


class RequestValidationError(_WithRefusal):
    pass


class DispatchBlockedError(_WithRefusal):
    pass
