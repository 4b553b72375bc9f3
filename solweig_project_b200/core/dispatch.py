"""Explicit device/backend resolution (reference solweig_core/dispatch.py:45-191).

Backends are keyed by the DECLARED device, never by probing: a ``cuda``
request resolves to this library's exact chain; a ``cpu`` request is
BLOCKED (this library has no CPU backend and never substitutes one)."""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any

from .request import SolveRequestView
from .status import DispatchBlockedError, DispatchStatus, FallbackReason, RefusalReason, TypedRefusal

BACKEND_EXACT_CHAIN = "b200-exact-chain"
_BACKENDS: dict[str, tuple[str, ...]] = {
    "cpu": (),
    "cuda": (BACKEND_EXACT_CHAIN,),
}


@dataclass(frozen=True)
class DispatchPlan:
    device: str
    backend: str
    profile_id: str
    logical_domain_id: str
    fallback_reason: FallbackReason | None = None
    status: DispatchStatus = DispatchStatus.READY

    def describe(self) -> dict[str, Any]:
        return {"device": self.device, "backend": self.backend, "profile_id": self.profile_id,
                "logical_domain_id": self.logical_domain_id,
                "fallback_reason": self.fallback_reason.value if self.fallback_reason else None,
                "status": self.status.value}


@dataclass(frozen=True)
class DispatchResult:
    status: DispatchStatus
    plan: DispatchPlan | None = None
    refusal: TypedRefusal | None = None

    @property
    def ready(self) -> bool:
        return self.status is DispatchStatus.READY

    def raise_if_blocked(self) -> DispatchPlan:
        if self.status is not DispatchStatus.READY or self.plan is None:
            raise DispatchBlockedError(self.refusal or TypedRefusal(RefusalReason.UNKNOWN_BACKEND, "dispatch blocked"))
        return self.plan


def supported_devices() -> tuple[str, ...]:
    return tuple(sorted(_BACKENDS))


def resolve(request: SolveRequestView, prefer_backend: str | None = None) -> DispatchResult:
    request.validate()
    if request.device not in _BACKENDS:
        return DispatchResult(DispatchStatus.BLOCKED, refusal=TypedRefusal(
            RefusalReason.UNSUPPORTED_DEVICE, f"device {request.device!r} is outside {sorted(_BACKENDS)}",
            {"device": request.device}))
    backends = _BACKENDS[request.device]
    if not backends:
        return DispatchResult(DispatchStatus.BLOCKED, refusal=TypedRefusal(
            RefusalReason.UNSUPPORTED_DEVICE,
            "device 'cpu' was declared but this library only provides the CUDA exact chain; refusing loudly "
            "instead of substituting another backend", {"device": request.device}))
    backend = backends[0]
    if prefer_backend is not None:
        if prefer_backend not in backends:
            return DispatchResult(DispatchStatus.BLOCKED, refusal=TypedRefusal(
                RefusalReason.UNKNOWN_BACKEND, f"backend {prefer_backend!r} is not registered for "
                f"{request.device!r}", {"device": request.device, "backend": prefer_backend}))
        backend = prefer_backend
    return DispatchResult(DispatchStatus.READY, plan=DispatchPlan(
        device=request.device, backend=backend, profile_id=request.profile_id,
        logical_domain_id=request.logical_domain_id))
