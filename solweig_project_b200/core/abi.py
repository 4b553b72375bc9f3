"""Buffer view (reference solweig_core/abi.py:87-365): a borrowed, optionally
frozen view of a host array with its logical placement."""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

from .status import (AbiValidationError, NonContiguousError, RefusalReason, StaleBufferError, TypedRefusal)

RESIDENCY_CPU = "cpu"


@dataclass
class ArrayView:
    owner: np.ndarray
    dtype: str
    shape: tuple
    strides: tuple
    global_origin: tuple = (0, 0)
    logical_domain_id: str = ""
    residency: str = RESIDENCY_CPU
    read_only: bool = False
    _digest: str | None = None

    @classmethod
    def from_numpy(cls, arr, *, global_origin=(0, 0), logical_domain_id="", freeze=False):
        if not isinstance(arr, np.ndarray):
            raise AbiValidationError(TypedRefusal(RefusalReason.ABI_INVALID, "owner must be a numpy array"))
        view = cls(owner=arr, dtype=arr.dtype.str, shape=tuple(arr.shape), strides=tuple(arr.strides),
                   global_origin=tuple(global_origin), logical_domain_id=logical_domain_id, read_only=freeze)
        if freeze:
            view._digest = hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()
        return view

    def require_contiguous(self) -> np.ndarray:
        if not self.owner.flags.c_contiguous:
            raise NonContiguousError(TypedRefusal(RefusalReason.NON_CONTIGUOUS,
                                                  "strided buffer handed to a contiguous consumer",
                                                  {"strides": list(self.strides)}))
        return self.owner

    def to_contiguous(self) -> np.ndarray:
        return np.ascontiguousarray(self.owner)

    def assert_not_mutated(self) -> None:
        if self._digest is None:
            return
        if hashlib.sha256(np.ascontiguousarray(self.owner).tobytes()).hexdigest() != self._digest:
            raise StaleBufferError(TypedRefusal(RefusalReason.STALE_BUFFER,
                                                "frozen view's owner was mutated after the view was lent",
                                                {"logical_domain_id": self.logical_domain_id}))
