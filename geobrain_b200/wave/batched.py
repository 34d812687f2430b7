"""Batched propagation of many models (placeholder until the batched engine lands)."""
from __future__ import annotations


class AcousticBatch:  # pragma: no cover - filled in with the batched engine
    pass


def acoustic_forward_batched(*args, **kwargs):  # pragma: no cover
    raise NotImplementedError
