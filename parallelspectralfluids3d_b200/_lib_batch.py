"""ctypes declarations of the batched and serving entry points (``include/psf/batch.h``)."""

from __future__ import annotations


def declare(L) -> None:
    """Set argument/result types of the batch symbols that the build exports."""
    return None
