"""cupyram_b200: B200-native split-step Pade parabolic-equation engine.

Drop-in for clapeyre/cupyram's public API (``cupyram/__init__.py``):
``CuPyRAM``, ``compute_pade_coefficients`` and ``AsyncBatcher``.
"""
from .cupyram import CuPyRAM
from .pade import compute_pade_coefficients, compute_pade_coefficients_batch
from .batching import AsyncBatcher

__version__ = "0.1.0"
__all__ = ["CuPyRAM", "compute_pade_coefficients", "AsyncBatcher"]
