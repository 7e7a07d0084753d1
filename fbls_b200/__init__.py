"""fbls_b200: the FBLS search hot path (fold, doubled prefix sums, template
scan, evidence) as hand-written CUDA for the B200 (sm_100a) behind a C ABI.

Importing the package does not touch the GPU; the compute entry points load
the in-tree native library and fail loudly when it is missing.
"""
from .config import SearchConfig  # noqa: F401

__all__ = ["SearchConfig", "api", "synth"]
__version__ = "0.1.0"
