"""B200-native (sm_100a) backend for meikey's candidate-key search path.

One fused CUDA kernel runs seed expansion (ChaCha20 or counter), SHA-512 and clamping,
a comb-table fixed-base multiply, pooled Montgomery inversion, compression, base64 and
multi-needle matching; the host confirms every hit.  See include/meikey_b200.h.
"""
from ._lib import (MODE_CONTAINS, MODE_REGEX, MODE_SUFFIX, SEED_CHACHA20, SEED_COUNTER,  # noqa: F401
                   SEED_INCREMENTAL)
from .engine import Context, GpuError, Graph, Job, Needle, Server, search_many  # noqa: F401

__all__ = ["Context", "Job", "Graph", "Server", "Needle", "GpuError", "search_many", "SEED_CHACHA20", "SEED_COUNTER", "SEED_INCREMENTAL", "MODE_CONTAINS",
           "MODE_SUFFIX", "MODE_REGEX"]
