"""B200-native solver for the BFPn pencil-beam per-depth-step hot path.

The numerical work runs in hand-written sm_100a CUDA kernels behind the C ABI
of include/bfpn_capi.h (lib/libbfpn_b200.so); this package holds the kernels
(csrc/), the ctypes binding (capi) and the reference-style run configuration
(config).
"""
from . import capi, config  # noqa: F401
from .capi import Context, BfpnError, read_tables, footprint_bytes  # noqa: F401
from .config import parse_args, make_config, RunConfig  # noqa: F401

__all__ = ["capi", "config", "Context", "BfpnError", "read_tables", "footprint_bytes", "parse_args",
           "make_config", "RunConfig"]
