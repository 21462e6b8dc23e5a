"""liteqg_b200: LiteQG's quantized-graph query path on one NVIDIA B200.

``liteqg_b200.symphonyqg.Index`` is the drop-in for the reference's
``symphonyqg.Index``; ``include/lqg.h`` is the C ABI beneath it.
"""
from . import symphonyqg
from .symphonyqg import Index

__all__ = ["Index", "symphonyqg"]
