"""Oracle for the cudaPIC hot path: CPU restatement (C) of every reference
kernel plus FP64 eduPIC references, loaded through ctypes.

Test infrastructure only: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product package ``cudapic_b200``
never imports it.
"""
from .pyoracle import *  # noqa: F401,F403
