"""B200-native implementation of Cortado's progressive error-bounded float32
encode/decode path (store, init_send, init_recv, resi_send, resi_recv), with
the reference's stream, .stor and .stor.meta formats.

The compute path is libcortado.so (hand-written sm_100a kernels behind the C
ABI in include/cortado.h); this package holds its Python binding
(``ops.Codec``), the host-side storage/bound logic (``storage``) and the
synthetic field generators used by tests and benchmarks (``fields``).
"""
from . import storage  # noqa: F401

__all__ = ["storage", "ops", "fields"]
