"""nnm: B200-native k-NN graph construction, merge and search.

The compute runs in lib/libnnm.so (hand-written sm_100a CUDA behind the C ABI
of include/nnm.h); this package is the Python host side.
"""
from . import datasets  # noqa: F401
from ._lib import Context, Index, NnmError, entry_init, load, make_opts, mlp_init  # noqa: F401
