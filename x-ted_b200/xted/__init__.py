"""xted: B200-native unit-cost tree edit distance (host side).

The compute path is the CUDA library ``lib/libxted.so`` behind the C ABI in
``include/xted.h``; this package binds it with ctypes and mirrors the
reference's interface (``standard_ted``, the dataset parsers).
"""
from . import gen, trees  # noqa: F401
from ._lib import (ORIENT_AUTO, ORIENT_LEFT, ORIENT_RIGHT, XTED_EAGAIN, XTED_ECUDA,  # noqa: F401
                   XTED_EINVAL, XTED_ENODEV, XTED_FAULT_HOLD_PAIR, XTED_ENOMEM, XTED_ENOTFOUND, XTED_ETIMEOUT, XTED_ETOOBIG,
                   XTED_MAX_NODES, LIB_PATH, XtedError)
from .api import Context, default_context, distance_noalloc, pair_cells, standard_ted, validate  # noqa: F401
from .trees import Tree, from_adjacency, from_parent, load_pair, node_process, pre_process  # noqa: F401
