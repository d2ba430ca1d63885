"""3dpipe_b200: a B200-native (sm_100a) rebuild of 3DPipe's spatial-join hot path.

The package directory name starts with a digit, so import it with
``importlib.import_module("3dpipe_b200")``.  The compute path is the in-tree
CUDA library libtdp.so (C ABI in include/tdp.h); this package only binds it.
"""
from . import tdp  # noqa: F401
from . import shard  # noqa: F401
from .tdp import Context, TdpError, FORM_PLAIN, FORM_TUNED, QUERY_NN, QUERY_WITHIN  # noqa: F401
