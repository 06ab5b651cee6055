"""B200-native individualization-refinement canonical labeling.

Import as ``importlib.import_module("gpu-canonical-labeling_b200")``.  The
package exposes the graph model and arena (``graphs``) and the binding of
the CUDA library's C ABI (``api``).
"""
import os as _os

# The serving loop (api.Server) runs about a dozen CUDA streams; the default
# of 8 hardware work queues makes streams share queues, so a short batch can
# wait behind a long search issued on another stream.  Effective only if
# CUDA has not started in this process yet.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import graphs  # noqa: E402,F401
from .api import (  # noqa: E402,F401
    BatchResult, CanonResult, Context, GclError, Nauty_Parallel, Server, canon, canon_batch,
    default_context, group_order, is_isomorphic, load_library, perm_group_order,
)
