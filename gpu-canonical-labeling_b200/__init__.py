"""B200-native individualization-refinement canonical labeling.

Import as ``importlib.import_module("gpu-canonical-labeling_b200")``.  The
package exposes the graph model and arena (``graphs``) and the binding of
the CUDA library's C ABI (``api``).
"""
from . import graphs  # noqa: F401
from .api import (  # noqa: F401
    BatchResult, CanonResult, Context, GclError, Nauty_Parallel, Server, canon, canon_batch,
    default_context, is_isomorphic, load_library,
)
