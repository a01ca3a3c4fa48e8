"""Host-side Python binding of libcb200 (the B200 explicit residual-and-update path of COREFL)."""
from . import abi, cases, field
from .lib import CB2Error, Context, load

__all__ = ["abi", "cases", "field", "Context", "CB2Error", "load"]
