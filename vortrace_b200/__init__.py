"""vortrace_b200 -- exact ray walks through Voronoi meshes on NVIDIA B200.

Drop-in for the reference's ``vortrace`` projection path
(``vortrace.ProjectionCloud``); the work runs in libvortrace_b200.so, a C-ABI
library of hand-written sm_100a kernels, called through ctypes.
"""
import logging

from . import grid
from .vortrace import ProjectionCloud

__version__ = "0.1.0"


def set_verbose(verbose: bool) -> None:
    """Enable or disable status messages on stdout (the reference's
    ``vortrace.set_verbose``)."""
    from . import _lib
    _lib.load().vt_set_verbose(int(bool(verbose)))


def get_verbose() -> bool:
    """Return the current verbose setting."""
    from . import _lib
    return bool(_lib.load().vt_get_verbose())


logging.getLogger("vortrace").addHandler(logging.NullHandler())

__all__ = ["ProjectionCloud", "grid", "set_verbose", "get_verbose", "__version__"]
