"""mdforce: B200 (sm_100a) molecular-dynamics force path of md.error.

Host-side mirror of the reference's interaction-engine API over the C ABI of
libmdforce.so (include/mdforce.h).  Importing fails loudly when the native
library is missing; there is no CPU fallback.
"""
from ._lib import lib, LIB_PATH, EXPORTED  # noqa: F401
from .core import *  # noqa: F401,F403
from . import systems  # noqa: F401
from . import topology  # noqa: F401
from . import optibasis  # noqa: F401

__version__ = lib.md_version().decode()
