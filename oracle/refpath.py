"""ORACLE (test infrastructure only): where the md.error reference tree is.

The checker builds (oracle/ref/Makefile), the golden-fixture scripts and the
tests that read reference files directly take the tree's location from the
environment variable MDERROR_REFERENCE; when it is unset they look at the
build container's mount point.  Tests skip when the tree is absent (the GPU
boxes carry only the prebuilt checker libraries)."""
import os

ENV = "MDERROR_REFERENCE"
_DEFAULT = "/root/reference"


def reference_root():
    """The reference tree's root, or None when it is not present."""
    p = os.environ.get(ENV, _DEFAULT)
    return p if p and os.path.isdir(p) else None
