"""Where the reference checkout lies (test infrastructure only).

The environment variable ZERORK_REFERENCE names it; without it the
container's mount point /root/reference is used.  Only the oracle build
recipe, the fixture generators under tests/golden and the CPU tests that
compare against the reference library read it; nothing under zerork_b200/
does, and the GPU tests run from committed fixtures alone.
"""
import os

REFERENCE = os.environ.get("ZERORK_REFERENCE", "/root/reference")
REF_DATA = os.path.join(REFERENCE, "data", "mechanisms")


def available():
    return os.path.isdir(os.path.join(REFERENCE, "src", "zerork"))
