"""Location of the reference source tree (test infrastructure only).

The environment variable CHRONOS_REFERENCE_DIR names the reference's source
tree (the ChronosLab checkout whose C++ the oracle recipe compiles and whose
example files some CPU tests read).  When it is unset, the build image's
read-only mount is used if it exists; this function is the only place that
names it.  None means the reference tree is not available (as on a machine
that only runs the prebuilt oracle/_ref libraries): callers skip what needs it.
"""
import os

_IMAGE_MOUNT = "/root/reference"


def reference_dir():
    d = os.environ.get("CHRONOS_REFERENCE_DIR")
    if d:
        return d if os.path.isdir(d) else None
    return _IMAGE_MOUNT if os.path.isdir(_IMAGE_MOUNT) else None


def reference_file(*parts):
    """Path of a file inside the reference tree, or None if it is not there."""
    d = reference_dir()
    if d is None:
        return None
    p = os.path.join(d, *parts)
    return p if os.path.exists(p) else None
