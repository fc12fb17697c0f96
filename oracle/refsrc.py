"""Where the reference tree is read from (test infrastructure only).

The reference's sources are needed only to build its CPU copy
(oracle/ref_cpu/build_ref.sh) and to regenerate the golden fixtures; both
read the tree named by the environment variable DYNAMAP_REFERENCE, whose
default is given here and in build_ref.sh.  Boxes without the tree skip
those steps.
"""
from __future__ import annotations

import os

DEFAULT = "/root/reference"


def reference_root() -> str:
    return os.environ.get("DYNAMAP_REFERENCE", DEFAULT)


def present() -> bool:
    return os.path.isdir(os.path.join(reference_root(), "include"))
