"""Location of the reference's source checkout (TEST INFRASTRUCTURE).

The CPU oracle (oracle/_ref, built by oracle/Makefile) and the host data-model test compile the
reference's own sources where they lie. Their location is read from the environment variable
FOCALORS_REFERENCE; when it is unset, the checkout location of the build container is used. Nothing
at run time on a GPU machine reads the sources: only the built oracle library travels.
"""
from __future__ import annotations

import os

_DEFAULT = "/root/reference"


def reference_dir() -> str:
    return os.environ.get("FOCALORS_REFERENCE", _DEFAULT)


def available() -> bool:
    return os.path.isdir(os.path.join(reference_dir(), "pe", "poisson"))
