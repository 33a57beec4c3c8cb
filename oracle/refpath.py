"""Test infrastructure: where the reference's sources are mounted.

The one place that names the default location; the environment variable
DELTA_RAY_REFERENCE overrides it.  Only the oracle's build recipe (through
__graft_entry__.build), the loader tests and the fixture scripts read it; the
product never does, and neither does anything that runs on a GPU box.
"""
import os

DEFAULT = "/root/reference"


def reference_dir():
    return os.environ.get("DELTA_RAY_REFERENCE", DEFAULT)
