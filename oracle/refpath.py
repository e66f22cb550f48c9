"""Where the checkers look for the reference project's sources and data
(TEST INFRASTRUCTURE ONLY: the recipes under oracle/, the fixture scripts and
the tests read the reference tree; the product never does).

One setting: the GD_REFERENCE environment variable, the root of the
reference project (the folder holding src/ and data/).  When it is unset, the
recipes use REF_DEFAULT, the read-only mount point of the reference tree on
the development machine; oracle/Makefile's REF has the same default.  Where
neither holds the sources (for example on a machine that only runs the GPU
tests), reference_sources() is None and the tests that need them skip.
"""

from __future__ import annotations

import os
from pathlib import Path

REF_DEFAULT = "/root/reference"


def reference_path() -> Path:
    """The configured reference root, whether or not it exists."""
    return Path(os.environ.get("GD_REFERENCE") or REF_DEFAULT)


def reference_sources() -> Path | None:
    """The reference root if its src/ and data/ folders are present, else None."""
    p = reference_path()
    return p if (p / "src").is_dir() and (p / "data").is_dir() else None
